"""Generate the golden fixtures in this folder from the reference itself.

Run once, in a container where the reference checkout is present:

    python tests/golden/make_golden.py <reference checkout>
    (or set SPECTRAL_REFERENCE_DIR)

What is pinned (each array is produced by the reference's own code, unmodified):

* ``data_ref.npz`` -- outputs of the reference's host-side spectral data loaders
  (``data.py:6-182``): ``ColourSystem`` (CMF resampled to the bands, XYZ->RGB
  matrix ``T``, normalisation factor), ``RefractiveIndex`` for the three
  refractiveindex.info tables, ``SpecularVec`` (the ``k_1`` vector of
  ``main.py:71-76``) and ``EEMMatrix`` (``uv_green``, ``main.py:78-83``), at the
  reference's default spectral grid (25 bands, 10..1210 nm) and at the
  380..740 nm grid of the synthetic box workloads.  The raw input tables are
  not copied: loader tests that need them read the reference tree when it is
  present and are skipped otherwise.
* ``scene_ref.npz`` -- the reference's default scene (``create_scene``,
  ``main.py:89-247``): its meshes and material dictionaries, and the same
  scene flattened by ``setup_scene`` (``main.py:513-539``),
  the reference BVH (``build_bvh``, ``main.py:437-507``) with its node table and
  triangle permutation, the scene sizing of ``get_scene_dimensions``
  (``main.py:398-435``) and the per-band light CDF of ``main.py:590-627``.

Taichi is not importable here, so ``main.py`` cannot be imported as a module.
The pure-Python functions (``create_scene``, ``get_scene_dimensions``,
``build_bvh``, ``setup_scene``) are lifted out of its syntax tree and executed
unmodified, with the module globals they read; the Taichi fields that
``setup_scene`` fills are replaced by numpy arrays of the same dtype and by
plain record objects, and ``update_camera`` (a kernel) by a no-op.
"""
import ast
import os
import sys
import types

import numpy as np


def _load_data_module(ref):
    spec_path = os.path.join(ref, "data.py")
    mod = types.ModuleType("ref_data")
    mod.__file__ = spec_path
    exec(compile(open(spec_path).read(), spec_path, "exec"), mod.__dict__)
    return mod


def _lift_functions(ref, names, globs):
    path = os.path.join(ref, "main.py")
    tree = ast.parse(open(path).read(), path)
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    assert {n.name for n in body} == set(names), "reference functions not found"
    mod = ast.Module(body=body, type_ignores=[])
    exec(compile(mod, path, "exec"), globs)
    return {n: globs[n] for n in names}


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    cwd = os.getcwd()
    os.chdir(ref)  # the reference opens its data files by relative path
    try:
        data = _load_data_module(ref)
        out = {}
        for tag, (lmin, lmax) in {"ref": (10, 1210), "box": (380, 740)}.items():
            B = 25
            cs = data.ColourSystem(file_path="data/CMF/cie_cmf_xray_swir_vis.txt",
                                   red=[0.64, 0.33], green=[0.30, 0.60], blue=[0.15, 0.06],
                                   white=[0.33242, 0.34743], spectral_bands=B,
                                   wavelength_min=lmin, wavelength_max=lmax)
            out[f"{tag}_cmf"] = np.asarray(cs.cmf)
            out[f"{tag}_T"] = np.asarray(cs.T)
            out[f"{tag}_norm"] = np.float64(cs.normalization_factor)
            for metal in ("gold", "silver", "silicon"):
                ri = data.RefractiveIndex(file_path=f"data/refraction_index/{metal}.yml",
                                          spectral_bands=B, wavelength_min=lmin, wavelength_max=lmax)
                out[f"{tag}_{metal}_n"] = np.asarray(ri.n)
                out[f"{tag}_{metal}_k"] = np.asarray(ri.k)
            kv = data.SpecularVec(file_path="data/SpecVecs/spectrum_data_k_0_10.txt", scale=1e-6,
                                  spectral_bands=B, wavelength_min=lmin, wavelength_max=lmax)
            out[f"{tag}_k1"] = np.asarray(kv.vec)
            eem = data.EEMMatrix(file_path="data/EEMs/uv_green.txt", wavelength_min=lmin,
                                 wavelength_max=lmax, spectral_bands=B)
            out[f"{tag}_eem_uv_green"] = np.asarray(eem.matrix)
        np.savez_compressed(os.path.join(here, "data_ref.npz"), **out)

        # ---- default scene + reference BVH --------------------------------
        B = 25
        g = {"np": np, "SPECTRAL_BANDS": B, "print": lambda *a, **k: None}
        g["gold_ior"] = data.RefractiveIndex(file_path="data/refraction_index/silicon.yml",
                                             spectral_bands=B, wavelength_min=10, wavelength_max=1210)
        g["k_1"] = data.SpecularVec(file_path="data/SpecVecs/spectrum_data_k_0_10.txt", scale=1e-6,
                                    spectral_bands=B, wavelength_min=10, wavelength_max=1210)
        fns = _lift_functions(ref, ["create_scene", "get_scene_dimensions", "build_bvh"], g)
        scene = fns["create_scene"]()
        dims = fns["get_scene_dimensions"](scene)

        # run the reference's own setup_scene (main.py:509-631) against stand-ins
        # for the Taichi fields it writes; numpy arrays take the fields' dtypes
        mats = scene["materials"]
        M, T = dims["num_materials"], dims["num_triangles"]
        L = max(dims["max_num_lights_per_band"], 1)
        ns = types.SimpleNamespace
        tri_field = [ns() for _ in range(T)]
        node_field = [ns(aabb=ns(min=None, max=None), left_child=0, right_child=0, num_tris=0,
                         tri_start_idx=0) for _ in range(dims["num_bvh_nodes"])]
        g.update(
            PROP_REFRACTIVE_INDEX=0, PROP_EXTINCTION_COEFFICIENT=1, PROP_ROUGHNESS=2,
            PROP_SCATTERING_COEFFICIENT=3, PROP_EMISSION=4, PROP_ANISTROPY_FACTOR=5,
            PROP_IS_TRUE_VOLUME=0, PROP_SURFACE_EMISSION=1,
            material_props_f32=np.zeros((M, 6, B), np.float32),
            material_props_int=np.zeros((M, 2, B), np.int32),
            material_props_single_int=np.zeros(M, np.int32),
            triangles=tri_field, bvh_nodes=node_field, scene_dims=dims,
            num_lights_per_band=np.zeros(B, np.int32),
            total_light_area_field=np.zeros(B, np.float32),
            light_source_tri_indices=np.zeros((B, L), np.int32),
            light_source_cdf=np.zeros((B, L), np.float32),
            cam_origin={}, cam_lookat={}, cam_up={}, update_camera=lambda: None)
        _lift_functions(ref, ["setup_scene"], g)["setup_scene"](scene)

        # original (pre-BVH) triangle order, flattened as main.py:513-539 does
        orig = []
        for mesh in scene["meshes"]:
            verts = np.array(mesh["vertices"], dtype=np.float32)
            for face in mesh["faces"]:
                orig.append(np.concatenate([verts[face[0]], verts[face[1]], verts[face[2]]]))
        key = {o.tobytes(): i for i, o in enumerate(orig)}
        assert len(key) == T, "duplicate triangles make the permutation ambiguous"
        perm = np.array([key[np.concatenate([np.asarray(t.v0, np.float32), np.asarray(t.v1, np.float32),
                                             np.asarray(t.v2, np.float32)]).tobytes()]
                         for t in tri_field], np.int32)
        f32 = lambda key_: np.array([getattr(t, key_) for t in tri_field], dtype=np.float32)
        sc = {k: f32(k) for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area")}
        sc["mat_id"] = np.array([t.material_id for t in tri_field], np.int32)
        sc["bvh_perm"] = perm  # reordered slot -> original triangle index
        used = [n for n in node_field if n.aabb.min is not None]
        N = len(used)
        sc["node_min"] = np.array([n.aabb.min for n in used], np.float32)
        sc["node_max"] = np.array([n.aabb.max for n in used], np.float32)
        sc["node_left"] = np.array([n.left_child for n in used], np.int32)
        sc["node_right"] = np.array([n.right_child for n in used], np.int32)
        sc["node_num_tris"] = np.array([n.num_tris for n in used], np.int32)
        sc["node_tri_start"] = np.array([n.tri_start_idx for n in used], np.int32)
        ntri = sc["node_num_tris"]
        sc.update(light_cdf=g["light_source_cdf"], light_idx=g["light_source_tri_indices"],
                  num_lights=g["num_lights_per_band"], light_area=g["total_light_area_field"])
        sc["dims"] = np.array([dims["num_materials"], dims["num_triangles"], dims["num_bvh_nodes"],
                               dims["max_num_lights_per_band"]], np.int64)
        sc.update(mat_f32=g["material_props_f32"], mat_i32=g["material_props_int"],
                  mat_eem=g["material_props_single_int"])
        cam = scene["camera"]
        sc["camera"] = np.array([cam["origin"], cam["lookat"], cam["up"]], np.float32)
        # the scene dictionary itself (inputs of setup_scene), so the package's
        # flattening can be checked against the reference's
        import json
        sc["num_meshes"] = np.int64(len(scene["meshes"]))
        for mi, mesh in enumerate(scene["meshes"]):
            sc[f"mesh{mi}_vertices"] = np.asarray(mesh["vertices"], np.float64)
            sc[f"mesh{mi}_faces"] = np.asarray(mesh["faces"], np.int64)
            sc[f"mesh{mi}_material_id"] = np.int64(mesh["material_id"])
            if "vertex_normals" in mesh:
                sc[f"mesh{mi}_vertex_normals"] = np.asarray(mesh["vertex_normals"], np.float64)
        to_py = lambda v: [float(x) for x in v] if not isinstance(v, (int, float)) else v
        sc["materials_json"] = np.array(json.dumps([{k: to_py(v) for k, v in m.items()} for m in mats]))
        np.savez_compressed(os.path.join(here, "scene_ref.npz"), **sc)
        print(f"scene: {T} tris, {N} nodes, {int((ntri > 0).sum())} leaves; dims {dims}")
    finally:
        os.chdir(cwd)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPECTRAL_REFERENCE_DIR")
    if not ref or not os.path.isfile(os.path.join(ref, "main.py")):
        sys.exit("usage: make_golden.py <reference checkout> (or set SPECTRAL_REFERENCE_DIR)")
    main(ref)
