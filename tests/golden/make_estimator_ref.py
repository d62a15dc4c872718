"""Fixtures of the reference's estimator, computed by the reference's own code.

Run once, where the reference checkout is present (this container):

    python tests/golden/make_estimator_ref.py <reference checkout>
    (or set SPECTRAL_REFERENCE_DIR)

The reference's hot path is Taichi code (``main.py:682-1590``) and Taichi is
not installable offline.  Every ``@ti.func`` of that path, the ``@ti.dataclass``
records it uses (``main.py:254-359``), the render constants
(``main.py:13-35``), the ``cast_rays`` and ``update_camera`` kernels and the
host-side ``get_scene_dimensions`` / ``build_bvh`` / ``setup_scene`` are lifted
out of ``main.py``'s syntax tree UNMODIFIED (the only rewrite maps the ``**``
operator onto Taichi's integer-power semantics) and executed against the
stand-in of ``taichi_standin.py`` (float32 arithmetic with one rounding per
operation; ``ti.random()`` fed from a given draw list or from the Philox
stream the oracle uses).  Nothing of the reference is copied into the repo:
only inputs and the outputs its code produced.

Outputs:

* ``estimator_ref.npz`` -- function-level cases: ``intersect_triangle``,
  ``intersect_aabb``, ``trace``, ``complex_sqrt`` / ``complex_div``,
  ``fresnel_spectral``, ``normaldistrobution_ggx``, ``geometry_smith_ggx``,
  ``importance_sample_ggx``, ``evaluate_henyey_greenstein``,
  ``sample_henyey_greenstein``, ``cosine_weighted_hemisphere_direction``,
  ``random_in_unit_sphere``, ``evaluate_bsdf``, ``shadow_transmittance``,
  ``sample_direct_light``, ``scatter_surface``, ``scatter_volume``; each with
  its inputs, the random draws it was given, the draws it consumed and its
  outputs.  Scene-dependent functions run on the reference's default scene
  (``scene_ref.npz``, its own ``setup_scene`` output, with the ``uv_green``
  EEM of ``data_ref.npz``).
* ``paths_ref.npz`` -- whole paths: ``cast_rays`` for a set of pixels and
  passes of three scenes (the reference's default scene at its own
  constants; the synthetic box scene, whose rough dielectric sphere makes the
  reference compute NaN deposits after a path's throughput reaches zero; a
  small volume scene with an HG medium that fluoresces), every deposit
  recorded separately, with the scenes exactly as the reference's
  ``setup_scene`` laid them out (triangles in its BVH order, its node table,
  light CDF and camera basis).
"""
import ast
import multiprocessing as mp
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import taichi_standin as S  # noqa: E402

HOT = ["random_in_unit_sphere", "cosine_weighted_hemisphere_direction", "evaluate_henyey_greenstein",
       "sample_henyey_greenstein", "intersect_aabb", "intersect_triangle", "trace", "complex_mul", "complex_div",
       "complex_mod_sq", "complex_sqrt", "normaldistrobution_ggx", "geometry_smith_ggx", "fresnel_spectral",
       "importance_sample_ggx", "get_mat", "scatter_surface", "scatter_volume", "sample_direct_light",
       "evaluate_bsdf", "shadow_transmittance", "cast_rays", "update_camera"]
HOST = ["get_scene_dimensions", "build_bvh", "setup_scene"]
CLASSES = ["Triangle", "BVHNode", "MaterialSample", "Ray", "ShadowRay", "HitRecord", "VolumeEvent", "SurfaceEvent",
           "NEE_Sample"]
ASSIGNS = ["ASPECT_RATIO", "IMAGE_WIDTH", "IMAGE_HEIGHT", "RESOLUTION_SCALE", "EPSILON", "ESCAPE", "MAX_PATH_LENGTH",
           "SAMPLES_PER_PIXEL", "SCATTER_BOUNCES", "SPECTRAL_BANDS", "WAVELENGTH_MAX", "WAVELENGTH_MIN",
           "WAVELENGTH_STEP", "RENDER_WIDTH", "RENDER_HEIGHT", "PROP_REFRACTIVE_INDEX", "PROP_EXTINCTION_COEFFICIENT",
           "PROP_ROUGHNESS", "PROP_SCATTERING_COEFFICIENT", "PROP_EMISSION", "PROP_ANISTROPY_FACTOR",
           "NUM_F32_PROPERTIES", "PROP_IS_TRUE_VOLUME", "PROP_SURFACE_EMISSION", "NUM_INT_PROPERTIES",
           "SpectralVector", "SpectralBool", "AABB"]


def reference_dir(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("SPECTRAL_REFERENCE_DIR")
    if not ref or not os.path.isfile(os.path.join(ref, "main.py")):
        sys.exit("usage: make_estimator_ref.py <reference checkout> (or set SPECTRAL_REFERENCE_DIR)")
    return ref


class _TaichiPow(ast.NodeTransformer):
    """``a ** b`` -> ``ti_pow(a, b)``: Taichi lowers a constant integer power to
    multiplications, where Python would call a float32 ``pow``."""

    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Pow):
            call = ast.Call(func=ast.Name("ti_pow", ast.Load()), args=[node.left, node.right], keywords=[])
            return ast.copy_location(call, node)
        return node


def lift(ref, overrides=None):
    """Namespace holding the reference's constants, records and functions."""
    path = os.path.join(ref, "main.py")
    tree = ast.parse(open(path).read(), path)
    g = {"ti": S.ti, "tm": S.tm, "np": np, "ti_pow": S.ti_pow, "print": lambda *a, **k: None}
    nodes, found = [], set()
    for n in tree.body:
        if isinstance(n, ast.Assign) and len(n.targets) == 1 and isinstance(n.targets[0], ast.Name) \
                and n.targets[0].id in ASSIGNS:
            nodes.append(n)
            found.add(n.targets[0].id)
        elif isinstance(n, ast.ClassDef) and n.name in CLASSES:
            nodes.append(n)
            found.add(n.name)
        elif isinstance(n, ast.FunctionDef) and n.name in HOT:
            nodes.append(_TaichiPow().visit(n))
            found.add(n.name)
        elif isinstance(n, ast.FunctionDef) and n.name in HOST:
            nodes.append(n)
            found.add(n.name)
    missing = set(HOT + HOST + CLASSES + ASSIGNS) - found
    assert not missing, f"not found in main.py: {sorted(missing)}"
    mod = ast.Module(body=nodes, type_ignores=[])
    ast.fix_missing_locations(mod)
    exec(compile(mod, path, "exec"), g)
    g.update(overrides or {})
    return g


# --------------------------------------------------------------------------- scenes
def reference_setup(g, scene, eems):
    """Run the reference's own get_scene_dimensions / build_bvh / setup_scene
    (main.py:398-631) on a create_scene() dictionary; returns the fields it
    fills as arrays in the reference layout (triangles in BVH order)."""
    B = g["SPECTRAL_BANDS"]
    dims = g["get_scene_dimensions"](scene)
    M, T = dims["num_materials"], dims["num_triangles"]
    L = max(dims["max_num_lights_per_band"], 1)
    ns = types.SimpleNamespace
    tri = [ns() for _ in range(T)]
    nodes = [ns(aabb=ns(min=None, max=None), left_child=0, right_child=0, num_tris=0, tri_start_idx=0)
             for _ in range(dims["num_bvh_nodes"])]
    cam = {}
    h = dict(g)
    h.update(material_props_f32=np.zeros((M, 6, B), np.float32), material_props_int=np.zeros((M, 2, B), np.int32),
             material_props_single_int=np.zeros(M, np.int32), triangles=tri, bvh_nodes=nodes, scene_dims=dims,
             num_lights_per_band=np.zeros(B, np.int32), total_light_area_field=np.zeros(B, np.float32),
             light_source_tri_indices=np.zeros((B, L), np.int32), light_source_cdf=np.zeros((B, L), np.float32),
             cam_origin=cam, cam_lookat=cam, cam_up=cam, update_camera=lambda: None)
    # the host functions read their globals from the namespace they were defined in
    for name in HOST:
        fn = g[name]
        h[name] = types.FunctionType(fn.__code__, h, name, fn.__defaults__)
    h["setup_scene"](scene)
    used = [n for n in nodes if n.aabb.min is not None]
    a = {k: np.array([getattr(t, k) for t in tri], np.float32)
         for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area")}
    a["mat_id"] = np.array([t.material_id for t in tri], np.int32)
    a["node_min"] = np.array([n.aabb.min for n in used], np.float32)
    a["node_max"] = np.array([n.aabb.max for n in used], np.float32)
    a["node_left"] = np.array([n.left_child for n in used], np.int32)
    a["node_right"] = np.array([n.right_child for n in used], np.int32)
    a["node_num_tris"] = np.array([n.num_tris for n in used], np.int32)
    a["node_tri_start"] = np.array([n.tri_start_idx for n in used], np.int32)
    a.update(mat_f32=h["material_props_f32"], mat_i32=h["material_props_int"], mat_eem=h["material_props_single_int"],
             light_cdf=h["light_source_cdf"], light_idx=h["light_source_tri_indices"],
             num_lights=h["num_lights_per_band"], light_area=h["total_light_area_field"])
    a["eem"] = np.asarray(eems, np.float32)
    c = scene["camera"]
    a["camera"] = np.array([c["origin"], c["lookat"], c["up"]], np.float32)
    return a


def bind(g, a):
    """Point the lifted functions at a scene (the fields of main.py:361-394, 1683-1709)."""
    tri_t, node_t, aabb_t = g["Triangle"], g["BVHNode"], g["AABB"]
    g["triangles"] = S.RecordField([
        tri_t(v0=S.Vec(a["v0"][i]), v1=S.Vec(a["v1"][i]), v2=S.Vec(a["v2"][i]), n0=S.Vec(a["n0"][i]),
              n1=S.Vec(a["n1"][i]), n2=S.Vec(a["n2"][i]), normal=S.Vec(a["normal"][i]), material_id=int(a["mat_id"][i]),
              area=a["area"][i]) for i in range(a["v0"].shape[0])])
    g["bvh_nodes"] = S.RecordField([
        node_t(aabb=aabb_t(min=S.Vec(a["node_min"][i]), max=S.Vec(a["node_max"][i])),
               left_child=int(a["node_left"][i]), right_child=int(a["node_right"][i]),
               num_tris=int(a["node_num_tris"][i]), tri_start_idx=int(a["node_tri_start"][i]))
        for i in range(a["node_min"].shape[0])])
    g["material_props_f32"] = S.Field(np.asarray(a["mat_f32"], np.float32))
    g["material_props_int"] = S.Field(np.asarray(a["mat_i32"], np.int32))
    g["material_props_single_int"] = S.Field(np.asarray(a["mat_eem"], np.int32))
    g["reemission_matrix"] = S.Field(np.asarray(a["eem"], np.float32))
    g["light_source_cdf"] = S.Field(np.asarray(a["light_cdf"], np.float32))
    g["light_source_tri_indices"] = S.Field(np.asarray(a["light_idx"], np.int32))
    g["num_lights_per_band"] = S.Field(np.asarray(a["num_lights"], np.int32))
    g["total_light_area_field"] = S.Field(np.asarray(a["light_area"], np.float32))
    for k in ("cam_origin", "cam_lookat", "cam_up", "cam_u", "cam_v", "cam_w"):
        g[k] = S.Field(np.zeros(3, np.float32), vec=True)
    g["cam_origin"][None], g["cam_lookat"][None], g["cam_up"][None] = a["camera"]
    g["update_camera"]()  # main.py:633-640, the reference's own camera basis
    return g


# --------------------------------------------------------------------------- workers
_G = None


def _worker_init(ref, overrides, arrays):
    global _G
    _G = bind(lift(ref, overrides), arrays)


def _cast_rays_job(job):
    """cast_rays (main.py:1502-1590) for some pixels of one pass."""
    pixels, pass_idx, band, seed = job
    g = _G
    W, H = g["RENDER_WIDTH"], g["RENDER_HEIGHT"]
    dom = S.PixelDomain([(p % W, p // W) for p in pixels], W, seed, pass_idx)
    g["pixels_geometry"] = dom
    g["active_wavelength_idx"] = S.Field(np.zeros((W, H), np.int32))
    g["transport_wavelength_idx"] = S.Field(np.zeros((W, H), np.int32))
    log = S.DepositLog()
    g["block_accumulator"] = log
    with np.errstate(all="ignore"):
        g["cast_rays"](band, 0)
    return log.log, dom.draws


def _draws(rng, n, k):
    return (rng.integers(0, 1 << 24, size=(n, k)) * (1.0 / 16777216.0)).astype(np.float32)


def _unit(rng, n):
    d = rng.normal(size=(n, 3))
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def _call(g, fn, args, draws):
    S.RNG.replay(draws)
    with np.errstate(all="ignore"):
        out = g[fn](*args)
    return out, S.RNG.n


def function_cases(g, a, rng):
    """Function-level cases (inputs, draws, outputs)."""
    V = lambda x: S.Vec(x)
    out = {}
    B = g["SPECTRAL_BANDS"]
    M = a["mat_f32"].shape[0]
    lo, hi = a["node_min"][0], a["node_max"][0]

    # intersect_triangle: random triangles and rays, a share aimed at the triangle
    n = 3000
    v = rng.uniform(-1, 1, size=(n, 3, 3)).astype(np.float32)
    o = rng.uniform(-2, 2, size=(n, 3)).astype(np.float32)
    w = rng.dirichlet([1, 1, 1], size=n)
    tgt = (w[:, :1] * v[:, 0] + w[:, 1:2] * v[:, 1] + w[:, 2:] * v[:, 2]).astype(np.float32)
    d = np.where(rng.uniform(size=(n, 1)) < 0.6, tgt - o, rng.normal(size=(n, 3))).astype(np.float32)
    d[: n // 10, 2] = 0.0  # axis-parallel components
    v[n // 10: n // 5, 2] = v[n // 10: n // 5, 0]  # degenerate (zero-area) triangles
    res = []
    for i in range(n):
        tri = g["Triangle"](v0=V(v[i, 0]), v1=V(v[i, 1]), v2=V(v[i, 2]))
        r, _ = _call(g, "intersect_triangle", (V(o[i]), V(d[i]), tri), [])
        res.append(list(r))
    out["tri_in"] = np.concatenate([o, d, v.reshape(n, 9)], 1)
    out["tri_out"] = np.array(res, np.float32)

    # intersect_aabb
    n = 3000
    bmin = rng.uniform(-1, 0.5, size=(n, 3)).astype(np.float32)
    bmax = (bmin + rng.uniform(0, 1, size=(n, 3))).astype(np.float32)
    bmax[: n // 10, 1] = bmin[: n // 10, 1]  # flat boxes
    o = rng.uniform(-2, 2, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 8, 0] = 0.0
    inv = (np.float32(1.0) / d).astype(np.float32)
    res = []
    for i in range(n):
        box = g["AABB"](min=V(bmin[i]), max=V(bmax[i]))
        r, _ = _call(g, "intersect_aabb", (V(o[i]), V(inv[i]), box), [])
        res.append(int(bool(r)))
    out["aabb_in"] = np.concatenate([o, inv, bmin, bmax], 1).astype(np.float32)
    out["aabb_out"] = np.array(res, np.int32)

    # trace on the scene
    n = 1500
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = _unit(rng, n)
    res = []
    for i in range(n):
        h, _ = _call(g, "trace", (V(o[i]), V(d[i])), [])
        res.append([h.t, *h.normal, *h.shading_normal, h.material_id, h.u, h.v, h.is_hit, h.is_front_face, h.tri_idx])
    out["trace_in"] = np.concatenate([o, d], 1)
    out["trace_out"] = np.array(res, np.float64).astype(np.float32)

    # complex_sqrt / complex_div
    n = 2000
    z = rng.normal(size=(n, 4)).astype(np.float32) * np.float32(3)
    z[: n // 5, 1] = 0.0
    res = []
    for i in range(n):
        r1, _ = _call(g, "complex_sqrt", (S.ti.Vector([z[i, 0], z[i, 1]]),), [])
        r2, _ = _call(g, "complex_div", (S.ti.Vector([z[i, 0], z[i, 1]]), S.ti.Vector([z[i, 2], z[i, 3]])), [])
        res.append([*r1, *r2])
    out["complex_in"] = z
    out["complex_out"] = np.array(res, np.float32)

    # fresnel_spectral (dielectrics, conductors, both sides, grazing)
    n = 3000
    x = np.stack([rng.uniform(-1.2, 1.2, n), rng.uniform(1.0, 2.5, n), rng.choice([0.0, 1e-7, 0.5], n),
                  rng.uniform(0.2, 3.0, n), rng.choice([0.0, 1e-6], n) + rng.uniform(0, 8, n) * (rng.uniform(size=n) < .5)],
                 1).astype(np.float32)
    res = [_call(g, "fresnel_spectral", tuple(x[i]), [])[0] for i in range(n)]
    out["fresnel_in"] = x
    out["fresnel_out"] = np.array(res, np.float32)

    # normaldistrobution_ggx, geometry_smith_ggx, importance_sample_ggx
    n = 3000
    x = np.stack([rng.uniform(-0.1, 1.0, n), rng.uniform(0.0, 1.0, n)], 1).astype(np.float32)
    out["ggx_d_in"] = x
    out["ggx_d_out"] = np.array([_call(g, "normaldistrobution_ggx", tuple(x[i]), [])[0] for i in range(n)], np.float32)
    nv, vv, lv = _unit(rng, n), _unit(rng, n), _unit(rng, n)
    r = rng.uniform(0.0, 1.0, n).astype(np.float32)
    out["ggx_g_in"] = np.concatenate([nv, vv, lv, r[:, None]], 1)
    out["ggx_g_out"] = np.array([_call(g, "geometry_smith_ggx", (V(nv[i]), V(vv[i]), V(lv[i]), r[i]), [])[0]
                                 for i in range(n)], np.float32)
    xi = _draws(rng, n, 2)
    nv[: n // 10] = np.array([0, 1, 0], np.float32)  # the other tangent frame
    out["ggx_sample_in"] = np.concatenate([xi, nv, r[:, None]], 1)
    out["ggx_sample_out"] = np.array([list(_call(g, "importance_sample_ggx",
                                                 (S.tm.vec2(xi[i, 0], xi[i, 1]), V(nv[i]), r[i]), [])[0])
                                      for i in range(n)], np.float32)

    # Henyey-Greenstein
    n = 3000
    x = np.stack([rng.uniform(-1, 1, n), rng.choice([0.0, 5e-5, 0.3, -0.6, 0.7, 0.95], n)], 1).astype(np.float32)
    out["hg_eval_in"] = x
    out["hg_eval_out"] = np.array([_call(g, "evaluate_henyey_greenstein", tuple(x[i]), [])[0] for i in range(n)],
                                  np.float32)
    dr = _draws(rng, n, 4)
    wv = _unit(rng, n)
    res, used = [], []
    for i in range(n):
        r_, k = _call(g, "sample_henyey_greenstein", (V(wv[i]), x[i, 1]), dr[i])
        res.append(list(r_))
        used.append(k)
    out["hg_sample_in"] = np.concatenate([wv, x[:, 1:]], 1)
    out["hg_sample_draws"] = dr
    out["hg_sample_out"] = np.array(res, np.float32)
    out["hg_sample_used"] = np.array(used, np.int32)

    # cosine_weighted_hemisphere_direction, random_in_unit_sphere
    res, res2 = [], []
    for i in range(n):
        res.append(list(_call(g, "cosine_weighted_hemisphere_direction", (V(wv[i]),), dr[i])[0]))
        res2.append(list(_call(g, "random_in_unit_sphere", (), dr[i])[0]))
    out["cos_hemi_in"] = wv
    out["cos_hemi_draws"] = dr
    out["cos_hemi_out"] = np.array(res, np.float32)
    out["sphere_draws"] = dr
    out["sphere_out"] = np.array(res2, np.float32)

    # evaluate_bsdf (vol, surf, V, L, N, band)
    n = 2500
    vol = rng.integers(0, M, n)
    surf = rng.integers(0, M, n)
    Nn = _unit(rng, n)
    Vv = _unit(rng, n)
    Vv = np.where((Vv * Nn).sum(1, keepdims=True) < 0, -Vv, Vv).astype(np.float32)
    Lv = _unit(rng, n)
    Lv[: n // 3] = np.where((Lv[: n // 3] * Nn[: n // 3]).sum(1, keepdims=True) < 0, -Lv[: n // 3], Lv[: n // 3])
    wl = rng.integers(0, B, n)
    res = []
    for i in range(n):
        (bsdf, pdf), _ = _call(g, "evaluate_bsdf", (int(vol[i]), int(surf[i]), V(Vv[i]), V(Lv[i]), V(Nn[i]), int(wl[i]), 0),
                               [])
        res.append([bsdf, pdf])
    out["bsdf_in"] = np.concatenate([vol[:, None], surf[:, None], Vv, Lv, Nn, wl[:, None]], 1).astype(np.float32)
    out["bsdf_out"] = np.array(res, np.float32)

    # shadow_transmittance (origin, dir, max_dist, light tri, medium, band)
    lights = np.unique(a["light_idx"][a["light_cdf"] > 0])
    n = 1200
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    lt = np.where(rng.uniform(size=n) < 0.7, rng.choice(lights, n), rng.integers(0, a["v0"].shape[0], n))
    P = ((a["v0"][lt] + a["v1"][lt] + a["v2"][lt]) / 3).astype(np.float32)
    d = P - o
    dist = np.linalg.norm(d, axis=1).astype(np.float32)
    d = (d / dist[:, None]).astype(np.float32)
    vol = rng.integers(0, M, n)
    wl = rng.integers(0, B, n)
    res = [_call(g, "shadow_transmittance", (V(o[i]), V(d[i]), dist[i], int(lt[i]), int(vol[i]), int(wl[i])), [])[0]
           for i in range(n)]
    out["shadow_in"] = np.concatenate([o, d, dist[:, None], lt[:, None], vol[:, None], wl[:, None]], 1).astype(np.float32)
    out["shadow_out"] = np.array(res, np.float32)

    # sample_direct_light (ray, normal, surface material or -1)
    n = 1200
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = _unit(rng, n)
    Nn = _unit(rng, n)
    act = rng.integers(0, B, n)
    trn = np.where(rng.uniform(size=n) < 0.7, act, rng.integers(0, B, n))
    vol = rng.integers(0, M, n)
    surf = np.where(rng.uniform(size=n) < 0.3, -1, rng.integers(0, M, n))
    dr = _draws(rng, n, 8)
    res, used = [], []
    for i in range(n):
        ray = g["Ray"](position=V(o[i]), direction=V(d[i]), active_wavelength_idx=int(act[i]),
                       transport_wavelength_idx=int(trn[i]), vol_mat_id=int(vol[i]), throughput=1.0)
        r_, k = _call(g, "sample_direct_light", (ray, V(Nn[i]), int(surf[i])), dr[i])
        res.append([r_.contribution_factor, r_.emission, r_.weight])
        used.append(k)
    out["nee_in"] = np.concatenate([o, d, act[:, None], trn[:, None], vol[:, None], Nn, surf[:, None]], 1).astype(
        np.float32)
    out["nee_draws"] = dr
    out["nee_out"] = np.array(res, np.float32)
    out["nee_used"] = np.array(used, np.int32)

    # scatter_surface (ray, volume event): every material as the surface
    n = 2500
    d = _unit(rng, n)
    Nn = _unit(rng, n)
    Nn = np.where((Nn * d).sum(1, keepdims=True) > 0, -Nn, Nn).astype(np.float32)
    act = rng.integers(0, B, n)
    vol = rng.integers(0, M, n)
    hm = rng.integers(0, M, n)
    dr = _draws(rng, n, 10)
    res, used = [], []
    for i in range(n):
        ray = g["Ray"](position=V([0, 0, 0]), direction=V(d[i]), active_wavelength_idx=int(act[i]),
                       transport_wavelength_idx=int(act[i]), vol_mat_id=int(vol[i]), throughput=1.0)
        ev = g["VolumeEvent"](hit_mat_id=int(hm[i]), shading_normal=V(Nn[i]), normal=V(Nn[i]), is_front_face=1)
        r_, k = _call(g, "scatter_surface", (ray, ev), dr[i])
        res.append([r_.did_reflect, *r_.direction, r_.estimator, r_.pdf, r_.new_wavelength])
        used.append(k)
    out["surface_in"] = np.concatenate([d, act[:, None], vol[:, None], hm[:, None], Nn], 1).astype(np.float32)
    out["surface_draws"] = dr
    out["surface_out"] = np.array(res, np.float32)
    out["surface_used"] = np.array(used, np.int32)

    # scatter_volume (ray): free flight against the scene
    n = 1500
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = _unit(rng, n)
    act = rng.integers(0, B, n)
    vol = rng.integers(0, M, n)
    dr = _draws(rng, n, 10)
    res, used = [], []
    for i in range(n):
        ray = g["Ray"](position=V(o[i]), direction=V(d[i]), active_wavelength_idx=int(act[i]),
                       transport_wavelength_idx=int(act[i]), vol_mat_id=int(vol[i]), throughput=1.0,
                       penetrated_tri_idx=-1)
        e, k = _call(g, "scatter_volume", (ray,), dr[i])
        res.append([e.hit_action, e.travel_distance, e.estimator, *e.normal, *e.shading_normal, e.is_front_face,
                    e.hit_mat_id, e.tri_idx, *e.direction, e.new_wavelength_idx, e.penetrated_tri_idx])
        used.append(k)
    out["volume_in"] = np.concatenate([o, d, act[:, None], vol[:, None]], 1).astype(np.float32)
    out["volume_draws"] = dr
    out["volume_out"] = np.array(res, np.float64).astype(np.float32)
    out["volume_used"] = np.array(used, np.int32)
    return out


def scene_consts(g, a, width, height, depth, lmin, lmax):
    B = g["SPECTRAL_BANDS"]
    return {"RENDER_WIDTH": width, "RENDER_HEIGHT": height, "MAX_PATH_LENGTH": depth, "WAVELENGTH_MIN": lmin,
            "WAVELENGTH_MAX": lmax, "WAVELENGTH_STEP": (lmax - lmin) / (B - 1)}


def run_paths(ref, overrides, arrays, jobs, procs):
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_worker_init, initargs=(ref, overrides, arrays)) as pool:
        return pool.map(_cast_rays_job, jobs, chunksize=1)


def main(ref):
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    procs = max(1, min(32, os.cpu_count() or 1))
    base = lift(ref)
    scene_ref = dict(np.load(os.path.join(HERE, "scene_ref.npz")))
    data_ref = np.load(os.path.join(HERE, "data_ref.npz"))
    B = base["SPECTRAL_BANDS"]
    # the reference's default scene: its setup_scene output, EEM id 1 = uv_green (main.py:78-83, 1684)
    eem = np.zeros((2, B, B), np.float32)
    eem[1] = data_ref["ref_eem_uv_green"]
    ref_arrays = {k: scene_ref[k] for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "mat_id", "node_min",
                                            "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start",
                                            "mat_f32", "mat_i32", "mat_eem", "light_cdf", "light_idx", "num_lights",
                                            "light_area", "camera")}
    ref_arrays["eem"] = eem

    # ---- function-level cases on the reference scene
    g = bind(lift(ref), ref_arrays)
    out = function_cases(g, ref_arrays, np.random.default_rng(2024))
    out["eps"] = np.float32(g["EPSILON"])
    out["escape"] = np.float32(g["ESCAPE"])
    out["lambda_min"] = np.float32(g["WAVELENGTH_MIN"])
    out["lambda_max"] = np.float32(g["WAVELENGTH_MAX"])
    out["scatter_bounces"] = np.int32(g["SCATTER_BOUNCES"])
    np.savez_compressed(os.path.join(HERE, "estimator_ref.npz"), **out)
    print("function cases:", {k: v.shape for k, v in out.items() if k.endswith("_out")})

    # ---- whole paths
    from importlib import import_module
    configs = import_module("spectral_b200.configs")
    scenes = {}
    # (1) the reference's default scene at the reference's own constants
    scenes["ref"] = (ref_arrays, {}, 300, [0, 1, 2], [3, 12, 21])
    # (2) the synthetic box (GGX dielectric sphere, alpha 0.1) at 48x48, depth 8, reference FOV
    sc, cf, ex = configs.box_scene(sphere_slices=12, sphere_stacks=13, width=48, height=48)
    gb = lift(ref, scene_consts(base, None, 48, 48, 8, 380.0, 740.0))
    arr = reference_setup(gb, sc, np.zeros((1, B, B), np.float32))
    scenes["box"] = (arr, scene_consts(base, None, 48, 48, 8, 380.0, 740.0), 400, [0, 1], [5, 17])
    # (3) a small volume scene: HG medium that fluoresces + fluorescent wall, depth 12
    sc, cf, ex = configs.volume_scene(medium_slices=8, medium_stacks=9, width=32, height=32, depth=12,
                                      fluorescent_medium=True)
    gv = lift(ref, scene_consts(base, None, 32, 32, 12, 380.0, 740.0))
    arr = reference_setup(gv, sc, ex["eems"])
    scenes["volume"] = (arr, scene_consts(base, None, 32, 32, 12, 380.0, 740.0), 400, [0, 1], [2, 9])
    paths = {}
    seed = 0
    for name, (arr, ov, npix_sel, passes, bands) in scenes.items():
        gg = lift(ref, ov)
        W, H = gg["RENDER_WIDTH"], gg["RENDER_HEIGHT"]
        rng = np.random.default_rng(77)
        pix = np.sort(rng.choice(W * H, min(npix_sel, W * H), replace=False)).astype(np.int32)
        jobs = []
        chunk = max(1, len(pix) // (2 * procs))
        for p, b in zip(passes, bands):
            for s in range(0, len(pix), chunk):
                jobs.append((pix[s:s + chunk].tolist(), p, b, seed))
        res = run_paths(ref, ov, arr, jobs, procs)
        dep_pix, dep_pass, dep_band, dep_val, draws = [], [], [], [], []
        for (pl, p, b, _), (log, dr) in zip(jobs, res):
            for (i, j, bb, v) in log:
                dep_pix.append(j * W + i)
                dep_pass.append(p)
                dep_band.append(bb)
                dep_val.append(v)
            draws.extend(dr)
        for k, v in arr.items():
            paths[f"{name}_{k}"] = v
        gb = bind(lift(ref, ov), arr)  # camera basis by the reference's update_camera
        for k in ("cam_origin", "cam_u", "cam_v", "cam_w"):
            paths[f"{name}_{k}"] = np.array(list(gb[k][None]), np.float32)
        paths[f"{name}_config"] = np.array([W, H, B, gg["MAX_PATH_LENGTH"], gg["SCATTER_BOUNCES"]], np.int32)
        paths[f"{name}_lambda"] = np.array([gg["WAVELENGTH_MIN"], gg["WAVELENGTH_MAX"], gg["EPSILON"], gg["ESCAPE"],
                                            gg["ASPECT_RATIO"]], np.float64)
        paths[f"{name}_pixels"] = pix
        paths[f"{name}_passes"] = np.array(passes, np.int32)
        paths[f"{name}_bands"] = np.array(bands, np.int32)
        paths[f"{name}_seed"] = np.int32(seed)
        paths[f"{name}_dep_pixel"] = np.array(dep_pix, np.int32)
        paths[f"{name}_dep_pass"] = np.array(dep_pass, np.int32)
        paths[f"{name}_dep_band"] = np.array(dep_band, np.int32)
        paths[f"{name}_dep_value"] = np.array(dep_val, np.float32)
        paths[f"{name}_draws"] = np.array(draws, np.int32)
        vals = np.array(dep_val, np.float64)
        print(f"{name}: {len(jobs)} jobs, {len(vals)} deposits, {int(np.isnan(vals).sum())} NaN, "
              f"sum {np.nansum(vals):.6g}")
    paths["scenes"] = np.array(list(scenes.keys()))
    np.savez_compressed(os.path.join(HERE, "paths_ref.npz"), **paths)


if __name__ == "__main__":
    main(reference_dir(sys.argv))
