"""Host-side data and scene compilation against the reference's own outputs."""
import json
import os

import numpy as np
import pytest

from helpers import golden_data, golden_scene, orc, oracle_config, oracle_scene, random_rays, sb
from spectral_b200 import configs, spectral_data as sd


def reference_scene_dict():
    g = golden_scene()
    meshes = []
    for i in range(int(g["num_meshes"])):
        m = {"vertices": g[f"mesh{i}_vertices"], "faces": g[f"mesh{i}_faces"],
             "material_id": int(g[f"mesh{i}_material_id"])}
        if f"mesh{i}_vertex_normals" in g:
            m["vertex_normals"] = g[f"mesh{i}_vertex_normals"]
        meshes.append(m)
    mats = json.loads(str(g["materials_json"]))
    cam = {"origin": g["camera"][0], "lookat": g["camera"][1], "up": g["camera"][2]}
    return {"meshes": meshes, "materials": mats, "camera": cam}


def test_flatten_matches_setup_scene_bit_exact():
    g = golden_scene()
    t = sb.flatten_triangles(reference_scene_dict(), exact=True)
    perm = g["bvh_perm"]
    for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "mat_id"):
        assert np.array_equal(t[k][perm], g[k]), k


def test_flatten_vectorised_close():
    g = golden_scene()
    t = sb.flatten_triangles(reference_scene_dict(), exact=False)
    perm = g["bvh_perm"]
    for k in ("normal", "area", "n0"):
        assert np.allclose(t[k][perm], g[k], rtol=1e-6, atol=1e-7), k


def test_scene_dimensions_and_materials():
    g = golden_scene()
    sc = reference_scene_dict()
    d = sb.get_scene_dimensions(sc, 25)
    assert [d["num_materials"], d["num_triangles"], d["num_bvh_nodes"], d["max_num_lights_per_band"]] == \
        list(g["dims"])
    mf, mi, me = sb.material_tables(sc["materials"], 25)
    assert np.array_equal(mf, g["mat_f32"]) and np.array_equal(mi, g["mat_i32"]) and np.array_equal(me, g["mat_eem"])


def test_material_band_count_validated():
    with pytest.raises(ValueError):
        sb.material_tables([{"roughness": [0.1] * 24}], 25)


def test_display_matrix_matches_reference():
    d = golden_data()
    assert np.allclose(sd.srgb_xyz_to_rgb(), d["ref_T"], rtol=1e-13, atol=1e-15)


def test_loaders_match_reference(reference_tree):
    d = golden_data()
    p = lambda *a: os.path.join(reference_tree, "data", *a)
    for tag, (lo, hi) in {"ref": (10, 1210), "box": (380, 740)}.items():
        cs = sd.ColourSystem(p("CMF", "cie_cmf_xray_swir_vis.txt"), [0.64, 0.33], [0.30, 0.60], [0.15, 0.06],
                             [0.33242, 0.34743], lo, hi, 25)
        assert np.array_equal(cs.cmf, d[f"{tag}_cmf"])
        assert np.allclose(cs.T, d[f"{tag}_T"], rtol=1e-14)
        assert cs.normalization_factor == pytest.approx(float(d[f"{tag}_norm"]), rel=1e-14)
        for metal in ("gold", "silver", "silicon"):
            ri = sd.RefractiveIndex(p("refraction_index", f"{metal}.yml"), lo, hi, 25)
            assert np.array_equal(ri.n, d[f"{tag}_{metal}_n"]) and np.array_equal(ri.k, d[f"{tag}_{metal}_k"])
        kv = sd.SpecularVec(p("SpecVecs", "spectrum_data_k_0_10.txt"), 1e-6, lo, hi, 25)
        assert np.array_equal(kv.vec, d[f"{tag}_k1"])
        eem = sd.EEMMatrix(lo, hi, 25, file_path=p("EEMs", "uv_green.txt"))
        assert np.allclose(eem.matrix, d[f"{tag}_eem_uv_green"], rtol=1e-12, atol=1e-15)


def test_eem_fixture_has_stokes_mask():
    m = golden_data()["ref_eem_uv_green"]
    assert np.all(np.tril(m) == 0) and m.max() == pytest.approx(0.839444, rel=1e-5)


def test_cie_fit_shape():
    lam = np.arange(380, 781, 1.0)
    xyz = sd.cie1931_fit(lam)
    assert 550 <= lam[np.argmax(xyz[:, 1])] <= 560
    assert xyz[:, 1].max() == pytest.approx(1.0, abs=0.02)
    assert 590 <= lam[np.argmax(xyz[:, 0])] <= 605 and 440 <= lam[np.argmax(xyz[:, 2])] <= 450


def test_gaussian_stokes_eem():
    lam = configs.wavelengths()
    m = sd.gaussian_stokes_eem(lam, 40, 15, 0.6)
    d = lam[None, :] - lam[:, None]
    assert np.all(m[d < 0] == 0)
    rows = m.max(axis=1)
    assert np.allclose(rows[rows > 0], 0.6)
    assert np.argmax(m[0]) == np.argmin(np.abs(lam - (lam[0] + 40)))


def test_reflectance_encoding_gives_albedo():
    lam = configs.wavelengths()
    rho = sd.logistic(lam, 550, 0.03)
    k = sd.reflectance_to_k(rho, lam)
    sigma_a = 4 * np.pi * k / (lam * 1e-9)
    assert np.allclose(1.0 / (1.0 + sigma_a), np.clip(rho, 0.01, 0.99), rtol=1e-9)


def test_workload_sizes():
    s, c, _ = configs.box_scene()
    assert sb.get_scene_dimensions(s, 25)["num_triangles"] == 2062
    assert (c.width, c.height, c.max_path_length, c.samples_per_pixel) == (256, 256, 8, 75)
    s, c, _ = configs.volume_scene()
    assert sb.get_scene_dimensions(s, 25)["num_triangles"] == 12 + 2 + 20000
    assert (c.width, c.max_path_length, c.samples_per_pixel) == (512, 32, 525)
    s, c, _ = configs.terrain_scene(grid=64, sphere_slices=20, sphere_stacks=21)
    assert sb.get_scene_dimensions(s, 25)["num_triangles"] == 2 * 63 * 63 + 20 * 40 + 16
    assert (c.width, c.max_path_length, c.samples_per_pixel) == (1024, 12, 275)


def test_host_bvh_is_valid_and_traces_like_brute_force():
    s, c, ex = configs.box_scene(sphere_slices=16, sphere_stacks=17)
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    T = comp.num_tris
    assert sorted(bvh["tri_perm"]) == list(range(T))
    leaves = bvh["node_num_tris"] > 0
    covered = np.zeros(T, int)
    for n in np.nonzero(leaves)[0]:
        covered[bvh["node_tri_start"][n]:bvh["node_tri_start"][n] + bvh["node_num_tris"][n]] += 1
    assert np.all(covered == 1)
    # every node box contains its children's boxes (up to the padding of flat boxes)
    for n in np.nonzero(~leaves)[0]:
        for ch in (bvh["node_left"][n], bvh["node_right"][n]):
            assert np.all(bvh["node_min"][n] <= bvh["node_min"][ch] + 2e-6)
            assert np.all(bvh["node_max"][n] >= bvh["node_max"][ch] - 2e-6)
    # and every leaf box contains its triangles
    perm = bvh["tri_perm"]
    for n in np.nonzero(leaves)[0]:
        sl = perm[bvh["node_tri_start"][n]:bvh["node_tri_start"][n] + bvh["node_num_tris"][n]]
        for k in ("v0", "v1", "v2"):
            assert np.all(comp.tris[k][sl] >= bvh["node_min"][n]) and np.all(comp.tris[k][sl] <= bvh["node_max"][n])
    sc = oracle_scene(comp, bvh, s["camera"])
    ocfg = oracle_config(c)
    rays = random_rays(5000, 11, lo=-0.45, hi=0.45)
    tri, t, _, _ = orc.trace(sc, ocfg, rays)
    tri_b, t_b = orc.trace_brute(sc, ocfg, rays)
    assert np.array_equal(t, t_b)
    assert np.all(t[tri != tri_b] == t_b[tri != tri_b])


def test_host_bvh_capacity_error():
    import ctypes
    from spectral_b200 import _lib
    v = np.random.default_rng(0).uniform(size=(100, 3)).astype(np.float32)
    small = np.zeros(3, np.float32)
    ii = np.zeros(1, np.int32)
    perm = np.zeros(100, np.int32)
    nn = ctypes.c_int32()
    f = lambda a: a.ctypes.data_as(_lib.F32P)
    i = lambda a: a.ctypes.data_as(_lib.I32P)
    st = _lib.load().ts_build_bvh_host(100, f(v), f(v + 1), f(v + 2), 0, 0, 0.0, 0.0, 1, f(small), f(small), i(ii),
                                       i(ii), i(ii), i(ii), i(perm), ctypes.byref(nn))
    assert st == 4 and nn.value > 1  # TS_ERR_CAPACITY, needed node count reported
    assert b"hold 1 nodes" in _lib.load().ts_last_error(None)
