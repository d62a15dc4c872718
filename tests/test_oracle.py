"""The CPU oracle against the reference's own outputs and analytic known answers."""
import numpy as np
import pytest

from helpers import golden_compiled, golden_scene, light_tables, oracle_config, oracle_scene, orc, random_rays, sb


def test_philox_known_answers():
    # Random123 kat_vectors for philox4x32-10
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_sweep_builder_reproduces_reference_bvh():
    g = golden_scene()
    perm = g["bvh_perm"]
    inv = np.argsort(perm)
    b = orc.build_bvh_sweep(g["v0"][inv], g["v1"][inv], g["v2"][inv])
    for k in ("node_min", "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start"):
        assert np.array_equal(b[k], g[k]), k
    # leaves hold the same triangles; only the order inside a leaf may differ
    # (numpy's argsort does not fix the order of equal centroids)
    for n in np.nonzero(g["node_num_tris"] > 0)[0]:
        s, c = g["node_tri_start"][n], g["node_num_tris"][n]
        assert set(b["perm"][s:s + c]) == set(perm[s:s + c])


def test_light_tables_match_setup_scene():
    g = golden_scene()
    cdf, idx, nl, area = light_tables(g["mat_i32"], g["mat_id"], g["area"], 25)
    assert np.array_equal(cdf, g["light_cdf"]) and np.array_equal(idx, g["light_idx"])
    assert np.array_equal(nl, g["num_lights"]) and np.array_equal(area, g["light_area"])


def test_reference_traversal_equals_brute_force():
    cs, bvh, cam = golden_compiled()
    sc = oracle_scene(cs, bvh, cam)
    cfg = oracle_config(sb.RenderConfig())
    rays = random_rays(20000, 3)
    tri, t, u, v = orc.trace(sc, cfg, rays)
    tri_b, t_b = orc.trace_brute(sc, cfg, rays)
    assert np.array_equal(t, t_b)
    # differing triangles are exact distance ties (brute force keeps the lowest index)
    diff = tri != tri_b
    assert diff.mean() < 0.01
    assert np.all(t[diff] == t_b[diff])
    assert (tri >= 0).mean() > 0.5


def test_double_traversal_close():
    cs, bvh, cam = golden_compiled()
    sc = oracle_scene(cs, bvh, cam)
    cfg = oracle_config(sb.RenderConfig())
    rays = random_rays(5000, 4)
    tri, t, _, _ = orc.trace(sc, cfg, rays)
    tri_d, t_d, _, _ = orc.trace(sc, cfg, rays, use_double=True)
    hit = tri >= 0
    assert np.mean(tri == tri_d) > 0.99
    same = hit & (tri == tri_d)
    assert np.all(np.abs(t[same] - t_d[same]) <= 1e-5 * t_d[same])


@pytest.mark.parametrize("n,k", [(1.5, 0.0), (1.33, 0.0), (0.2, 3.0), (1.5, 8.0), (3.0, 1e-2)])
def test_fresnel_normal_incidence(n, k):
    want = ((n - 1) ** 2 + k ** 2) / ((n + 1) ** 2 + k ** 2)
    assert orc.fresnel(1.0, 1.0, 0.0, n, k, True) == pytest.approx(want, rel=1e-12)
    assert orc.fresnel(1.0, 1.0, 0.0, n, k, False) == pytest.approx(want, rel=2e-6)


def test_fresnel_grazing_and_matched():
    assert orc.fresnel(0.0, 1.0, 0.0, 1.5, 0.0, True) == pytest.approx(1.0, abs=1e-9)
    assert orc.fresnel(0.7, 1.5, 0.0, 1.5, 0.0, True) == pytest.approx(0.0, abs=1e-12)


def test_ggx_normalisation():
    # integral of D(h) cos(theta_h) over the hemisphere is 1 (alpha = roughness^2)
    from scipy.integrate import quad
    for r in (0.2, 0.5, 0.9):
        val, _ = quad(lambda m: orc.ggx_d(m, r, True) * m, 0.0, 1.0, points=[0.99, 0.999], limit=400)
        assert 2 * np.pi * val == pytest.approx(1.0, rel=1e-6), r


def test_henyey_greenstein_normalisation():
    mu = np.linspace(-1.0, 1.0, 4001)
    for g in (0.0, 0.3, 0.7, -0.5):
        p = np.array([orc.hg_eval(m, g, True) for m in mu])
        assert 2 * np.pi * np.trapezoid(p, mu) == pytest.approx(1.0, rel=2e-3), g


def _emitter_scene(emission):
    B = 25
    air = {"refractive_index": [1.0] * B, "is_true_volume": [1] * B}
    light = {"refractive_index": [1.0] * B, "surface_emission": [1] * B, "emission": list(emission)}
    quad = {"vertices": [[-5, -5, 0], [5, -5, 0], [5, 5, 0], [-5, 5, 0]], "faces": [[0, 1, 2], [0, 2, 3]],
            "material_id": 1}
    return {"meshes": [quad], "materials": [air, light],
            "camera": {"origin": [0, 0, 3], "lookat": [0, 0, 0], "up": [0, 1, 0]}}


def test_direct_view_of_emitter_known_answer():
    """Camera ray straight onto a light: deposit = emission * (1/(1+1e-6))^2 (main.py:1270-1275, 1552-1557)."""
    em = np.linspace(1.0, 25.0, 25)
    scene = _emitter_scene(em)
    cfg = sb.RenderConfig(width=8, height=8, max_path_length=3)
    comp = sb.compile_scene(scene, 25)
    bvh = orc.build_bvh_sweep(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    bvh["tri_perm"] = bvh.pop("perm")
    sc = oracle_scene(comp, bvh, scene["camera"])
    ocfg = oracle_config(cfg)
    for band in (0, 7, 24):
        out, st = orc.render_pass(sc, ocfg, 0, band, np.arange(64), use_double=True)
        want = em[band] / (1 + 1e-6) ** 2
        assert np.allclose(out[:, band], want, rtol=1e-12)
        assert np.count_nonzero(out) == 64


def test_render_pass_is_deterministic_and_stream_dependent():
    from spectral_b200 import configs
    scene, cfg, ex = configs.box_scene(width=16, height=16)
    comp = sb.compile_scene(scene, cfg.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = orc.build_bvh_sweep(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    bvh["tri_perm"] = bvh.pop("perm")
    sc = oracle_scene(comp, bvh, scene["camera"])
    ocfg = oracle_config(cfg)
    a, _ = orc.render_pass(sc, ocfg, 5, 3, np.arange(256))
    b, _ = orc.render_pass(sc, ocfg, 5, 3, np.arange(256), nthreads=1)
    c, _ = orc.render_pass(sc, ocfg, 6, 3, np.arange(256))
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    assert np.isfinite(a).all()


def test_fp32_and_fp64_estimators_agree_statistically():
    from spectral_b200 import configs
    scene, cfg, ex = configs.box_scene(width=8, height=8)
    comp = sb.compile_scene(scene, cfg.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = orc.build_bvh_sweep(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    bvh["tri_perm"] = bvh.pop("perm")
    sc = oracle_scene(comp, bvh, scene["camera"])
    ocfg = oracle_config(cfg)
    pix = np.arange(64)
    f32 = np.zeros((64, 25))
    f64 = np.zeros((64, 25))
    for p in range(25 * 8):
        orc.render_pass(sc, ocfg, p, p % 25, pix, out=f32)
        orc.render_pass(sc, ocfg, p, p % 25, pix, out=f64, use_double=True)
    # same random streams: the totals agree to within the paths that branch differently
    assert abs(f32.sum() - f64.sum()) <= 2e-2 * f64.sum()
