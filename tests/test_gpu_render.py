"""Render parity of the CUDA estimator against the oracle, and the film API."""
import numpy as np
import pytest
import torch

from helpers import golden_compiled, orc, oracle_config, oracle_scene, sb
from spectral_b200 import configs, spectral_data as sd
from test_gpu_trace import renderer_for

pytestmark = pytest.mark.gpu


def setup(scene_fn, **kw):
    s, c, ex = scene_fn(**kw)
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    return s, c, ex, comp, bvh


def oracle_passes(comp, bvh, scene, cfg, passes, use_double=False):
    sc = oracle_scene(comp, bvh, scene["camera"])
    ocfg = oracle_config(cfg)
    npix = cfg.width * cfg.height
    out = np.zeros((npix, cfg.bands))
    for p in passes:
        orc.render_pass(sc, ocfg, p, p % cfg.bands, np.arange(npix), out=out, use_double=use_double)
    return out


def gpu_passes(scene, cfg, ex, bvh, kernel, passes, sort_keys=0, node_width=0, traversal="default",
               queue_capacity=0, quantize=False):
    c2 = sb.RenderConfig(**{**cfg.__dict__, "kernel": kernel, "sort_keys": sort_keys, "traversal": traversal,
                            "queue_capacity": queue_capacity})
    with sb.Renderer(scene, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh,
                     bvh_params={"width": node_width, "quantize": quantize}) as r:
        for p in passes:
            r.cast_rays(p % cfg.bands, pass_idx=p)
        g = r.block_film.cpu().numpy().reshape(cfg.bands, -1).T.copy()
        assert r.check_device() == 0
    return g


def crn_agreement(g, o):
    """Same random streams: totals agree, and nearly every cell agrees up to rounding.

    The GPU's transcendental functions round differently from the host libm's
    by an ulp or so; along long volume paths that drifts to ~1e-5, and a few
    paths take a different branch.  1e-3 separates the two cases."""
    assert np.isfinite(g).all() and np.isfinite(o).all()
    assert abs(g.sum() - o.sum()) <= 2e-3 * abs(o.sum()) + 1e-9
    close = np.isclose(g, o, rtol=1e-3, atol=1e-9)
    assert close.mean() > 0.995, close.mean()


@pytest.mark.parametrize("kernel,node_width", [("mega", 2), ("wavefront", 2), ("mega", 4), ("wavefront", 8)])
def test_box_scene_common_random_numbers(kernel, node_width):
    s, c, ex, comp, bvh = setup(configs.box_scene, width=48, height=48)
    passes = range(25)
    crn_agreement(gpu_passes(s, c, ex, bvh, kernel, passes, node_width=node_width),
                  oracle_passes(comp, bvh, s, c, passes))


@pytest.mark.parametrize("kernel,node_width", [("mega", 2), ("wavefront", 4), ("mega", 8)])
def test_volume_fluorescence_common_random_numbers(kernel, node_width):
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=40, height=40, medium_slices=30, medium_stacks=31,
                                fluorescent_medium=True, depth=16)
    passes = range(25)
    crn_agreement(gpu_passes(s, c, ex, bvh, kernel, passes, node_width=node_width),
                  oracle_passes(comp, bvh, s, c, passes))


@pytest.mark.parametrize("kernel,node_width,quantize,qcap", [("mega", 2, False, 0), ("wavefront", 4, False, 0),
                                                             ("wavefront", 4, True, 64 * 64 * 25),
                                                             ("mega", 8, True, 0)])
def test_opaque_terrain_common_random_numbers(kernel, node_width, quantize, qcap):
    """An opaque scene (GGX conductors, a displaced sphere, eight area lights):
    every node layout, both renderers and the regenerating loop against the
    oracle with the same random streams."""
    s, c, ex, comp, bvh = setup(configs.terrain_scene, grid=96, sphere_slices=40, sphere_stacks=41, width=64,
                                height=64)
    passes = range(25)
    g = gpu_passes(s, c, ex, bvh, kernel, passes, node_width=node_width, quantize=quantize, queue_capacity=qcap)
    crn_agreement(g, oracle_passes(comp, bvh, s, c, passes))
    assert g.sum() > 0


def test_reference_scene_common_random_numbers():
    """The reference's own scene, BVH, EEM (uv_green) and spectral grid."""
    cs, bvh, cam = golden_compiled()
    cfg = sb.RenderConfig(width=40, height=40)
    from test_gpu_trace import renderer_for
    r = renderer_for(cs, bvh, cam, width=40, height=40, kernel="wavefront")
    for p in range(25):
        r.cast_rays(p, pass_idx=p)
    g = r.block_film.cpu().numpy().reshape(25, -1).T.copy()
    r.close()
    sc = oracle_scene(cs, bvh, cam)
    ocfg = oracle_config(cfg)
    o = np.zeros((1600, 25))
    for p in range(25):
        orc.render_pass(sc, ocfg, p, p, np.arange(1600), out=o)
    crn_agreement(g, o)


def test_wavefront_equals_megakernel():
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=64, height=64, medium_slices=30, medium_stacks=31,
                                fluorescent_medium=True)
    passes = range(30)
    a = gpu_passes(s, c, ex, bvh, "mega", passes)
    b = gpu_passes(s, c, ex, bvh, "wavefront", passes)
    d = gpu_passes(s, c, ex, bvh, "wavefront", passes, sort_keys=1)
    # the same paths (no multiply-add contraction anywhere); only the order of
    # the FP64 film additions differs between the two kernels
    assert np.allclose(a, b, rtol=1e-12, atol=1e-15)
    # the order of a queue (shading by material; tracing by octant and by
    # light) never changes a path
    assert np.array_equal(b, d)
    assert np.array_equal(b, gpu_passes(s, c, ex, bvh, "wavefront", passes, sort_keys=7))
    # node widths and traversal loops change only which boxes are opened, never a result
    for w in (4, 8):
        e = gpu_passes(s, c, ex, bvh, "wavefront", passes, node_width=w)
        assert np.array_equal(b, e), w
    assert np.array_equal(b, gpu_passes(s, c, ex, bvh, "wavefront", passes, traversal="speculative"))
    assert np.array_equal(a, gpu_passes(s, c, ex, bvh, "mega", passes, traversal="speculative"))


def test_wavefront_queue_capacity_changes_no_result():
    """A pass over queue_capacity path slots -- the regenerating loop (unsorted
    queues), or depth-synchronous chunks of the frame with a ragged last chunk
    (sorted queues) -- deposits the same paths into the same cells as a
    whole-frame pass."""
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=64, height=64, medium_slices=30, medium_stacks=31,
                                fluorescent_medium=True)
    passes = range(10)
    whole = gpu_passes(s, c, ex, bvh, "wavefront", passes)
    for cap, sk in ((1000, 0), (777, 7), (4096, 1), (1 << 20, 0)):
        assert np.array_equal(whole, gpu_passes(s, c, ex, bvh, "wavefront", passes, sort_keys=sk,
                                                queue_capacity=cap)), cap
    # a capacity set after the first pass (buffers already sized for the whole frame)
    c2 = sb.RenderConfig(**{**c.__dict__, "kernel": "wavefront"})
    with sb.Renderer(s, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        for p in passes:
            if p == 3:
                r.set_launch_config(queue_capacity=513)
            r.cast_rays(p % c.bands, pass_idx=p)
        g = r.block_film.cpu().numpy().reshape(c.bands, -1).T.copy()
        assert r.check_device() == 0
        # 64*64 pixels over 513 slots: at least 8 slot generations of iterations
        assert 8 <= r.wave_loop_iterations() <= (64 * 64 // 513 + 3) * (c.max_path_length + 1) + 4
    assert np.array_equal(whole, g)


def gpu_bundles(scene, cfg, ex, bvh, kernel, bundles, queue_capacity=0, sort_keys=0, loop_host=0):
    """(first_pass, first_band, num_passes) launches into one film."""
    c2 = sb.RenderConfig(**{**cfg.__dict__, "kernel": kernel, "queue_capacity": queue_capacity,
                            "sort_keys": sort_keys, "loop_host": loop_host})
    with sb.Renderer(scene, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        for p0, b0, n in bundles:
            r.cast_rays_bundle(b0, n, pass_idx=p0)
        g = r.block_film.cpu().numpy().reshape(cfg.bands, -1).T.copy()
        assert r.check_device() == 0
    return g


def test_wavefront_regenerating_loop_single_pass():
    """queue_capacity > 0: a pass over fewer (or more) path slots than pixels,
    slots of ended paths starting the next pixels; the same paths and deposits
    as the depth-synchronous pass."""
    s, c, ex, comp, bvh = setup(configs.box_scene, width=48, height=48)
    passes = range(25)
    whole = gpu_passes(s, c, ex, bvh, "wavefront", passes)
    for cap in (1, 97, 1000, 48 * 48, 10000):
        assert np.array_equal(whole, gpu_passes(s, c, ex, bvh, "wavefront", passes, queue_capacity=cap)), cap


def test_wavefront_regenerating_loop_bundles():
    """A wavelength bundle through the wavefront loop: bit-identical to one pass
    per launch where no fluorescence moves deposits between bands; with it, the
    same deposits summed in another order."""
    s, c, ex, comp, bvh = setup(configs.box_scene, width=48, height=48)
    per_pass = gpu_passes(s, c, ex, bvh, "wavefront", range(50))
    for cap in (0, 500, 3 * 48 * 48):
        g = gpu_bundles(s, c, ex, bvh, "wavefront", [(0, 0, 25), (25, 0, 25)], queue_capacity=cap)
        assert np.array_equal(per_pass, g), cap
    # iterations launched from the host instead of the graph's while-loop
    g = gpu_bundles(s, c, ex, bvh, "wavefront", [(0, 0, 25), (25, 0, 25)], queue_capacity=500, loop_host=1)
    assert np.array_equal(per_pass, g)
    # bundles that start mid-block and wrap the band index
    per_pass = gpu_passes(s, c, ex, bvh, "wavefront", range(7, 27))
    assert np.array_equal(per_pass, gpu_bundles(s, c, ex, bvh, "wavefront", [(7, 7, 11), (18, 18, 9)],
                                                queue_capacity=300))
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=40, height=40, medium_slices=30, medium_stacks=31,
                                fluorescent_medium=True, depth=16)
    per_pass = gpu_passes(s, c, ex, bvh, "wavefront", range(25))
    mega = gpu_bundles(s, c, ex, bvh, "mega", [(0, 0, 25)])
    for cap in (0, 700, 10 * 1600):
        g = gpu_bundles(s, c, ex, bvh, "wavefront", [(0, 0, 25)], queue_capacity=cap)
        assert np.allclose(per_pass, g, rtol=1e-12, atol=1e-15), cap
        assert np.allclose(mega, g, rtol=1e-12, atol=1e-15), cap
    # sorted queues keep one launch per pass (depth-synchronous stages)
    assert np.array_equal(per_pass, gpu_bundles(s, c, ex, bvh, "wavefront", [(0, 0, 25)], sort_keys=1))


def test_wavefront_loop_follows_the_camera():
    """The captured loop takes the camera from its launch: a moved camera
    needs no new graph and renders the moved view."""
    s, c, ex, comp, bvh = setup(configs.box_scene, width=48, height=48)
    cam = s["camera"]
    moved = np.asarray(cam["origin"], np.float64) + np.array([0.35, -0.2, 0.1])
    films = []
    for bundle in (True, False):
        c2 = sb.RenderConfig(**{**c.__dict__, "kernel": "wavefront", "queue_capacity": 3 * 48 * 48})
        with sb.Renderer(s, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
            for blk, origin in enumerate((cam["origin"], moved, cam["origin"])):
                r.update_camera(origin, cam["lookat"], cam["up"])
                if bundle:
                    r.cast_rays_bundle(0, c.bands, pass_idx=blk * c.bands)
                else:
                    for b in range(c.bands):
                        r.cast_rays(b, pass_idx=blk * c.bands + b)
            films.append(r.block_film.cpu().numpy())
            assert r.check_device() == 0
    assert np.array_equal(films[0], films[1])


@pytest.mark.parametrize("kernel,cap", [("mega", 0), ("wavefront", 3 * 24 * 20)])
def test_render_bundles_whole_blocks(kernel, cap):
    """Renderer.render launches each whole block as one bundle: the films,
    counters and callbacks of the pass-by-pass cadence."""
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=24, height=20, medium_slices=12, medium_stacks=13,
                                fluorescent_medium=True, depth=8)
    B = c.bands
    c2 = sb.RenderConfig(**{**c.__dict__, "kernel": kernel, "queue_capacity": cap})
    out = []
    for bundles in (False, True):
        calls = []
        with sb.Renderer(s, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
            r.cast_rays(0)  # start off the block boundary: one single pass, then whole blocks
            r.render(2 * B + 7, callback=lambda rr: calls.append(rr.num_blocks_completed), bundles=bundles)
            out.append((r.mean_film.clone(), r.m2_film.clone(), r.block_film.clone(), r.total_samples,
                        r.num_blocks_completed, calls))
            assert r.check_device() == 0
    (m0, q0, b0, t0, n0, c0), (m1, q1, b1, t1, n1, c1) = out
    assert (t0, n0, c0) == (t1, n1, c1) == (2 * B + 8, 2, [1, 2])
    for a, b in ((m0, m1), (q0, q1), (b0, b1)):
        assert torch.allclose(a, b, rtol=1e-12, atol=0)


@pytest.mark.parametrize("kernel,cap", [("mega", 0), ("wavefront", 3 * 24 * 20)])
def test_deferred_passes_equal_immediate(kernel, cap):
    """defer_passes: the reference's pass-by-pass cadence, queued and launched
    as bundles -- with a film read mid-block and a camera move mid-block, which
    flush the queue -- renders the same films."""
    s, c, ex, comp, bvh = setup(configs.volume_scene, width=24, height=20, medium_slices=12, medium_stacks=13,
                                fluorescent_medium=True, depth=8)
    B = c.bands
    cam = s["camera"]
    moved = np.asarray(cam["origin"], np.float64) + np.array([0.2, 0.1, -0.1])
    out = []
    for defer in (False, True):
        c2 = sb.RenderConfig(**{**c.__dict__, "kernel": kernel, "queue_capacity": cap, "defer_passes": defer})
        with sb.Renderer(s, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
            mid = None
            for k in range(2 * B + 7):
                r.cast_rays(k % B)
                if k == 30:
                    mid = r.block_film.clone()
                if k == 40:
                    r.update_camera(moved, cam["lookat"], cam["up"])
                if (k + 1) % B == 0:
                    r.average_and_reset_block((k + 1) // B)
            out.append((r.mean_film.clone(), r.m2_film.clone(), r.block_film.clone(), mid, r.total_samples))
            assert r.check_device() == 0
    (a0, a1, a2, a3, t0), (b0, b1, b2, b3, t1) = out
    assert t0 == t1 == 2 * B + 7
    for x, y in ((a0, b0), (a1, b1), (a2, b2), (a3, b3)):
        assert torch.allclose(x, y, rtol=1e-12, atol=0)


def test_statistical_parity_three_sigma():
    """Independent streams: per-cell means agree within 3 combined standard errors."""
    s, c, ex, comp, bvh = setup(configs.box_scene, width=16, height=16)
    nb = 24
    B = c.bands
    c2 = sb.RenderConfig(**{**c.__dict__, "kernel": "wavefront", "seed": 1234})
    with sb.Renderer(s, c2, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        r.render(nb * B)
        mg = r.mean_film.cpu().numpy().reshape(B, -1).T
        seg = r.standard_error().cpu().numpy().reshape(B, -1).T
    sc = oracle_scene(comp, bvh, s["camera"])
    ocfg = oracle_config(c)
    npix = c.width * c.height
    blocks = np.zeros((nb, npix, B))
    for b in range(nb):
        for k in range(B):
            orc.render_pass(sc, ocfg, b * B + k, k, np.arange(npix), out=blocks[b])
    mo = blocks.mean(0)
    seo = blocks.std(0, ddof=1) / np.sqrt(nb)
    se = np.sqrt(seg ** 2 + seo ** 2)
    ok = se > 0
    z = np.abs(mg - mo)[ok] / se[ok]
    assert (z <= 3).mean() > 0.98, (z <= 3).mean()
    assert abs(mg.sum() - mo.sum()) <= 4 * np.sqrt((se ** 2).sum())


def test_accumulate_resolve_and_reset():
    s, c, ex, comp, bvh = setup(configs.box_scene, width=24, height=20)
    B = c.bands
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        blocks = []
        for b in range(3):
            for k in range(B):
                r.cast_rays(k)
            blocks.append(r.block_film.cpu().numpy().copy())
            r.average_and_reset_block(b + 1)
            assert np.all(r.block_film.cpu().numpy() == 0)
        mean = r.mean_film.cpu().numpy()
        m2 = r.m2_film.cpu().numpy()
        want = ((blocks[0] * 1 + blocks[1]) / 2 * 2 + blocks[2]) / 3
        assert np.allclose(mean, want, rtol=1e-12, atol=1e-14)
        assert np.allclose(m2, sum(b * b for b in blocks), rtol=1e-12, atol=1e-14)
        # spectral_accumulator uses the reference's [i, j, k] indexing
        assert r.spectral_accumulator.shape == (24, 20, B)
        assert r.spectral_accumulator[5, 7, 3].item() == mean[3, 7, 5]
        # XYZ (color_rays, first half)
        xyz = r.resolve_xyz().cpu().numpy()
        cmf = ex["cmf"].astype(np.float32).astype(np.float64)
        want_xyz = np.einsum("bhw,bc->hwc", mean, cmf) * r.cmf_scale
        assert np.allclose(xyz, want_xyz, rtol=1e-5, atol=1e-7)
        host = r.resolve_xyz_host()
        assert np.array_equal(host, xyz)
        # full color_rays at a display resolution with nearest upscale
        r.config.image_width, r.config.image_height = 48, 40
        rgb = r.color_rays().cpu().numpy()
        T = sd.srgb_xyz_to_rgb()
        i = np.arange(48)
        j = np.arange(40)
        ri = (i.astype(np.float32) / np.float32(48) * np.float32(24)).astype(int)
        rj = (j.astype(np.float32) / np.float32(40) * np.float32(20)).astype(int)
        up = want_xyz[rj][:, ri]
        hdr = np.einsum("ij,hwj->hwi", T, up)
        with np.errstate(invalid="ignore"):
            want_rgb = (hdr / (hdr + 1.0)) ** 0.5
        fin = np.isfinite(want_rgb)
        assert np.allclose(rgb[fin], want_rgb[fin], rtol=1e-4, atol=1e-5)
        r.clear_pixel_space()
        for f in (r.block_film, r.mean_film, r.m2_film):
            assert torch.count_nonzero(f).item() == 0


def test_visualize_normals_matches_trace():
    s, c, ex, comp, bvh = setup(configs.box_scene, width=32, height=32)
    from helpers import camera_rays
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        nrm = r.visualize_normals().cpu().numpy().reshape(-1, 3)
    sc = oracle_scene(comp, bvh, s["camera"])
    rays = camera_rays(s["camera"], 32, 32, fov_scale=c.fov_scale)
    tri, t, u, v = orc.trace(sc, oracle_config(c), rays)
    perm = bvh["tri_perm"]
    hit = tri >= 0
    assert np.array_equal(hit, nrm.sum(1) > 0)
    slots = tri[hit]
    n0, n1, n2 = (comp.tris[k][perm[slots]] for k in ("n0", "n1", "n2"))
    w = 1 - u[hit] - v[hit]
    ns = w[:, None] * n0 + u[hit][:, None] * n1 + v[hit][:, None] * n2
    ns /= np.linalg.norm(ns, axis=1, keepdims=True)
    assert np.allclose(nrm[hit], ns * 0.5 + 0.5, atol=2e-6)


def test_counted_pass_matches_plain_pass():
    s, c, ex, comp, bvh = setup(configs.box_scene, width=32, height=32)
    with sb.Renderer(s, sb.RenderConfig(**{**c.__dict__, "kernel": "mega"}), eems=ex["eems"], cmf=ex["cmf"],
                     bvh=bvh) as r:
        r.cast_rays(5, pass_idx=9)
        a = r.block_film.cpu().numpy().copy()
        r.clear_pixel_space()
        w = r.cast_rays_counted(5, pass_idx=9)
        b = r.block_film.cpu().numpy()
    assert np.array_equal(a, b)
    assert w["paths"] == 32 * 32 and w["traces"] >= w["vertices"] >= w["paths"] // 2
    assert w["node_visits"] > w["traces"] and w["tri_tests"] > 0


def test_invalid_arguments_raise():
    s, c, ex, comp, bvh = setup(configs.box_scene, width=8, height=8)
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        with pytest.raises(sb.SpectralError, match="band out of range"):
            r.cast_rays(25)
        with pytest.raises(sb.SpectralError, match="num_blocks_completed"):
            r.average_and_reset_block(0)
        bad = dict(s)
        bad["meshes"] = [dict(s["meshes"][0], material_id=99)]
        with pytest.raises(sb.SpectralError, match="material id 99"):
            r.setup_scene(bad, eems=ex["eems"], cmf=ex["cmf"])
        bad2 = {"meshes": [dict(s["meshes"][0])], "materials": [dict(m) for m in s["materials"]]}
        bad2["materials"][1] = dict(bad2["materials"][1], eem_id=3)
        with pytest.raises(sb.SpectralError, match="EEM"):
            r.setup_scene(bad2, eems=np.zeros((2, 25, 25)), cmf=ex["cmf"])
        nan = dict(s)
        m0 = dict(s["meshes"][0])
        m0["vertices"] = np.array(m0["vertices"], np.float64)
        m0["vertices"][0, 0] = np.nan
        nan["meshes"] = [m0]
        with pytest.raises(sb.SpectralError, match="non-finite"):
            r.setup_scene(nan, eems=ex["eems"], cmf=ex["cmf"])
        with pytest.raises(sb.SpectralError, match="negative queue_capacity"):
            r.set_launch_config(queue_capacity=-1)
        # the context stays usable after rejected uploads
        r.setup_scene(s, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh)
        r.cast_rays(3)
        assert r.check_device() == 0


def test_scene_without_lights_renders_zero():
    s, c, ex = configs.box_scene(width=16, height=16)
    s = dict(s)
    s["meshes"] = [m for m in s["meshes"] if not s["materials"][m["material_id"]]["surface_emission"][0]]
    for kernel in ("mega", "wavefront"):
        with sb.Renderer(s, sb.RenderConfig(**{**c.__dict__, "kernel": kernel}), eems=ex["eems"],
                         cmf=ex["cmf"]) as r:
            for k in range(25):
                r.cast_rays(k)
            assert torch.count_nonzero(r.block_film).item() == 0
