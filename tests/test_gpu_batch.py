"""Wavelength bundles (ts_render_passes, ts_adjoint_passes) and the multi-scene
batch (ts_batch_*): the same paths as one pass per launch on one scene."""
import pytest
import torch

from helpers import sb
from spectral_b200 import batch as sbatch
from spectral_b200 import configs

pytestmark = pytest.mark.gpu


def make(scene_fn, **kw):
    s, c, ex = scene_fn(**kw)
    c.kernel = "mega"
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    return s, c, ex, bvh


def renderer(args):
    s, c, ex, bvh = args
    return sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh)


def same_film(a, b):
    """Equal up to the order of FP64 additions (volume fluorescence lets two passes of
    one launch deposit into the same cell, which they add atomically in either order)."""
    return torch.allclose(a, b, rtol=1e-12, atol=0)


def single_scene_mean(args, blocks, first_pass=0):
    with renderer(args) as r:
        B = r.config.bands
        for blk in range(blocks):
            for k in range(B):
                r.cast_rays(k, pass_idx=first_pass + blk * B + k)
            r.average_and_reset_block(blk + 1)
        out = (r.mean_film.clone(), r.m2_film.clone())
        assert r.check_device() == 0
    return out


SCENES = [
    (configs.box_scene, dict(width=32, height=24, depth=5)),
    (configs.volume_scene, dict(width=24, height=24, medium_slices=12, medium_stacks=13, fluorescent_medium=True,
                                depth=9)),
    (configs.box_scene, dict(width=16, height=16, depth=12, sphere_slices=12, sphere_stacks=13)),
]


def test_bundle_equals_single_passes():
    args = make(SCENES[1][0], **SCENES[1][1])
    ref = single_scene_mean(args, 2, first_pass=40)
    with renderer(args) as r:
        B = r.config.bands
        for blk in range(2):
            r.cast_rays_bundle(0, B, pass_idx=40 + blk * B)
            r.average_and_reset_block(blk + 1)
        assert same_film(r.mean_film, ref[0]) and same_film(r.m2_film, ref[1])
        # a partial bundle from the middle of the band range, wrapping past the last band
        r.clear_pixel_space()
        r.cast_rays_bundle(20, 10, pass_idx=7)
        a = r.block_film.clone()
        r.clear_pixel_space()
        for i in range(10):
            r.cast_rays((20 + i) % B, pass_idx=7 + i)
        assert same_film(r.block_film, a)
        with pytest.raises(sb.SpectralError):
            r.cast_rays_bundle(0, B + 1, pass_idx=0)


def test_adjoint_bundle_equals_single_passes():
    args = make(SCENES[1][0], **SCENES[1][1])
    with renderer(args) as r:
        B = r.config.bands
        pm, pe = r.param_count()
        adj = torch.rand((B, r.config.height, r.config.width), dtype=torch.float64, device="cuda")
        g1 = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
        g2 = torch.zeros_like(g1)
        for p in range(60):
            r.adjoint_pass((3 + p) % B, 11 + p, adj, g1)
        r.adjoint_passes(3, 60, 11, adj, g2)
        # the same path terms; only the order of the FP64 atomic sums differs
        assert torch.allclose(g1, g2, rtol=1e-9, atol=1e-12 * float(g1.abs().max()))


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_single_scene_renders(use_graph):
    args = [make(fn, **kw) for fn, kw in SCENES]
    refs = [single_scene_mean(a, 3, first_pass=25) for a in args]
    rs = [renderer(a) for a in args]
    with sbatch.Batch(rs, use_graph=use_graph) as b:
        b.reset(first_pass=25)
        for _ in range(3):
            b.step()
        assert b.check() == 0
        for i, (r, (mean, m2)) in enumerate(zip(rs, refs)):
            if i == 1:  # fluorescent medium
                assert same_film(r.mean_film, mean) and same_film(r.m2_film, m2)
            else:  # one deposit per cell and launch: bit for bit
                assert torch.equal(r.mean_film, mean) and torch.equal(r.m2_film, m2)
        # an inactive scene keeps its film while the others advance
        keep = rs[1].mean_film.clone()
        b.set_active([True, False, True])
        b.step()
        assert torch.equal(rs[1].mean_film, keep)
        assert list(b.blocks) == [4, 3, 4]
        ref4 = single_scene_mean(args[0], 4, first_pass=25)
        assert torch.equal(rs[0].mean_film, ref4[0])
    for r in rs:
        r.close()


def test_render_to_rmse_stops_each_scene():
    args = [make(fn, **kw) for fn, kw in SCENES[:2]]
    rs = [renderer(a) for a in args]
    with sbatch.Batch(rs) as b:
        b.reset()
        blocks, secs = b.render_to_rmse(target=0.05, max_blocks=200)
        assert secs > 0
        for r, nb in zip(rs, blocks):
            assert 2 <= nb < 200
            assert sbatch.relative_rmse_estimate(r, int(nb)) <= 0.05
    for r in rs:
        r.close()


def test_batch_rejects_mixed_bvh_widths():
    a = make(SCENES[0][0], **SCENES[0][1])
    s, c, ex, _ = make(SCENES[2][0], **SCENES[2][1])
    r1 = renderer(a)
    r2 = sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh_params={"width": 4})
    with pytest.raises(sb.SpectralError):
        sbatch.Batch([r1, r2])
    r1.close()
    r2.close()


def test_stream_batch_equals_single_scene_renders():
    """Each scene's block as one regenerating-loop launch on a pool of streams:
    the films of one launch per pass, whatever BVH widths the scenes have."""
    args = [make(fn, **kw) for fn, kw in SCENES]
    refs = [single_scene_mean(a, 3, first_pass=25) for a in args]
    rs = [renderer(a) for a in args[:2]]
    s, c, ex, bvh = args[2]
    rs.append(sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh, bvh_params={"width": 4}))
    with sbatch.StreamBatch(rs, streams=2) as b:
        b.reset(first_pass=25)
        for _ in range(3):
            b.step()
        assert b.check() == 0
        for i, (r, (mean, m2)) in enumerate(zip(rs, refs)):
            assert r.config.kernel == "wavefront" and r.config.queue_capacity > 0
            if i == 1:  # fluorescent medium
                assert same_film(r.mean_film, mean) and same_film(r.m2_film, m2)
            else:
                assert torch.equal(r.mean_film, mean) and torch.equal(r.m2_film, m2)
        keep = rs[1].mean_film.clone()
        b.set_active([True, False, True])
        b.step()
        b.synchronize()
        assert torch.equal(rs[1].mean_film, keep)
        assert list(b.blocks) == [4, 3, 4]
        ref4 = single_scene_mean(args[0], 4, first_pass=25)
        assert torch.equal(rs[0].mean_film, ref4[0])
        b.reset()
        blocks, secs = b.render_to_rmse(target=0.05, max_blocks=200)
        for r, nb in zip(rs, blocks):
            assert 2 <= nb < 200
            assert sbatch.relative_rmse_estimate(r, int(nb)) <= 0.05
    for r in rs:
        r.close()


@pytest.mark.parametrize("queue_capacity,use_graph", [(0, True), (3000, True), (3000, False)])
def test_batch_loop_equals_single_scene_renders(queue_capacity, use_graph):
    """The batch loop (every scene's block in one regenerating wavefront loop,
    the step one CUDA graph) gives each scene the films of its own single-pass
    renders -- with path slots for all items, and with a few thousand slots that
    the scenes' items regenerate through."""
    scenes = [make(fn, **kw) for fn, kw in SCENES]
    refs = [single_scene_mean(a, 2, first_pass=30) for a in scenes]
    rs = [renderer(a) for a in scenes]
    try:
        with sbatch.Batch(rs, kernel="wavefront", queue_capacity=queue_capacity, use_graph=use_graph) as b:
            b.reset(first_pass=30)
            b.step()
            b.step()
            assert b.check() == 0
            for r, (mean, m2) in zip(rs, refs):
                assert same_film(r.mean_film, mean) and same_film(r.m2_film, m2)
            # inactive scenes keep their films; the others go on
            before = [r.mean_film.clone() for r in rs]
            b.set_active([1, 0, 1])
            b.step()
            assert b.check() == 0
            assert torch.equal(rs[1].mean_film, before[1])
            assert not torch.equal(rs[0].mean_film, before[0])
    finally:
        for r in rs:
            r.close()


def test_views_share_one_scene_and_batch_together():
    """A view renders the owner's scene through its own camera, resolution and
    film without a second upload: the same film as a separate context holding
    the same scene and camera, alone and in a batch loop with its owner."""
    import dataclasses
    args = make(configs.box_scene, width=32, height=24, depth=5)
    s, c, ex, bvh = args
    cam2 = {"origin": [0.2, 0.1, 0.45], "lookat": [0.0, -0.1, -0.5], "up": [0.0, 1.0, 0.0]}
    c2 = dataclasses.replace(c, width=40, height=30, seed=5, scene_id=3)
    ref_owner = single_scene_mean(args, 1, first_pass=10)
    ref_view = single_scene_mean((dict(s, camera=cam2), c2, ex, bvh), 1, first_pass=10)
    with renderer(args) as r:
        v = r.view(c2, camera=cam2)
        try:
            assert v.scene_info()["device_bytes"] < r.scene_info()["device_bytes"]
            B = c.bands
            for k in range(B):
                v.cast_rays(k, pass_idx=10 + k)
            v.average_and_reset_block(1)
            assert same_film(v.mean_film, ref_view[0])
            for kernel in ("wavefront", "mega"):
                with sbatch.Batch([r, v], kernel=kernel) as b:
                    b.reset(first_pass=10)
                    b.step()
                    assert b.check() == 0
                    assert same_film(r.mean_film, ref_owner[0]) and same_film(v.mean_film, ref_view[0])
        finally:
            v.close()
