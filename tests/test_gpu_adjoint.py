"""The path-replay adjoint kernel (ts_adjoint_pass) against the oracle's
forward-mode adjoint on identical paths, against finite differences of the
GPU renderer with common random numbers, and through torch.autograd."""
import numpy as np
import pytest
import torch

from helpers import orc, oracle_config, oracle_scene, sb
from spectral_b200 import autodiff, configs

pytestmark = pytest.mark.gpu


def volume_setup(W, depth=8, slices=12):
    s, c, ex = configs.volume_scene(width=W, height=W, medium_slices=slices, medium_stacks=slices + 1,
                                    fluorescent_medium=True, depth=depth)
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    c.kernel = "mega"
    return s, c, ex, comp, bvh


def named_params(M, B, b=10):
    """(name, index): medium (material 8), walls (3 fluorescent back, 5 left, 6 right),
    light (7), air (0) and the fluorescent EEM (1)."""
    P = orc.param_index
    return [("medium k", P(M, B, 8, 1, b)), ("medium sigma_s", P(M, B, 8, 3, b)), ("medium g", P(M, B, 8, 5, b)),
            ("medium roughness", P(M, B, 8, 2, b)), ("medium emission", P(M, B, 8, 4, b)),
            ("left k", P(M, B, 5, 1, b)), ("left roughness", P(M, B, 5, 2, b)), ("back k", P(M, B, 3, 1, b)),
            ("light emission", P(M, B, 7, 4, b)), ("right sigma_s", P(M, B, 6, 3, b)),
            ("air k", P(M, B, 0, 1, b)), ("medium k band 3", P(M, B, 8, 1, 3)),
            ("left k band 20", P(M, B, 5, 1, 20)), ("medium sigma_s band 17", P(M, B, 8, 3, 17)),
            ("eem 10->14", orc.eem_param_index(M, B, 1, 10, 14)), ("eem 10->10", orc.eem_param_index(M, B, 1, 10, 10))]


def test_adjoint_equals_oracle_adjoint_on_identical_paths():
    s, c, ex, comp, bvh = volume_setup(24)
    B, M = c.bands, comp.mat_f32.shape[0]
    npix = c.width * c.height
    adj_np = np.random.default_rng(0).uniform(0.5, 1.5, size=(npix, B))
    adj = torch.tensor(adj_np.T.reshape(B, c.height, c.width).copy(), dtype=torch.float64, device="cuda")
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        pm, pe = r.param_count()
        assert (pm, pe) == (M * 6 * B, comp.eem.shape[0] * B * B)
        grad = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
        for p in range(25):
            r.adjoint_pass(p % B, p, adj, grad)
        assert r.check_device() == 0
        g = grad.cpu().numpy()
    params = named_params(M, B)
    ids = [i for _, i in params]
    sc, oc = oracle_scene(comp, bvh, s["camera"]), oracle_config(c)
    g32, g64 = np.zeros(len(ids)), np.zeros(len(ids))
    for p in range(25):
        orc.adjoint_pass(sc, oc, p, p % B, np.arange(npix), adj_np, ids, grad=g32, use_double=False)
        orc.adjoint_pass(sc, oc, p, p % B, np.arange(npix), adj_np, ids, grad=g64, use_double=True)
    assert np.isfinite(g).all()
    for (name, i), o32, o64 in zip(params, g32, g64):
        # FP32 oracle: the same float paths; FP64: the same paths, rounding apart
        assert abs(g[i] - o32) <= 1e-3 * abs(o32) + 1e-12, (name, g[i], o32)
        assert abs(g[i] - o64) <= 5e-3 * abs(o64) + 1e-12, (name, g[i], o64)


def gpu_loss(r, adj, mat, eem, p0, npasses):
    r.update_materials(mat, eem)
    r.clear_pixel_space()
    B = r.config.bands
    for p in range(p0, p0 + npasses):
        r.cast_rays(p % B, pass_idx=p)
    return float((r.block_film * adj).sum())


def test_adjoint_matches_finite_differences():
    """Central differences of the rendered loss (common random numbers, h = 1e-2
    relative) in batches of passes; the adjoint over the same passes must agree
    within the batches' combined standard error (decisions that flip under the
    perturbation make the differences noisy), and within 1 % where no sampling
    decision depends on the parameter."""
    s, c, ex, comp, bvh = volume_setup(128)
    B, M = c.bands, comp.mat_f32.shape[0]
    smooth = {"left k", "light emission", "right sigma_s", "medium emission"}
    checked = ["medium k", "medium sigma_s", "medium g", "eem 10->14", "left k", "light emission", "right sigma_s",
               "left roughness"]
    params = [(n, i) for n, i in named_params(M, B) if n in checked]
    nb, npasses = 8, 100
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        pm, pe = r.param_count()
        adj = torch.tensor(np.random.default_rng(1).uniform(0.5, 1.5, size=(B, c.height, c.width)),
                           dtype=torch.float64, device="cuda")
        mat0 = torch.tensor(comp.mat_f32, dtype=torch.float32, device="cuda")
        eem0 = torch.tensor(comp.eem, dtype=torch.float32, device="cuda")
        ad = {n: [] for n, _ in params}
        fd = {n: [] for n, _ in params}
        for bi in range(nb):
            p0 = 5000 + bi * npasses
            r.update_materials(mat0, eem0)
            grad = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
            for p in range(p0, p0 + npasses):
                r.adjoint_pass(p % B, p, adj, grad)
            g = grad.cpu().numpy()
            for name, i in params:
                ad[name].append(g[i])
                mat, eem = mat0.clone(), eem0.clone()
                flat, j = (mat.view(-1), i) if i < pm else (eem.view(-1), i - pm)
                v0 = float(flat[j])
                h = 1e-2 * abs(v0)
                flat[j] = v0 + h
                hp = float(flat[j]) - v0
                lp = gpu_loss(r, adj, mat, eem, p0, npasses)
                flat[j] = v0 - h
                hm = v0 - float(flat[j])
                lm = gpu_loss(r, adj, mat, eem, p0, npasses)
                fd[name].append((lp - lm) / (hp + hm))
        assert r.check_device() == 0
    for name, _ in params:
        a, f = np.array(ad[name]), np.array(fd[name])
        if name in smooth:
            assert abs(a.mean() - f.mean()) <= 1e-2 * abs(f.mean()), (name, a.mean(), f.mean())
        else:
            se = np.hypot(a.std(ddof=1), f.std(ddof=1)) / np.sqrt(nb)
            assert abs(a.mean() - f.mean()) <= 4.0 * se, (name, a.mean(), f.mean(), se)


def test_autograd_render_film():
    s, c, ex, comp, bvh = volume_setup(32)
    B = c.bands
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        mat = autodiff.material_table(r).requires_grad_(True)
        eem = autodiff.eem_table(r).requires_grad_(True)
        film = autodiff.render_film(r, mat, eem, first_pass=50, num_blocks=2)
        assert film.shape == (B, c.height, c.width) and film.dtype == torch.float64
        # the same film as the plain render API
        r.clear_pixel_space()
        for k in range(2 * B):
            r.cast_rays(k % B, pass_idx=50 + k)
            if (k + 1) % B == 0:
                r.average_and_reset_block((k + 1) // B)
        # equal up to the order of the FP64 additions of fluorescence-shifted deposits
        assert torch.allclose(film, r.mean_film, rtol=1e-12, atol=0)
        xyz = autodiff.film_to_xyz(film, comp.cmf, r.cmf_scale)
        target = torch.zeros_like(xyz)
        loss = ((xyz - target) ** 2).sum()
        loss.backward()
        # backward equals a direct adjoint with dLoss/dfilm / num_blocks
        adj = (torch.einsum("hwc,bc->bhw", 2.0 * xyz.detach(), torch.as_tensor(comp.cmf, dtype=torch.float64,
                                                                                device="cuda")) * r.cmf_scale) / 2
        pm, pe = r.param_count()
        grad = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
        for k in range(2 * B):
            r.adjoint_pass(k % B, 50 + k, adj.contiguous(), grad)
        assert torch.allclose(mat.grad.double().view(-1), grad[:pm].float().double(), rtol=1e-5, atol=0)
        assert torch.allclose(eem.grad.double().view(-1), grad[pm:].float().double(), rtol=1e-5, atol=0)
        assert torch.count_nonzero(mat.grad[:, 0, :]) == 0  # refractive index: not differentiable
        assert r.check_device() == 0


def test_update_materials_replaces_tables():
    s, c, ex, comp, bvh = volume_setup(24)
    B = c.bands
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh) as r:
        def render():
            r.clear_pixel_space()
            for p in range(B):
                r.cast_rays(p, pass_idx=p)
            return r.block_film.clone()
        a = render()
        mat = torch.tensor(comp.mat_f32, device="cuda")
        eem = torch.tensor(comp.eem, device="cuda")
        r.update_materials(mat, eem)
        assert torch.equal(render(), a)  # same tables: the same image, bit for bit
        mat[7, 4, :] *= 2.0  # twice the light emission: every deposit doubles
        r.update_materials(mat, None)
        assert torch.allclose(render(), 2.0 * a, rtol=1e-6, atol=0)
        with pytest.raises(ValueError):
            r.update_materials(mat[:, :5].contiguous(), None)


@pytest.mark.parametrize("fluorescent", [False, True])
def test_recorded_forward_gives_the_same_gradient(fluorescent):
    """ts_record_paths: the adjoint of passes whose forward render recorded each
    path's total skips the weight replay for paths that stayed in their band
    (all of them without a fluorescent medium; the moved ones are replayed) --
    the same gradient as the two-replay adjoint, also after the records went
    stale (camera moved and back)."""
    from spectral_b200 import configs
    s, c, ex = configs.volume_scene(width=24, height=24, medium_slices=12, medium_stacks=13, depth=9,
                                    fluorescent_medium=fluorescent)
    c.kernel = "wavefront"  # recorded renders take the megakernel whatever the launch settings
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        B = c.bands
        pm, pe = r.param_count()
        adj = torch.rand((B, c.height, c.width), dtype=torch.float64, device="cuda")
        g0 = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
        r.adjoint_passes(0, 2 * B, 100, adj, g0)
        r.record_paths(100, 2 * B)
        for blk in range(2):
            r.cast_rays_bundle(0, B, pass_idx=100 + blk * B)
        film_rec = r.block_film.clone()
        g1 = torch.zeros_like(g0)
        r.adjoint_passes(0, 2 * B, 100, adj, g1)
        assert r.check_device() == 0
        scale = g0.abs().max()
        assert scale > 0
        assert torch.allclose(g1, g0, rtol=1e-4, atol=1e-7 * float(scale))
        # recording changed no image: the same passes without records
        r.record_paths(0, 0)
        r.clear_pixel_space()
        for blk in range(2):
            r.cast_rays_bundle(0, B, pass_idx=100 + blk * B)
        assert torch.allclose(r.block_film, film_rec, rtol=1e-12, atol=0)
        # stale records are not used
        r.record_paths(100, 2 * B)
        for blk in range(2):
            r.cast_rays_bundle(0, B, pass_idx=100 + blk * B)
        cam = s["camera"]
        r.update_camera([0.0, 0.1, 0.45], cam["lookat"], cam["up"])
        r.update_camera(cam["origin"], cam["lookat"], cam["up"])
        g2 = torch.zeros_like(g0)
        r.adjoint_passes(0, 2 * B, 100, adj, g2)
        assert torch.allclose(g2, g0, rtol=1e-9, atol=1e-12 * float(scale))  # FP64 atomics in another order
