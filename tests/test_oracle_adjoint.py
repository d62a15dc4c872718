"""The oracle's forward-mode adjoint (CPU, no GPU): it follows the FP64
estimator exactly and its gradient equals finite differences of the FP64
oracle with common random numbers wherever the parameter moves no sampling
decision (wall albedo through k, emission, wall scattering)."""
import numpy as np
import pytest

from helpers import orc, oracle_config, oracle_scene, sb
from spectral_b200 import configs


@pytest.fixture(scope="module")
def small_volume():
    s, c, ex = configs.volume_scene(width=20, height=20, medium_slices=12, medium_stacks=13, fluorescent_medium=True,
                                    depth=8)
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    sc = oracle_scene(comp, bvh, s["camera"])
    return sc, oracle_config(c), c, comp


def test_dual_values_equal_fp64_film(small_volume):
    sc, oc, c, comp = small_volume
    npix, B, M = c.width * c.height, c.bands, comp.mat_f32.shape[0]
    adj = np.ones((npix, B))
    a = np.zeros((npix, B))
    b = np.zeros((npix, B))
    ids = [orc.param_index(M, B, 5, 1, 3)]
    for p in range(5):
        orc.render_pass(sc, oc, p, p % B, np.arange(npix), out=a, use_double=True)
        orc.adjoint_pass(sc, oc, p, p % B, np.arange(npix), adj, ids, out=b)
    assert np.array_equal(a, b)


def test_smooth_parameters_match_finite_differences(small_volume):
    sc, oc, c, comp = small_volume
    npix, B, M = c.width * c.height, c.bands, comp.mat_f32.shape[0]
    adj = np.random.default_rng(0).uniform(0.5, 1.5, size=(npix, B))
    pix = np.arange(npix)
    passes = range(25)
    params = [orc.param_index(M, B, 5, 1, 10),   # left wall k (its albedo)
              orc.param_index(M, B, 5, 1, 20),
              orc.param_index(M, B, 7, 4, 10),   # light emission
              orc.param_index(M, B, 6, 3, 10),   # right wall sigma_s
              orc.param_index(M, B, 8, 4, 10)]   # medium emission
    g = np.zeros(len(params))
    for p in passes:
        orc.adjoint_pass(sc, oc, p, p % B, pix, adj, params, grad=g)
    mat = sc._keep["mat_f32"].reshape(-1)

    def loss():
        out = np.zeros((npix, B))
        for p in passes:
            orc.render_pass(sc, oc, p, p % B, pix, out=out, use_double=True)
        return float((out * adj).sum())

    for gi, i in zip(g, params):
        v0 = float(mat[i])
        h = 1e-3 * abs(v0) if v0 != 0 else 1e-4
        mat[i] = np.float32(v0 + h)
        hp = float(mat[i]) - v0
        lp = loss()
        mat[i] = np.float32(v0 - h)
        hm = v0 - float(mat[i])
        lm = loss()
        mat[i] = np.float32(v0)
        fd = (lp - lm) / (hp + hm)
        assert abs(gi - fd) <= 2e-3 * abs(fd), (i, gi, fd)
