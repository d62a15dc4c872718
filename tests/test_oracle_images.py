"""The FP64 oracle reference images (tests/golden/oracle_*.npz) are what the
oracle renders: a fresh FP64 render of a few of their pixels, on other random
streams, agrees with them within the combined Monte Carlo error."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, orc, oracle_config, oracle_scene, sb
from spectral_b200 import configs


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"oracle_{name}.npz")))


@pytest.mark.parametrize("name", ["box", "terrain", "volume"])
def test_fixture_shapes(name):
    d = load(name)
    P = d["pixels"].shape[0]
    assert d["mean"].shape == (P, 25) and d["sem"].shape == (P, 25) and d["xyz"].shape == (P, 3)
    assert int(d["spp"]) >= 64000 and np.isfinite(d["mean"]).all() and (d["sem"] >= 0).all()


def test_box_fixture_matches_a_fresh_oracle_render():
    d = load("box")
    s, c, ex = configs.box_scene()
    comp = sb.compile_scene(s, c.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    c.seed = 4242  # streams independent of the fixture's
    sc, oc = oracle_scene(comp, bvh, s["camera"]), oracle_config(c)
    pick = np.arange(0, d["pixels"].shape[0], 64)  # 64 of the 4096 pixels
    pix = d["pixels"][pick]
    blocks = 120
    B = c.bands
    acc = np.zeros((pix.shape[0], B))
    sq = np.zeros((pix.shape[0], B))
    for b in range(blocks):
        blk = np.zeros((pix.shape[0], B))
        for k in range(B):
            orc.render_pass(sc, oc, b * B + k, k, pix, out=blk, use_double=True)
        acc += blk
        sq += blk * blk
    mean = acc / blocks
    sem = np.sqrt(np.maximum(sq / blocks - mean * mean, 0) / (blocks - 1))
    diff = mean - d["mean"][pick]
    tot = np.sqrt(sem ** 2 + d["sem"][pick].astype(np.float64) ** 2)
    ok = np.abs(diff) <= 3 * tot + 1e-12
    assert ok.mean() > 0.97, ok.mean()
    # the sums over all cells agree within 4 combined standard errors
    assert abs(diff.sum()) <= 4 * np.sqrt((tot ** 2).sum())
