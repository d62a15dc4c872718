"""Converged GPU images against the FP64 oracle images: per pixel and band
within 3 standard errors of the combined Monte Carlo error (independent
random streams), and image totals within 4."""
import os

import numpy as np
import pytest
import torch

from helpers import GOLDEN, sb
from spectral_b200 import configs

pytestmark = pytest.mark.gpu


# Per-cell coverage of the 3-sigma band converges slowly where the path
# contributions are heavy-tailed: a cell whose sample missed its rare bright
# paths has both a low mean and a low variance estimate.  Measured on the
# volume scene: 94.9 % at 24 blocks, 96.4 % at 48, 97.4 % at 96, 98.4 % at 192,
# with the image total unbiased throughout (z within +-0.7).
@pytest.mark.parametrize("name,fn,blocks,coverage", [("box", configs.box_scene, 160, 0.98),
                                                    ("volume", configs.volume_scene, 48, 0.95)])
def test_converged_image_within_3_sigma_of_oracle(name, fn, blocks, coverage):
    d = dict(np.load(os.path.join(GOLDEN, f"oracle_{name}.npz")))
    s, c, ex = fn()
    c.kernel = "mega"
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        B = c.bands
        for b in range(blocks):
            r.cast_rays_bundle(0, B, pass_idx=b * B)
            r.average_and_reset_block(b + 1)
        n = blocks
        pix = torch.as_tensor(d["pixels"].astype(np.int64), device="cuda")
        mean = r.mean_film.reshape(B, -1)[:, pix].T.cpu().numpy()
        m2 = r.m2_film.reshape(B, -1)[:, pix].T.cpu().numpy()
        assert r.check_device() == 0
    sem = np.sqrt(np.maximum(m2 / n - mean * mean, 0) / (n - 1))
    diff = mean - d["mean"].astype(np.float64)
    tot = np.sqrt(sem ** 2 + d["sem"].astype(np.float64) ** 2)
    ok = np.abs(diff) <= 3 * tot + 1e-12
    assert ok.mean() > coverage, ok.mean()
    assert abs(diff.sum()) <= 4 * np.sqrt((tot ** 2).sum()), (diff.sum(), np.sqrt((tot ** 2).sum()))
