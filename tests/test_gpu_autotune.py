"""The autotuner times launch candidates; tuning changes cost, never the image."""
import pytest
import torch

from helpers import sb
from spectral_b200 import autotune, configs
from spectral_b200 import batch as sbatch

pytestmark = pytest.mark.gpu


def test_tune_picks_a_candidate_and_keeps_the_image(tmp_path):
    s, c, ex = configs.box_scene(width=48, height=48, depth=6)
    cands = [autotune.Candidate(2, "default", "mega", 128, 0), autotune.Candidate(4, "default", "mega", 64, 5),
             autotune.Candidate(8, "default", "mega", 128, 5), autotune.Candidate(2, "speculative", "mega", 128, 0),
             autotune.Candidate(2, "default", "wavefront", 128, 0, 1, 16),
             autotune.Candidate(4, "default", "mega", 128, 0, occupancy=8)]
    cache = str(tmp_path / "tune.json")
    best, table = autotune.tune(s, c, eems=ex["eems"], cmf=ex["cmf"], candidates=cands, passes=3, cache=cache)
    assert best in cands and len(table) == len(cands) and all(ms > 0 for _, ms in table)
    again, _ = autotune.tune(s, c, eems=ex["eems"], cmf=ex["cmf"], candidates=cands, cache=cache)
    assert again == best  # from the cache

    def film(cand):
        with sb.Renderer(s, cand.apply(c), eems=ex["eems"], cmf=ex["cmf"], bvh_params={"width": cand.width}) as r:
            for p in range(25):
                r.cast_rays(p, pass_idx=p)
            assert r.check_device() == 0
            return r.block_film.clone()

    ref = film(cands[0])
    for cand in cands[1:]:
        assert torch.allclose(film(cand), ref, rtol=1e-12, atol=0), cand


def test_tune_batch():
    rs = []
    for fn, kw in ((configs.box_scene, dict(width=32, height=32, depth=5)),
                   (configs.box_scene, dict(width=16, height=24, depth=9, seed=3))):
        s, c, ex = fn(**kw)
        c.kernel = "mega"
        rs.append(sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]))
    best, table = autotune.tune_batch(rs, block_sizes=(64, 128), blocks_per_sm=(5, 8), occupancies=(0, 8), steps=1)
    assert best in [t[0] for t in table] and all(ms > 0 for _, ms in table)
    with sbatch.Batch(rs, block_size=best[0], blocks_per_sm=best[1], occupancy=best[2]) as b:
        b.reset()
        b.step()
        assert b.check() == 0
    for r in rs:
        r.close()
