"""Host logic of batch.render_to_rmse (no GPU): the checking schedule, the
per-scene stop, the block limit and the time limit, on a stand-in batch whose
scenes' estimates fall as 1/sqrt(blocks)."""
import numpy as np
import pytest

from spectral_b200 import batch as sbatch


class StandInBatch:
    """Scenes whose relative RMSE estimate after n blocks is c / sqrt(n)."""

    def __init__(self, consts):
        self.renderers = list(consts)
        self.active = np.ones(len(consts), bool)
        self.blocks = np.zeros(len(consts), np.int64)
        self.steps = 0

    def step(self):
        self.blocks[self.active] += 1
        self.steps += 1

    def wait(self, i):
        pass

    def set_active(self, flags):
        self.active = np.asarray(flags, bool).copy()


def estimator(c, n):
    return c / np.sqrt(n)


@pytest.fixture(autouse=True)
def no_device_sync(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)


def test_each_scene_stops_once_its_estimate_reaches_the_target():
    consts = [0.1, 0.3, 1.0]  # reach 1 % at 100, 900 and 10,000 blocks
    b = StandInBatch(consts)
    blocks, secs = sbatch.render_to_rmse(b, target=0.01, estimator=estimator)
    need = [100, 900, 10000]
    for n, want, c in zip(blocks, need, consts):
        assert estimator(c, n) <= 0.01 + 1e-12
        # checks come where 1/sqrt(n) predicts the target, 90 % of the way: little overshoot
        assert want <= n <= 1.12 * want + 2, (n, want)
    assert b.steps == max(blocks) and not b.active.any() and secs >= 0


def test_next_check_at_most_doubles_and_always_advances():
    for n in (1, 2, 7, 100, 5000):
        for e in (0.011, 0.02, 0.5, 10.0):
            m = sbatch.next_check(n, e, 0.01)
            assert n < m <= 2 * n or (n == 1 and m == 2)


def test_block_limit_and_time_limit_stop_the_run():
    b = StandInBatch([1.0, 1.0])
    blocks, _ = sbatch.render_to_rmse(b, target=0.01, max_blocks=50, estimator=estimator)
    assert list(blocks) == [50, 50] and not b.active.any()
    b = StandInBatch([1.0])
    blocks, _ = sbatch.render_to_rmse(b, target=0.01, estimator=estimator, max_seconds=0.0)
    # the time limit is checked before each step: a limit already passed renders at most one
    assert b.steps <= 1 and b.active.all()
