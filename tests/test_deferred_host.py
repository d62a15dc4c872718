"""Host logic of deferred passes (RenderConfig.defer_passes), with the C library
replaced by a recorder: which launches a pass-by-pass call sequence turns into,
and that every film, camera, settings or block call flushes the queue first."""
import ctypes

import pytest

from helpers import sb  # noqa: F401  (registers the package)
from spectral_b200 import renderer as rmod


class Recorder:
    """Stands in for the loaded library: records ts_* calls, returns TS_OK."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if not name.startswith("ts_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append((name, args))
            return 0
        return call

    def launches(self):
        out = []
        for name, a in self.calls:
            if name == "ts_render_pass":
                out.append(("pass", a[1], a[2]))
            elif name == "ts_render_passes":
                out.append(("bundle", a[1], a[2], a[3]))
            else:
                out.append((name,))
        return out


@pytest.fixture
def make(monkeypatch):
    monkeypatch.setattr(rmod, "_stream", lambda: None)

    def build(defer=True, bands=5):
        r = object.__new__(rmod.Renderer)
        r.config = rmod.RenderConfig(width=4, height=4, bands=bands, defer_passes=defer)
        r.lib = Recorder()
        r._ctx = ctypes.c_void_p(1)
        r._pending = []
        r.total_samples = 0
        r.num_blocks_completed = 0
        r._cam = None
        return r
    return build


def test_reference_cadence_becomes_one_bundle_per_block(make):
    r = make()
    for k in range(12):
        r.cast_rays(k % 5)
        if (k + 1) % 5 == 0:
            r.average_and_reset_block((k + 1) // 5)
    r.check_device()
    assert r.lib.launches() == [("bundle", 0, 5, 0), ("ts_accumulate_block",),
                                ("bundle", 5, 5, 0), ("ts_accumulate_block",),
                                ("bundle", 10, 2, 0), ("ts_check_device",)]
    assert r.total_samples == 12


def test_calls_that_need_the_film_or_scene_flush_first(make):
    r = make()
    r.cast_rays(0)
    r.cast_rays(1)
    r.update_camera([0, 0, 3], [0, 0, 0], [0, 1, 0])
    r.cast_rays(2)
    r.set_launch_config(trace_budget=8)
    r.cast_rays(3)
    r.cast_rays(4)
    r.cast_rays_bundle(0, 5)
    r.cast_rays(0)
    r.clear_pixel_space()
    assert r.lib.launches() == [("bundle", 0, 2, 0), ("ts_set_camera",), ("pass", 2, 2),
                                ("ts_set_launch_config",), ("bundle", 3, 2, 3), ("bundle", 5, 5, 0),
                                ("pass", 10, 0), ("ts_reset",)]


def test_a_break_in_the_run_starts_a_new_launch(make):
    r = make()
    r.cast_rays(0, pass_idx=7)
    r.cast_rays(1, pass_idx=8)
    r.cast_rays(3, pass_idx=9)           # band skips: new run
    r.cast_rays(4, pass_idx=20)          # pass skips: new run
    r.cast_rays(0, pass_idx=0xFFFFFFFF)  # band wraps, pass does not follow 20: new run
    r.cast_rays(1, pass_idx=0)           # pass index wraps mod 2^32: same run
    r.cast_rays(9)                       # band out of range: launched (and rejected) at once, pass 6
    assert r.lib.launches() == [("bundle", 7, 2, 0), ("pass", 9, 3), ("pass", 20, 4),
                                ("bundle", 0xFFFFFFFF, 2, 0), ("pass", 6, 9)]


def test_runs_stop_at_b_passes_and_close_drops_the_queue(make):
    r = make(bands=3)
    for k in range(7):
        r.cast_rays(k % 3)
    assert r.lib.launches() == [("bundle", 0, 3, 0), ("bundle", 3, 3, 0)]
    r.close()
    assert r._pending == [] and r.lib.launches()[-1] == ("ts_destroy",)


def test_without_deferral_every_pass_launches(make):
    r = make(defer=False)
    for k in range(3):
        r.cast_rays(k)
    assert r.lib.launches() == [("pass", 0, 0), ("pass", 1, 1), ("pass", 2, 2)]


def test_huge_frames_flush_in_chunks_under_the_launch_limit(make):
    """A block whose paths exceed what one launch may hold (2^31 - 1) is
    launched in chunks of whole passes -- the same passes, no failure."""
    r = make(bands=25)
    r.config = rmod.RenderConfig(width=9500, height=9500, bands=25, defer_passes=True)
    for k in range(25):
        r.cast_rays(k)
    got = [c for c in r.lib.launches() if c[0] in ("pass", "bundle")]
    per = (2 ** 31 - 1) // (9500 * 9500)
    assert per == 23
    assert got == [("bundle", 0, 23, 0), ("bundle", 23, 2, 23)]
