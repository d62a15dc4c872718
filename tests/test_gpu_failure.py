"""Failure handling on the device, without a GPU fault.

The regenerating wavefront loop is the one device-side loop of the path: a
CUDA-graph while-loop whose condition a control kernel sets.  Its iterations
are bounded; a launch that reaches the bound stops on the device, sets the
iteration-cap bit and returns, so the host learns of it from
``ts_check_device`` and the context stays usable.  Here the bound is set
below what the work needs (``ts_set_loop_iteration_limit``) so that it fires.
"""
import numpy as np
import pytest

from helpers import sb
from spectral_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("loop_host", [0, 1])
def test_iteration_cap_stops_the_loop_and_the_context_recovers(loop_host):
    s, c, ex = configs.box_scene(width=48, height=48, depth=8)
    c.kernel = "wavefront"
    c.queue_capacity = 48 * 48  # one slot per pixel: a 25-pass bundle needs many iterations
    c.loop_host = loop_host
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        r.cast_rays_bundle(0, c.bands, pass_idx=0)
        want = r.block_film.cpu().numpy().copy()
        assert r.check_device() == 0
        full = r.wave_loop_iterations()
        assert full > 8

        r.clear_pixel_space()
        r.set_loop_iteration_limit(2)
        r.cast_rays_bundle(0, c.bands, pass_idx=0)  # returns: the stop happens on the device
        assert r.wave_loop_iterations() == 2
        with pytest.raises(sb.SpectralError, match="iteration cap reached") as err:
            r.check_device()
        assert err.value.status == 5  # TS_ERR_DEVICE_FAULT
        partial = r.block_film.cpu().numpy()
        assert partial.sum() < want.sum()  # the dropped paths deposited nothing

        # the next launch on the same context starts clean
        r.set_loop_iteration_limit(0)
        r.clear_pixel_space()
        r.cast_rays_bundle(0, c.bands, pass_idx=0)
        assert r.check_device() == 0
        assert r.wave_loop_iterations() == full
        assert np.array_equal(r.block_film.cpu().numpy(), want)


def test_iteration_limit_rejects_negative_values():
    s, c, ex = configs.box_scene(width=8, height=8)
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        with pytest.raises(sb.SpectralError, match="limit must be >= 0"):
            r.set_loop_iteration_limit(-1)
