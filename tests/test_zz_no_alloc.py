"""The allocation-free tile render, called through the C ABI, against ts_render_pass.

ts_render_tile_noalloc serves callers that cannot call cudaMalloc while they
render (a fixed device-memory budget after start-up, or a render loop inside a
framework that owns the allocator).  It must produce exactly what the regular
wavefront pass produces for the same pass, band and pixels, call after call.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import sb
from spectral_b200 import configs

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_noalloc_tiles_match_render_pass_on_consecutive_calls():
    s, c, ex = configs.box_scene(width=96, height=80)
    c.kernel = "wavefront"
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        lib = r.lib
        film = torch.zeros((c.bands, c.height, c.width), dtype=torch.float64, device="cuda")
        for call, (pass_idx, band) in enumerate([(3, 7), (4, 19)]):
            r.clear_pixel_space()
            r.cast_rays(band, pass_idx=pass_idx)          # the existing entry point, whole frame
            want = r.block_film.cpu().numpy().copy()
            film.zero_()
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            for y0 in (0, 40):                             # two 96 x 40 tiles cover the frame
                st = lib.ts_render_tile_noalloc(r._ctx, pass_idx, band, 0, y0, 96, 40,
                                                ctypes.c_void_p(film.data_ptr()), _stream())
                assert st == 0, lib.ts_last_error(r._ctx)
            torch.cuda.synchronize()
            got = film.cpu().numpy()
            assert np.count_nonzero(want) > 0
            assert np.allclose(got, want, rtol=1e-12, atol=0.0)
            if call == 1:
                # after the first call has looked the scratch address up, a call
                # leaves the device's free memory untouched
                assert torch.cuda.mem_get_info()[0] == free_before
        assert r.check_device() == 0


def test_noalloc_rejects_oversized_and_out_of_frame_tiles():
    s, c, ex = configs.box_scene(width=300, height=300)
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        lib = r.lib
        film = torch.zeros((c.bands, c.height, c.width), dtype=torch.float64, device="cuda")
        p = ctypes.c_void_p(film.data_ptr())
        assert lib.ts_render_tile_noalloc(r._ctx, 0, 0, 0, 0, 300, 300, p, _stream()) == 4  # TS_ERR_CAPACITY
        assert b"65536" in lib.ts_last_error(r._ctx)
        assert lib.ts_render_tile_noalloc(r._ctx, 0, 0, 250, 0, 64, 64, p, _stream()) == 1  # outside the frame
        # exactly the limit: the whole scratch layout in use, against the regular pass on that region
        assert lib.ts_render_tile_noalloc(r._ctx, 5, 11, 20, 30, 256, 256, p, _stream()) == 0
        torch.cuda.synchronize()
        got = film.cpu().numpy()
        r.clear_pixel_space()
        r.cast_rays(11, pass_idx=5)
        want = r.block_film.cpu().numpy()
        tile = (slice(None), slice(30, 286), slice(20, 276))
        assert np.count_nonzero(want[tile]) > 0
        assert np.allclose(got[tile], want[tile], rtol=1e-12, atol=0.0)
        outside = np.ones(got.shape, bool)
        outside[tile] = False
        assert not got[outside].any()  # nothing written outside the tile
        assert r.check_device() == 0
