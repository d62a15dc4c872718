"""Batched rendering of many scenes.

    batch = Batch([Renderer(scene_i, cfg_i, ...) for i in ...], use_graph=True)
    batch.reset(first_pass=0)
    batch.step()             # one spectral block of every active scene, block-averaged
    batch.set_active(flags)  # drop converged scenes from later steps

Two engines with this interface:

  * ``Batch``: all scenes in one persistent megakernel launch per step (a
    device slot table of scenes; the step's four kernels replayed as one CUDA
    graph);
  * ``StreamBatch``: each scene's block as one regenerating-wavefront-loop
    launch (all of the block's passes in flight), the scenes' launches spread
    over a pool of CUDA streams so that small scenes overlap.

Each renderer keeps its own scene, camera, resolution, depth and film; both
engines render exactly the paths ``cast_rays`` would render on each of them
(pass first_pass + B*k + b at band b in step k), so their films equal the
single-scene renders up to the order of FP64 additions (bit for bit where no
fluorescence moves deposits between bands).  ``render_to_rmse`` runs steps
until every scene's estimated relative XYZ RMSE reaches a target.
"""
import ctypes
import time

import numpy as np

from . import _lib
from .renderer import _stream


class TsBatchConfig(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("occupancy", ctypes.c_int32), ("kernel", ctypes.c_int32), ("queue_capacity", ctypes.c_int32),
                ("trace_budget", ctypes.c_int32)]


def _check(lib, status, handle):
    if status != _lib.TS_OK:
        msg = lib.ts_batch_last_error(handle)
        raise _lib.SpectralError(status, msg.decode() if msg else "")


class Batch:
    """Scenes (Renderer objects on one device, one BVH width) rendered together."""

    def __init__(self, renderers, block_size=0, blocks_per_sm=0, use_graph=True, occupancy=0, kernel="mega",
                 queue_capacity=0, trace_budget=0):
        """kernel="mega": one persistent megakernel per step; kernel="wavefront": one
        regenerating wavefront loop over all scenes' paths per step (queue_capacity
        path slots shared by the scenes, 0 = min(paths per step, 2^24)); with
        use_graph a step is one CUDA graph either way."""
        self.renderers = list(renderers)
        for r in self.renderers:
            r.flush()
        self.lib = _lib.load()
        n = len(self.renderers)
        arr = (ctypes.c_void_p * n)(*[r._ctx.value for r in self.renderers])
        k = {"mega": _lib.KERNEL_MEGA, "wavefront": _lib.KERNEL_WAVEFRONT}[kernel]
        cfg = TsBatchConfig(int(block_size), int(blocks_per_sm), 1 if use_graph else 0, int(occupancy), k,
                            int(queue_capacity), int(trace_budget))
        self._h = ctypes.c_void_p()
        _check(self.lib, self.lib.ts_batch_create(ctypes.byref(cfg), arr, n, ctypes.byref(self._h)), None)
        self.active = np.ones(n, bool)
        self.blocks = np.zeros(n, np.int64)
        self.first_pass = 0

    def close(self):
        if self._h:
            self.lib.ts_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self, first_pass=0):
        """Clear every film; the next step renders passes first_pass .. first_pass + B - 1."""
        for r in self.renderers:
            r.flush()
        _check(self.lib, self.lib.ts_batch_reset(self._h, int(first_pass) & 0xFFFFFFFF, _stream()), self._h)
        self.blocks[:] = 0
        self.first_pass = int(first_pass)
        for r in self.renderers:
            r.total_samples = 0
            r.num_blocks_completed = 0

    def set_active(self, flags):
        flags = np.asarray(flags, bool)
        arr = (ctypes.c_int32 * len(flags))(*[int(x) for x in flags])
        _check(self.lib, self.lib.ts_batch_set_active(self._h, arr, _stream()), self._h)
        self.active = flags.copy()

    def step(self):
        """One spectral block of every active scene, followed by its block average."""
        for r in self.renderers:
            r.flush()
        _check(self.lib, self.lib.ts_batch_step(self._h, _stream()), self._h)
        self.blocks[self.active] += 1
        for r, a, nb in zip(self.renderers, self.active, self.blocks):
            if a:
                r.total_samples = int(nb) * r.config.bands
                r.num_blocks_completed = int(nb)

    def check(self):
        bits = ctypes.c_uint32()
        _check(self.lib, self.lib.ts_batch_check(self._h, ctypes.byref(bits)), self._h)
        return bits.value

    def wait(self, i):
        """Make the current stream wait for scene i's last step (one stream here: nothing to do)."""

    def render_to_rmse(self, target=0.01, max_blocks=100000, min_blocks=2, estimator=None, max_seconds=None):
        """Steps until every scene's relative XYZ RMSE estimate is <= target.

        A scene's estimate is evaluated only when it is due: after an estimate e
        at n blocks the next check comes at the block count where 1/sqrt(n)
        scaling predicts the target (``next_check``).  Returns per-scene blocks
        rendered and the wall time (device-synchronised)."""
        return render_to_rmse(self, target, max_blocks, min_blocks, estimator, max_seconds)


class StreamBatch:
    """Scenes rendered block by block, each block one regenerating wavefront
    loop launch of the scene's own context (ts_render_passes with every pass of
    the block in flight: queue_capacity = B * pixels, at most 2^25), the scenes
    spread round-robin over ``streams`` CUDA streams.  Sets each renderer's
    launch configuration to that loop."""

    MAX_QUEUE_CAPACITY = 1 << 25

    def __init__(self, renderers, streams=8, trace_budget=16):
        import torch
        self.renderers = list(renderers)
        self.streams = [torch.cuda.Stream() for _ in range(max(1, int(streams)))]
        n = len(self.renderers)
        for r in self.renderers:
            cap = min(r.config.bands * r.config.width * r.config.height, self.MAX_QUEUE_CAPACITY)
            r.set_launch_config(kernel="wavefront", sort_keys=0, trace_budget=trace_budget, queue_capacity=cap)
        self.events = [None] * n
        self.active = np.ones(n, bool)
        self.blocks = np.zeros(n, np.int64)
        self.first_pass = 0

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self, first_pass=0):
        """Clear every film; the next step renders passes first_pass .. first_pass + B - 1."""
        for r in self.renderers:
            r.clear_pixel_space()
            r.total_samples = 0
            r.num_blocks_completed = 0
        self.blocks[:] = 0
        self.active[:] = True
        self.events = [None] * len(self.renderers)
        self.first_pass = int(first_pass)

    def set_active(self, flags):
        self.active = np.asarray(flags, bool).copy()

    def step(self):
        """One spectral block of every active scene, followed by its block average,
        each scene on its stream (after the work queued so far on the current stream)."""
        import torch
        cur = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(cur)
        for i, r in enumerate(self.renderers):
            if not self.active[i]:
                continue
            st = self.streams[i % len(self.streams)]
            B = r.config.bands
            nb = int(self.blocks[i])
            with torch.cuda.stream(st):
                r.cast_rays_bundle(0, B, pass_idx=self.first_pass + nb * B)
                r.average_and_reset_block(nb + 1)
                ev = torch.cuda.Event()
                ev.record(st)
            self.events[i] = ev
            self.blocks[i] = nb + 1
            r.total_samples = (nb + 1) * B

    def wait(self, i):
        """Make the current stream wait for scene i's last step."""
        import torch
        if self.events[i] is not None:
            torch.cuda.current_stream().wait_event(self.events[i])

    def synchronize(self):
        for s in self.streams:
            s.synchronize()

    def check(self):
        """Device error bits of every scene's context (OR)."""
        self.synchronize()
        bits = 0
        for r in self.renderers:
            bits |= r.check_device()
        return bits

    def render_to_rmse(self, target=0.01, max_blocks=100000, min_blocks=2, estimator=None, max_seconds=None):
        """As ``Batch.render_to_rmse``."""
        return render_to_rmse(self, target, max_blocks, min_blocks, estimator, max_seconds)


def render_to_rmse(batch, target=0.01, max_blocks=100000, min_blocks=2, estimator=None, max_seconds=None):
    """Steps ``batch`` until every scene's relative XYZ RMSE estimate is <= target
    (checks when due, ``next_check``), or until ``max_seconds`` have passed (the
    step under way completes); returns per-scene blocks and the wall time."""
    import torch
    estimator = estimator or relative_rmse_estimate
    due = np.full(len(batch.renderers), min_blocks, np.int64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while batch.active.any():
        if max_seconds is not None and time.perf_counter() - t0 > max_seconds:
            break
        batch.step()
        flags = batch.active.copy()
        for i, r in enumerate(batch.renderers):
            n = int(batch.blocks[i])
            if not flags[i] or (n < due[i] and n < max_blocks):
                continue
            batch.wait(i)
            e = estimator(r, n)
            if e <= target or n >= max_blocks:
                flags[i] = False
            else:
                due[i] = next_check(n, e, target)
        if (flags != batch.active).any():
            batch.set_active(flags)
    torch.cuda.synchronize()
    return batch.blocks.copy(), time.perf_counter() - t0


def next_check(n, estimate, target):
    """Block count at which to look again: where the estimate, falling as 1/sqrt(n),
    is predicted to reach the target (90 % of the way, at most doubling n)."""
    return n + max(1, min(n, int(n * ((estimate / target) ** 2 - 1) * 0.9)))


def xyz_mean_and_variance(renderer, nblocks):
    """Per-pixel XYZ of the block mean and its variance (bands taken as independent), float64 tensors."""
    import torch
    n = nblocks
    mean, m2 = renderer.mean_film, renderer.m2_film
    cmf = torch.as_tensor(renderer.compiled.cmf, dtype=torch.float64, device=mean.device) * renderer.cmf_scale
    var = (m2 / n - mean * mean).clamp_min(0.0) * (n / max(n - 1, 1)) / n
    xyz = torch.einsum("bhw,bc->hwc", mean, cmf)
    xvar = torch.einsum("bhw,bc->hwc", var, cmf * cmf)
    return xyz, xvar


def relative_rmse_estimate(renderer, nblocks):
    """sqrt(sum Var(XYZ)) / ||XYZ|| of the block mean: its expected relative RMSE against the converged image."""
    import torch
    xyz, xvar = xyz_mean_and_variance(renderer, nblocks)
    den = float(torch.sum(xyz * xyz))
    return float(torch.sqrt(torch.sum(xvar))) / max(float(np.sqrt(den)), 1e-300)
