"""Autotuner: picks the launch configuration of a scene by timing candidates.

Every candidate renders exactly the same paths (the random streams depend
only on seed, pass, pixel and draw index), so tuning never changes an image,
only its cost.  Knobs:

  * BVH node width 2 / 4 / 8, and for 4 / 8 full-precision or quantized
    child boxes (the scene is re-uploaded per layout; the host builder's tree
    is reused),
  * traversal loop of two-child nodes (default if-if / speculative while-while),
  * kernel: the persistent megakernel or the wavefront stages, and for the
    wavefront its queue sorting (sort_keys bit mask), the traversal steps
    between lane refills (trace_budget) and, for wavelength bundles, the
    queue capacity of the regenerating loop (path slots: how many passes'
    paths are in flight at once),
  * threads per block and resident blocks per SM of the persistent grid, and
    the megakernel's register budget (5 blocks/SM without spills, or 8 with).

Each candidate renders ``passes`` passes after ``warmup`` (CUDA events on the
current stream); the fastest wins.  Results are cached in a JSON file keyed by
a signature of the scene (triangles, materials, resolution, depth, bands).

    best, table = tune(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], cache="tune.json")
    r = Renderer(scene, best.apply(cfg), eems=..., cmf=..., bvh_params=best.bvh_params())
"""
import dataclasses
import hashlib
import json
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .renderer import Renderer
from .scene import compile_scene


@dataclass(frozen=True)
class Candidate:
    width: int = 2
    traversal: str = "default"
    kernel: str = "mega"
    block_size: int = 128
    blocks_per_sm: int = 0
    sort_keys: int = 0
    trace_budget: int = 0
    occupancy: int = 0
    queue_capacity: int = 0
    quantize: bool = False  # 4- / 8-wide nodes with 8-bit child boxes (64 / 96 B)

    def bvh_params(self):
        return {"width": self.width, "quantize": self.quantize}

    def apply(self, cfg):
        """A copy of cfg with this candidate's launch settings."""
        return dataclasses.replace(cfg, traversal=self.traversal, kernel=self.kernel, block_size=self.block_size,
                                   blocks_per_sm=self.blocks_per_sm, sort_keys=self.sort_keys,
                                   trace_budget=self.trace_budget, occupancy=self.occupancy,
                                   queue_capacity=self.queue_capacity)


def default_candidates(quick=False):
    out = [Candidate(w, "default", "mega", bs, bpsm) for w in (2, 4, 8) for bs in (64, 128) for bpsm in (0, 5)]
    out += [Candidate(w, "default", "mega", 128, 0, occupancy=8) for w in (2, 4, 8)]
    out += [Candidate(w, "default", "mega", 128, 0, occupancy=o, quantize=True) for w in (4, 8) for o in (0, 8)]
    out += [Candidate(2, "speculative", "mega", 128, 0), Candidate(2, "speculative", "mega", 128, 0, occupancy=8)]
    if not quick:
        out += [Candidate(w, "default", "wavefront", 128, 0, sk, tb)
                for w in (2, 4) for sk in (0, 1) for tb in (16, 32, 64)]
    return out


MAX_QUEUE_CAPACITY = 1 << 25


def bundle_wavefront_candidates(npix, bands, widths=(2, 4, (4, True), (8, True)), multiples=(2, 4, 8, 16, 32),
                                budgets=(16, 8)):
    """Regenerating-loop wavefront candidates for wavelength bundles: queue
    capacities of several frames' worth of path slots (passes in flight),
    up to the whole bundle, and traversal steps between lane refills (8 is
    faster on shallow BVHs and deep volume paths, 16 on the 2.6M-triangle
    terrain)."""
    caps = sorted({min(m * npix, bands * npix, MAX_QUEUE_CAPACITY) for m in multiples})
    lay = [w if isinstance(w, tuple) else (w, False) for w in widths]
    return [Candidate(w, "default", "wavefront", 256, 0, 0, tb, queue_capacity=qc, quantize=q)
            for w, q in lay for qc in caps for tb in budgets]


def signature(compiled, cfg, bundles=False):
    h = hashlib.sha1()
    for a in (compiled.tris["v0"], compiled.mat_f32, compiled.mat_i32):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(repr((cfg.width, cfg.height, cfg.bands, cfg.max_path_length, cfg.scatter_bounces)).encode())
    h.update(b"bundles" if bundles else b"passes")
    return h.hexdigest()[:16]


def _time_passes(r, passes, warmup, first_pass, bundles=False):
    """ms per pass: one launch per pass, or one launch per block (bundles)."""
    import torch
    B = r.config.bands
    if bundles:
        r.cast_rays_bundle(0, B, pass_idx=first_pass)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        blocks = max(1, passes // B)
        a.record()
        for k in range(blocks):
            r.cast_rays_bundle(0, B, pass_idx=first_pass + (k + 1) * B)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / (blocks * B)
    for p in range(warmup):
        r.cast_rays(p % B, pass_idx=first_pass + p)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for p in range(passes):
        r.cast_rays((warmup + p) % B, pass_idx=first_pass + warmup + p)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / passes


def tune(scene_dict, cfg, eems=None, cmf=None, candidates=None, passes=6, warmup=2, cache=None, quick=False,
         first_pass=1 << 24, bundles=False):
    """Time every candidate on this scene; returns (best Candidate, [(Candidate, ms per pass)]).

    bundles: time whole-block launches (cast_rays_bundle) instead of one launch
    per pass -- the two favour different block shapes.  Bundles are timed for
    the megakernel candidates and for the regenerating wavefront loop over a
    range of queue capacities (sorted-queue wavefront candidates are dropped:
    they launch per pass)."""
    compiled = compile_scene(scene_dict, cfg.bands, eems=eems, cmf=cmf)
    key = signature(compiled, cfg, bundles)
    if cache and os.path.exists(cache):
        stored = json.load(open(cache)).get(key)
        if stored:
            best = Candidate(**stored["best"])
            return best, [(Candidate(**c), ms) for c, ms in stored["table"]]
    bvh = _lib.build_bvh_host(compiled.tris["v0"], compiled.tris["v1"], compiled.tris["v2"])
    candidates = list(candidates or default_candidates(quick))
    if bundles:
        candidates = [c for c in candidates if c.kernel == "mega" or c.sort_keys == 0]
        extra = bundle_wavefront_candidates(cfg.width * cfg.height, cfg.bands)
        candidates += [c for c in extra if c not in candidates]
    table = []
    for layout in sorted({(c.width, c.quantize) for c in candidates}):
        group = [c for c in candidates if (c.width, c.quantize) == layout]
        with Renderer(scene_dict, group[0].apply(cfg), eems=eems, cmf=cmf, bvh=bvh,
                      bvh_params=group[0].bvh_params()) as r:
            for cand in group:
                r.set_launch_config(kernel=cand.kernel, traversal=cand.traversal, block_size=cand.block_size,
                                    blocks_per_sm=cand.blocks_per_sm, sort_keys=cand.sort_keys,
                                    trace_budget=cand.trace_budget, occupancy=cand.occupancy,
                                    queue_capacity=cand.queue_capacity)
                ms = _time_passes(r, passes, warmup, first_pass, bundles)
                if r.check_device() != 0:
                    ms = float("inf")
                table.append((cand, ms))
    best = min(table, key=lambda t: t[1])[0]
    if cache:
        data = json.load(open(cache)) if os.path.exists(cache) else {}
        data[key] = {"best": dataclasses.asdict(best), "table": [(dataclasses.asdict(c), ms) for c, ms in table]}
        with open(cache, "w") as f:
            json.dump(data, f, indent=1)
    return best, table


def tune_batch(renderers, block_sizes=(64, 128), blocks_per_sm=(5, 8), occupancies=(0, 8), steps=2):
    """Threads per block, blocks per SM of the persistent grid and register budget of
    the batched kernel, timed on ``steps`` steps of the given scenes (their BVH
    width is theirs; the films are cleared afterwards).
    Returns ((block_size, blocks_per_sm, occupancy), [(setting, ms per step)])."""
    import torch
    from .batch import Batch
    table = []
    for bs, bpsm, occ in [(a, b, c) for a in block_sizes for b in blocks_per_sm for c in occupancies]:
        with Batch(renderers, block_size=bs, blocks_per_sm=bpsm, use_graph=False, occupancy=occ) as b:
            b.reset(first_pass=1 << 24)
            b.step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                b.step()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            if b.check() != 0:
                ms = float("inf")
            b.reset()
        table.append(((bs, bpsm, occ), ms))
    return min(table, key=lambda t: t[1])[0], table
