"""FP64 oracle reference images of the synthetic workloads (test and bench fixtures).

    python tests/golden/make_oracle_images.py [box|terrain|volume ...] [--spp 64000] [--threads N]

For each workload, renders a stratified subset of pixels (a regular grid of
``side x side`` pixel centres) with the FP64 CPU oracle at ``spp`` samples
(whole 25-band blocks, Philox seed = workload seed + 1000, so its streams are
independent of any GPU render that uses the workload seed) and stores:

  pixels  [P]      pixel ids j * W + i
  mean    [P][B]   running mean over blocks of the per-band block sums (the film)
  sem     [P][B]   standard error of that mean (block-to-block spread / sqrt(n))
  xyz     [P][3]   XYZ of the mean through the workload's CMF and scale
  spp, blocks, seed, workload name

The BVH is the library's binned-SAH tree (built on the host, no GPU needed);
the closest hits, and therefore the images, do not depend on the tree.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402
import spectral_b200 as sb  # noqa: E402
from spectral_b200 import configs  # noqa: E402

# workload -> (generator, grid side of the pixel subset)
WORKLOADS = {"box": (configs.box_scene, 64), "terrain": (configs.terrain_scene, 64),
             "volume": (configs.volume_scene, 32)}


def grid_pixels(w, h, side):
    i = ((np.arange(side) + 0.5) * w / side).astype(np.int64)
    j = ((np.arange(side) + 0.5) * h / side).astype(np.int64)
    jj, ii = np.meshgrid(j, i, indexing="ij")
    return (jj * w + ii).reshape(-1).astype(np.int32)


def render(name, spp, threads, side=None):
    fn, default_side = WORKLOADS[name]
    side = side or default_side
    scene, cfg, ex = fn()
    comp = sb.compile_scene(scene, cfg.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"])
    seed = cfg.seed + 1000
    cfg.seed = seed
    osc = orc.oracle_scene(comp, bvh, scene["camera"])
    ocfg = orc.oracle_config(cfg)
    pix = grid_pixels(cfg.width, cfg.height, side)
    B = cfg.bands
    blocks = -(-spp // B)
    mean = np.zeros((pix.shape[0], B))
    m2 = np.zeros((pix.shape[0], B))
    blk = np.zeros((pix.shape[0], B))
    t0 = time.time()
    for b in range(blocks):
        blk[:] = 0.0
        for k in range(B):
            orc.render_pass(osc, ocfg, b * B + k, k, pix, out=blk, use_double=True, nthreads=threads)
        mean += (blk - mean) / (b + 1)
        m2 += blk * blk
        if (b + 1) % 256 == 0:
            print(f"{name}: {b + 1}/{blocks} blocks, {time.time() - t0:.0f} s", flush=True)
    n = blocks
    var = np.maximum(m2 / n - mean * mean, 0.0) * (n / max(n - 1, 1))
    sem = np.sqrt(var / n)
    cmf = np.asarray(ex["cmf"], np.float32).astype(np.float64)
    scale = 1.0 / float(np.sum(cmf[:, 1]))
    xyz = mean @ cmf * scale
    out = os.path.join(HERE, f"oracle_{name}.npz")
    np.savez_compressed(out, pixels=pix, mean=mean.astype(np.float32), sem=sem.astype(np.float32),
                        xyz=xyz.astype(np.float32), spp=np.int64(blocks * B), blocks=np.int64(blocks),
                        seed=np.int64(seed), workload=np.array(name))
    print(f"{name}: wrote {out} ({pix.shape[0]} pixels, {blocks * B} spp, {time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=["box", "terrain", "volume"])
    ap.add_argument("--spp", type=int, default=64000)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--side", type=int, default=0)
    a = ap.parse_args()
    for nm in a.names:
        render(nm, a.spp, a.threads, a.side or None)
