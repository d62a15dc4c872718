"""Benchmark: spectral path tracing on the large-mesh workload.

One step = one spectral block: the 25 sample passes of a wavelength cycle
(cast_rays at bands 0..24, each pass its own random stream) over every pixel
of the workload -- 1024x1024 paths per pass of depth <= 12 through a
2.59M-triangle scene (1024^2-vertex heightfield + 500k-triangle displaced
sphere, GGX conductors, 8 emissive quads, 25 bands over 380-740 nm).  The
metric is Mpaths/s (one path = one pixel x one band-pass, the reference's
unit); a step is 26.2M paths.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--kernel mega|wavefront] [--workload terrain|box|volume|batch|adjoint|rmse]

--impl reference times the reference's CPU path: the FP32 restatement of its
estimator (oracle/, pinned to the reference's own code; OpenMP over all host
threads) on the reference's BVH algorithm (the oracle's full-sweep SAH
builder), since the reference's own Taichi kernels cannot be installed here.
That arm loads no part of the CUDA library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes of one unit of work, for the roofline (layouts in csrc/common.cuh)
BYTES_NODE = 64      # one two-child BVH node (two child boxes + links); wide nodes 128 / 256 B
BYTES_NODE_Q = {4: 64, 8: 96}  # quantized wide nodes (origin, scales, links, 8-bit child boxes)
BYTES_TRI = 48       # one triangle test (v0, e1, e2 as float4)
BYTES_HIT = 48       # shading normals of a resolved hit (3 float4)
BYTES_MAT_VERTEX = 8 * 32  # material lookups per path vertex (8 x two float4)
BYTES_DEPOSIT = 16   # FP64 read-modify-write of a film cell


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20, help="timed steps (spectral blocks of 25 passes)")
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--kernel", default="mega", choices=["mega", "wavefront"])
    p.add_argument("--workload", default="terrain", choices=["terrain", "box", "volume", "batch", "adjoint", "rmse", "gradcheck", "inverse"])
    p.add_argument("--width", type=int, default=2, choices=[2, 4, 8], help="BVH node width")
    p.add_argument("--quantize", action="store_true", help="4- / 8-wide nodes with 8-bit child boxes (--no-tune)")
    p.add_argument("--traversal", default="default", choices=["default", "speculative"])
    p.add_argument("--leaf-max", type=int, default=0, help="largest BVH leaf the SAH may choose, 1..16 (--no-tune; 0 = 8)")
    p.add_argument("--cost-trav", type=float, default=0.0, help="SAH node-visit cost per triangle test (--no-tune; 0 = 1)")
    p.add_argument("--occupancy", type=int, default=0, choices=[0, 8], help="megakernel register budget (--no-tune)")
    p.add_argument("--launch", default="bundle", choices=["bundle", "pass"],
                   help="render each step's 25 passes in one launch (a wavelength bundle) or one launch per pass")
    p.add_argument("--budget", type=int, default=0, help="wavefront traversal steps between refills")
    p.add_argument("--queue-capacity", type=int, default=0,
                   help="wavefront path slots of the regenerating loop (--no-tune; 0 = one per pixel)")
    p.add_argument("--loop-host", action="store_true",
                   help="launch the wavefront loop's iterations from the host (for kernel profilers)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the time-to-RMSE and adjoint-cost legs")
    p.add_argument("--no-tune", action="store_true", help="use --kernel/--width/--traversal as given instead of "
                                                          "the autotuner's choice")
    p.add_argument("--rmse-seconds", type=float, default=60.0, help="time limit of each time-to-RMSE leg")
    p.add_argument("--rmse-target", type=float, default=0.01, help="relative XYZ RMSE target (--workload rmse)")
    p.add_argument("--rmse-workloads", default="box,terrain,volume", help="workloads of --workload rmse")
    p.add_argument("--batch-scenes", type=int, default=64, help="scenes of the batched workload (--workload batch)")
    p.add_argument("--batch-target", type=float, default=0.05, help="RMSE target of the batched workload")
    p.add_argument("--batch-engines", default="kernel,loop,streams",
                   help="batched engines to run to the target (--workload batch): kernel, loop, streams")
    p.add_argument("--batch-views", type=int, default=8,
                   help="scenes of the batched workload that get a second camera (a view on the same upload)")
    p.add_argument("--batch-seconds", type=float, default=0.0,
                   help="time limit of each batched engine's run to the target (0: none)")
    p.add_argument("--batch-plain-blocks", type=int, default=0,
                   help="time the plain arm on this many blocks per scene and scale it by the blocks the batched "
                        "engines needed (0: run the plain arm to the target too)")
    p.add_argument("--passes", type=int, default=25, help="passes per adjoint launch (--workload adjoint)")
    p.add_argument("--gradcheck-blocks", type=int, default=40, help="blocks per evaluation (--workload gradcheck)")
    p.add_argument("--gradcheck-res", type=int, default=128, help="resolution (--workload gradcheck)")
    p.add_argument("--iterations", type=int, default=200, help="Adam iterations (--workload inverse)")
    return p.parse_args()


def workload(name):
    from spectral_b200 import configs
    if name == "terrain":
        scene, cfg, ex = configs.terrain_scene()
        desc = ("terrain: 1024^2-vertex heightfield (2.09M tris, 6-octave value noise) + 500k-tri displaced "
                "sphere, GGX conductors, 8 emissive quads; 1024x1024, depth 12, 25 bands 380-740 nm, 256 spp")
    elif name == "box":
        scene, cfg, ex = configs.box_scene()
        desc = "box: 12-tri box + 2048-tri GGX dielectric sphere + quad light; 256x256, depth 8, 25 bands, 64 spp"
    elif name == "inverse-target":
        scene, cfg, ex = configs.volume_scene(width=256, height=256, depth=32)
        desc = ("inverse-rendering target: the volume scene at 256x256, depth 32, 25 bands, with the hidden "
                "79 parameters of seed 7 (wall albedos, sigma_a, g, roughnesses)")
    else:
        scene, cfg, ex = configs.volume_scene()
        desc = ("volume: box + 20k-tri HG medium (g 0.7) + fluorescent wall; 512x512, depth 32, 25 bands, "
                "512 spp")
    return scene, cfg, ex, desc


def apply_workload(r, name):
    """Workload state beyond the scene dictionary: the inverse-rendering target
    renders the hidden parameters of seed 7 (material table upload)."""
    if name != "inverse-target":
        return
    from spectral_b200 import autodiff, inverse
    hidden = inverse.Params.from_scene_params(inverse.scene_params(7), "cuda")
    mat = inverse.material_table(autodiff.material_table(r), hidden, r.config.wavelengths()).float().contiguous()
    r.update_materials(mat, None)


def step_config(cfg, ex, desc, world, num_tris):
    """The workload as both arms report it (identical dictionaries)."""
    npix = cfg.width * cfg.height
    # resident inputs: 96 B per triangle (positions + shading normals) and the
    # three FP64 film planes (block, mean, second moment)
    mb = (96 * num_tris + 3 * 8 * cfg.bands * npix) / 1e6
    l2 = ("inputs larger than L2: %.0f MB of triangles and film > 126 MB L2; no flush" % mb if mb > 126 else
          "inputs fit in L2 (%.0f MB of triangles and film): steady-state rate of a resident scene, no flush" % mb)
    return {"workload": desc, "paths_per_step": cfg.bands * npix, "passes_per_step": cfg.bands,
            "pixels": npix, "spp": ex["spp"], "passes_for_spp": cfg.samples_per_pixel, "l2": l2,
            "parallelism": f"{world} GPU(s), disjoint sample passes per GPU"}


def reference_tree(comp):
    """The reference's BVH algorithm (main.py:437-507: full-sweep SAH, <= 10
    triangles per leaf) restated in the oracle, in the reference layout."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    t = comp.tris
    b = orc.build_bvh_sweep(t["v0"], t["v1"], t["v2"])
    b["tri_perm"] = b.pop("perm")
    return b


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id=None):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.gpu_id is not None:
            cmd += ["-i", str(self.gpu_id)]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9], parts[4]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def gpu_uuid(dev):
    import torch
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        return f"GPU-{u}"
    except Exception:
        return None


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def profiled_traffic(kernel, workload_name, width, occupancy, bundles=False):
    """DRAM bytes per launch from the committed ncu summary (None if not captured)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    e = d.get(f"{workload_name}:{kernel}:w{width}" + (f":o{occupancy}" if occupancy else "") +
              (":bundle" if bundles else ""))
    return None if e is None else float(e["dram_bytes_per_launch"])


def cpu_oracle_rate(comp, bvh, scene, cfg, seconds, nthreads=0, passes=None):
    """Paths/s of the FP32 oracle on a pixel sample sized for ~``seconds``."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    osc = orc.oracle_scene(comp, bvh, scene["camera"])
    ocfg = orc.oracle_config(cfg)
    npix = cfg.width * cfg.height
    rng = np.random.default_rng(123)
    n = 1024
    pix = rng.choice(npix, min(n, npix), replace=False).astype(np.int32)
    t = time.perf_counter()
    orc.render_pass(osc, ocfg, 0, 12, pix, nthreads=nthreads)
    dt = max(time.perf_counter() - t, 1e-6)
    rate = len(pix) / dt
    # ~seconds of work: a random pixel subset, or whole passes when one pass is quicker
    want = max(1024, rate * seconds)
    n = int(min(npix, want))
    passes = max(1, int(round(want / npix))) if n == npix else 1
    pix = rng.choice(npix, n, replace=False).astype(np.int32)
    t = time.perf_counter()
    for k in range(passes):
        _, st = orc.render_pass(osc, ocfg, 1 + k, (12 + k) % cfg.bands, pix, nthreads=nthreads)
    dt = time.perf_counter() - t
    threads = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    return n * passes / dt, n * passes, dt, threads, st


def oracle_fixture(name):
    path = os.path.join(ROOT, "tests", "golden", f"oracle_{name}.npz")
    if not os.path.exists(path):
        return None
    import numpy as np
    return dict(np.load(path))


def rmse_leg(name, target, seconds, bundles=True):
    """Blocks until the image's estimated relative XYZ RMSE (its own per-pixel
    variance; the GPU estimator is unbiased) reaches ``target``, or ``seconds``
    run out; then the image is compared with the FP64 oracle fixture on the
    oracle's pixel subset (independent random streams): the difference must
    match the combined noise of both images (z near 0 means no bias)."""
    import numpy as np
    import torch
    import spectral_b200 as sb
    from spectral_b200 import batch as sbatch
    from spectral_b200 import autotune
    scene, cfg, ex, desc = workload(name)
    # launch settings from the autotuner: for bundles the megakernel and the
    # regenerating wavefront loop (queue capacities), per pass the megakernel
    cands = [c for c in autotune.default_candidates(quick=True) if c.kernel == "mega"]
    best, _ = autotune.tune(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], candidates=cands, passes=50 if bundles else 6,
                            first_pass=1 << 26, bundles=bundles)
    cfg = best.apply(cfg)
    r = sb.Renderer(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], bvh_params=best.bvh_params())
    apply_workload(r, name)
    B = cfg.bands
    r.cast_rays_bundle(0, B, pass_idx=0)
    r.clear_pixel_space()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nb, est = 0, float("inf")
    next_check = 2
    while True:
        if bundles:
            r.cast_rays_bundle(0, B, pass_idx=nb * B)
        else:
            for k in range(B):
                r.cast_rays(k, pass_idx=nb * B + k)
        nb += 1
        r.average_and_reset_block(nb)
        if nb >= next_check:
            est = sbatch.relative_rmse_estimate(r, nb)
            if est <= target:
                break
            # next check where 1/sqrt(n) scaling predicts the target (at most doubling n)
            next_check = nb + max(1, min(nb, int(nb * ((est / target) ** 2 - 1) * 0.9)))
        if time.perf_counter() - t0 > seconds:
            break
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    est = sbatch.relative_rmse_estimate(r, nb)
    out = {"workload": name, "target": target, "blocks": nb, "spp": nb * B, "seconds": secs,
           "launch": {"kernel": best.kernel, "width": best.width, "quantize": best.quantize, "traversal": best.traversal,
                      "block_size": best.block_size, "blocks_per_sm": best.blocks_per_sm,
                      "occupancy": best.occupancy, "queue_capacity": best.queue_capacity,
                      "trace_budget": best.trace_budget},
           "estimated_rmse": float(est), "reached": bool(est <= target),
           "launches": "one per block (wavelength bundle)" if bundles else "one per pass"}
    if est > target:
        # time to a target scales with its inverse square (variance ~ 1 / samples)
        out["seconds_extrapolated"] = secs * (est / target) ** 2
    fx = oracle_fixture(name)
    if fx is not None:
        xyz, xvar = sbatch.xyz_mean_and_variance(r, nb)
        W = cfg.width
        pix = fx["pixels"].astype(np.int64)
        g = xyz.reshape(-1, 3)[torch.as_tensor(pix, device=xyz.device)].cpu().numpy()
        gv = xvar.reshape(-1, 3)[torch.as_tensor(pix, device=xyz.device)].cpu().numpy()
        o = fx["xyz"].astype(np.float64)
        cmf = np.asarray(r.compiled.cmf, np.float64) * r.cmf_scale
        ov = (fx["sem"].astype(np.float64) ** 2) @ (cmf ** 2)
        norm = np.sqrt((o ** 2).sum())
        diff2 = ((g - o) ** 2).sum()
        expect2 = gv.sum() + ov.sum()
        # per-pixel sums of squared differences: spread of the difference statistic
        d2 = ((g - o) ** 2).sum(1)
        se2 = np.sqrt(max(float(((d2 - d2.mean()) ** 2).sum()), 1e-300))
        out["vs_oracle"] = {"oracle_spp": int(fx["spp"]), "pixels": int(pix.shape[0]),
                            "rmse_vs_oracle": float(np.sqrt(diff2) / norm),
                            "expected_from_noise": float(np.sqrt(expect2) / norm),
                            "oracle_noise_rmse": float(np.sqrt(ov.sum()) / norm),
                            "z": float((diff2 - expect2) / se2)}
    bits = r.check_device()
    r.close()
    out["device_error_bits"] = bits
    return out


def plain_seconds(name, blocks, timed_blocks=6):
    """The plain single-scene kernel -- the depth-synchronous wavefront pass,
    one launch per pass, no bundles -- on the first blocks of a time-to-RMSE
    leg (the same passes, so the same paths and the same image): seconds per
    block from CUDA events over ``timed_blocks`` blocks, and the seconds the
    leg's ``blocks`` take at that rate."""
    import torch
    import spectral_b200 as sb
    scene, cfg, ex, desc = workload(name)
    cfg.kernel = "wavefront"
    cfg.queue_capacity = 0
    cfg.sort_keys = 0
    cfg.trace_budget = 16
    r = sb.Renderer(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], bvh_params={"width": 4})
    apply_workload(r, name)
    B = cfg.bands
    for k in range(B):
        r.cast_rays(k, pass_idx=(1 << 26) + k)  # warm-up
    n = max(1, min(blocks, timed_blocks))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for b in range(n):
        for k in range(B):
            r.cast_rays(k, pass_idx=b * B + k)
        r.average_and_reset_block(b + 1)
    e1.record()
    torch.cuda.synchronize()
    per_block = e0.elapsed_time(e1) / n * 1e-3
    bits = r.check_device()
    r.close()
    return {"kernel": "depth-synchronous wavefront pass, one launch per pass (four-child nodes)",
            "seconds_per_block": per_block, "timed_blocks": n, "seconds_same_paths": per_block * blocks,
            "device_error_bits": bits}


def bench_gradcheck(args):
    """The adjoint of the inverse-rendering workload's 79 parameters against
    central finite differences (h = 1e-3, common random numbers): the volume
    scene (HG medium, fluorescent wall, depth 32), parameters of seed 8 (the
    fit's starting point).  Prints one JSON line with every parameter."""
    import numpy as np
    import torch
    import spectral_b200 as sb
    from spectral_b200 import configs, inverse
    res = args.gradcheck_res
    s, c, ex = configs.volume_scene(width=res, height=res, depth=32)
    c.kernel = "wavefront"
    c.queue_capacity = c.bands * res * res
    t0 = time.perf_counter()
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        p = inverse.Params.from_scene_params(inverse.scene_params(8), "cuda")
        rows = inverse.gradient_check(r, p, h=1e-3, blocks=args.gradcheck_blocks)
        bits = r.check_device()
    secs = time.perf_counter() - t0
    rel = np.array([abs(x["adjoint"] - x["fd"]) / max(abs(x["fd"]), 1e-300) for x in rows])
    # both sides are Monte Carlo estimates on the same paths; their errors are
    # positively correlated, so the combined error below is an upper bound
    sem = np.array([np.hypot(x["fd_sem"], np.nan_to_num(x["adjoint_sem"])) for x in rows])
    z = np.array([(x["adjoint"] - x["fd"]) / max(e, 1e-300) for x, e in zip(rows, sem)])
    noise = np.array([x["fd_sem"] / max(abs(x["fd"]), 1e-300) for x in rows])
    adj_noise = np.array([x["adjoint_sem"] / max(abs(x["adjoint"]), 1e-300) for x in rows])
    groups = {}
    for name in ("albedo_left", "albedo_right", "sigma_a", "g", "roughness"):
        idx = [i for i, x in enumerate(rows) if x["name"] == name]
        groups[name] = {"parameters": len(idx), "within_2pct": int((rel[idx] <= 0.02).sum()),
                        "max_rel_err": float(rel[idx].max()), "median_fd_rel_sem": float(np.median(noise[idx])),
                        "median_adjoint_rel_sem": float(np.median(adj_noise[idx])),
                        "max_abs_z": float(np.abs(z[idx]).max()),
                        "within_2pct_or_3_sem": int(((rel[idx] <= 0.02) | (np.abs(z[idx]) <= 3)).sum())}
    print(json.dumps({"metric": "adjoint vs central finite differences", "parameters": len(rows),
                      "groups": groups,
                      "within_2pct": int((rel <= 0.02).sum()), "max_rel_err": float(rel.max()),
                      "median_rel_err": float(np.median(rel)), "max_abs_z": float(np.abs(z).max()),
                      "max_fd_rel_sem": float(noise.max()), "h": "1e-3 relative to each parameter",
                      "z": "(adjoint - fd) / hypot(fd_sem, adjoint_sem); adjoint_sem from 10 groups of blocks",
                      "blocks": args.gradcheck_blocks,
                      "config": {"workload": f"volume scene (HG medium g 0.7, fluorescent wall) {res}x{res}, depth 32, "
                                             "25 bands; 79 parameters of seed 8"},
                      "seconds": secs, "device_error_bits": bits, "rows": rows}))


def bench_inverse(args):
    """The differentiable inverse-rendering workload as configured: the volume
    scene at 256x256 (depth 32), 79 parameters, target image at 4,100 spp from
    the hidden parameters of seed 7, start from seed 8, 2 blocks (50 passes) per
    forward and adjoint, Adam lr 1e-2 for --iterations steps.  Reports the loss
    history, seconds per iteration, the final image's relative XYZ RMSE
    against the target image, the noise floor (the hidden parameters' own
    loss) and the parameter errors."""
    import torch
    import spectral_b200 as sb
    from spectral_b200 import configs, inverse
    s, c, ex = configs.volume_scene(width=256, height=256, depth=32)
    c.kernel = "wavefront"
    c.queue_capacity = c.bands * 256 * 256
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        hidden = inverse.Params.from_scene_params(inverse.scene_params(7), "cuda")
        init = inverse.Params.from_scene_params(inverse.scene_params(8), "cuda")
        t0 = time.perf_counter()
        target = inverse.render_target(r, hidden, blocks=164)  # 4,100 spp
        torch.cuda.synchronize()
        t_target = time.perf_counter() - t0
        t0 = time.perf_counter()
        fit, hist = inverse.run(r, target, init, iterations=args.iterations, lr=1e-2, blocks=2)
        torch.cuda.synchronize()
        t_fit = time.perf_counter() - t0

        def image_rmse(p, blocks=40):
            """relative XYZ RMSE of p's image (blocks spectral blocks) against the target"""
            x = inverse.render_target(r, p, blocks=blocks)
            return float(torch.linalg.vector_norm(x - target) / torch.linalg.vector_norm(target))

        e_init, e_fit, e_hidden = image_rmse(init), image_rmse(fit), image_rmse(hidden)
        floor = inverse.image_loss(r, hidden, target)
        bits = r.check_device()
    print(json.dumps({"metric": "inverse rendering: relative XYZ RMSE of the fitted image against the target",
                      "value": e_fit, "unit": "relative RMSE", "higher_is_better": False,
                      "config": {"workload": "volume scene 256x256, depth 32, 25 bands; 79 parameters (2x25 wall "
                                             "albedos, 25-band sigma_a, g, 3 roughnesses); target 4,100 spp of "
                                             "seed 7, start seed 8, Adam lr 1e-2, 50 passes per forward and adjoint",
                                 "iterations": args.iterations},
                      "image_rmse": {"init": e_init, "fitted": e_fit, "hidden_params_at_same_spp": e_hidden},
                      "loss": {"first": hist[0], "last": hist[-1], "noise_floor": floor,
                               "history_every_10": hist[::10]},
                      "seconds_per_iteration": t_fit / args.iterations, "target_seconds": t_target,
                      "parameter_error": {"init": inverse.parameter_error(init, hidden),
                                          "fitted": inverse.parameter_error(fit, hidden)},
                      "device_error_bits": bits}))


def bench_rmse(args):
    """Seconds to a relative XYZ RMSE target on the single-scene workloads:
    the batched renderer (the autotuned wavelength bundles) renders blocks
    until the image's estimated RMSE reaches the target (measured end to end,
    with the bias check against the FP64 oracle image); the plain single-scene
    kernel is timed on the same paths.  Prints one JSON line."""
    rank, world, _ = dist_env()
    sampler = ClockSampler(gpu_uuid(0))
    sampler.start()
    legs = []
    for name in args.rmse_workloads.split(","):
        leg = rmse_leg(name, args.rmse_target, args.rmse_seconds, bundles=True)
        leg["plain"] = plain_seconds(name, leg["blocks"])
        leg["speedup_vs_plain"] = leg["plain"]["seconds_same_paths"] / leg["seconds"]
        legs.append(leg)
    clocks = sampler.stop()
    print(json.dumps({"metric": f"seconds to {args.rmse_target:.0%} relative XYZ RMSE", "unit": "s",
                      "higher_is_better": False, "n_gpus": 1, "data": "synthetic (seeded procedural scenes)",
                      "legs": legs, "clocks": clocks}))


def adjoint_leg():
    """Cost of the path-replay adjoint against the forward pass on the
    inverse-rendering scene (box + HG medium + fluorescent wall, 256^2, depth 32)."""
    import torch
    import spectral_b200 as sb
    from spectral_b200 import configs
    s, c, ex = configs.volume_scene(width=256, height=256, depth=32)
    c.kernel = "mega"
    r = sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"])
    B = c.bands
    pm, pe = r.param_count()
    adj = torch.rand((B, c.height, c.width), dtype=torch.float64, device="cuda")
    g = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
    r.cast_rays_bundle(0, B, pass_idx=0)
    r.adjoint_passes(0, B, 0, adj, g)
    r.cast_rays(0, pass_idx=0)

    def timed(fn, n):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    n = 2 * B
    f1 = timed(lambda: [r.cast_rays(p % B, pass_idx=1000 + p) for p in range(n)], n)
    fb = timed(lambda: [r.cast_rays_bundle(0, B, pass_idx=1000 + i * B) for i in range(2)], n)
    ab = timed(lambda: r.adjoint_passes(0, n, 1000, adj, g), n)  # both replays
    # the inverse workflow: the forward bundles record each path's total deposit,
    # the adjoint of the same passes then needs one replay per path
    r.record_paths(2000, n)
    fr = timed(lambda: [r.cast_rays_bundle(0, B, pass_idx=2000 + i * B) for i in range(2)], n)
    ar = timed(lambda: r.adjoint_passes(0, n, 2000, adj, g), n)
    r.record_paths(0, 0)
    bits = r.check_device()
    r.close()
    return {"workload": "inverse-rendering scene: box + 20k-tri HG medium (g 0.7) + fluorescent wall, 256x256, "
                        "depth 32, 25 bands; parameters " + str(pm + pe),
            "forward_ms_per_pass": f1, "forward_bundle_ms_per_pass": fb,
            "forward_bundle_recorded_ms_per_pass": fr, "adjoint_ms_per_pass": ar,
            "adjoint_two_replays_ms_per_pass": ab,
            "adjoint_over_forward": ar / f1, "adjoint_over_forward_bundle": ar / fb,
            "adjoint_over_recorded_forward_bundle": ar / fr,
            "what": "adjoint of passes whose forward bundles recorded each path's total deposit (ts_record_paths: "
                    "one gradient replay per path); adjoint_two_replays_ms_per_pass is the same adjoint without "
                    "records (weight replay + gradient replay)",
            "device_error_bits": bits}


def bench_adjoint(args):
    """Path-replay adjoint on the inverse-rendering scene: --steps launches of
    --passes passes each after --warmup, CUDA events; prints one JSON line."""
    import torch
    import spectral_b200 as sb
    from spectral_b200 import configs
    s, c, ex = configs.volume_scene(width=256, height=256, depth=32)
    c.kernel = "mega"
    r = sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"])
    B = c.bands
    pm, pe = r.param_count()
    adj = torch.rand((B, c.height, c.width), dtype=torch.float64, device="cuda")
    g = torch.zeros(pm + pe, dtype=torch.float64, device="cuda")
    P = args.passes
    for w in range(args.warmup):
        r.adjoint_passes(0, P, w * P, adj, g)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        r.adjoint_passes(0, P, (args.warmup + k) * P, adj, g)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    bits = r.check_device()
    r.close()
    paths = P * c.width * c.height
    print(json.dumps({"metric": "adjoint Mpaths/s", "value": paths / (ms * 1e-3) / 1e6, "unit": "Mpaths/s",
                      "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup, "n_gpus": 1,
                      "higher_is_better": True, "data": "synthetic (seeded procedural scene)",
                      "config": {"workload": f"inverse-rendering scene 256x256, depth 32; one step = the adjoint of "
                                             f"{P} passes", "parameters": pm + pe},
                      "device_error_bits": bits}))


def turned_camera(cam, degrees):
    """The camera at the same position, turned by ``degrees`` about its up axis."""
    import numpy as np
    o, c, u = (np.asarray(cam[k], np.float64) for k in ("origin", "lookat", "up"))
    u = u / np.linalg.norm(u)
    v = c - o
    a = np.radians(degrees)
    v = v * np.cos(a) + np.cross(u, v) * np.sin(a) + u * np.dot(u, v) * (1.0 - np.cos(a))  # Rodrigues
    return {"origin": o.tolist(), "lookat": (o + v).tolist(), "up": u.tolist()}


def bench_batch(args):
    """Batched workload: scenes of seeds 100.. (box / terrain / volume, 1k-500k
    triangles, 128^2-512^2, depth 4-16), the first --batch-views of them with
    a second camera (a view: another context on the same scene upload), each
    image rendered to a relative XYZ RMSE target: one image at a time with one
    megakernel launch per pass (plain), and all images together by the batched
    persistent megakernel replayed as a CUDA graph (kernel), by the batch loop
    (every image's block in one regenerating wavefront loop per step, one
    CUDA graph), and by the stream engine (each image's block one loop launch,
    images overlapping on a pool of streams).  The megakernel arms use two-child
    BVH nodes, the loop arms four-child nodes (each kernel's faster layout).

    Every arm renders the same paths (the same pass indices of the same random
    streams) and checks its estimate on the same schedule, so each arm needs
    the same blocks per image.  With --batch-plain-blocks N the plain arm is
    timed on N blocks of every image and its time to the target is the sum over
    images of (blocks the batched engines needed) x (measured seconds per
    block): a measured per-image throughput, not an extrapolated error."""
    import numpy as np
    import torch
    import spectral_b200 as sb
    from spectral_b200 import batch as sbatch
    from spectral_b200 import configs
    t0 = time.time()
    work = configs.batch_workload(100, args.batch_scenes)
    nviews = max(0, min(args.batch_views, len(work)))

    def image_set(width):
        owners, views = [], []
        for sc, cf, ex in work:
            cf.kernel = "mega"
            owners.append(sb.Renderer(sc, cf, eems=ex["eems"], cmf=ex["cmf"], bvh_params={"width": width}))
        for k in range(nviews):
            views.append(owners[k].view(camera=turned_camera(work[k][0]["camera"], 20.0)))
        return owners, owners + views

    engines_wanted = [e for e in args.batch_engines.split(",") if e]
    assert engines_wanted and all(e in ("kernel", "loop", "streams") for e in engines_wanted), args.batch_engines
    sets = {2: image_set(2)}
    if any(e in ("loop", "streams") for e in engines_wanted):
        sets[4] = image_set(4)
    build_s = time.time() - t0
    rs = sets[2][1]
    B = rs[0].config.bands
    target = args.batch_target
    limit = args.batch_seconds if args.batch_seconds > 0 else None

    def plain_block(r, nb):
        for k in range(B):
            r.cast_rays(k, pass_idx=nb * B + k)
        r.average_and_reset_block(nb + 1)

    plain, plain_block_s = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in rs:
        r.clear_pixel_space()
        if args.batch_plain_blocks > 0:
            torch.cuda.synchronize()
            ts0 = time.perf_counter()
            for nb in range(args.batch_plain_blocks):
                plain_block(r, nb)
            torch.cuda.synchronize()
            plain_block_s.append((time.perf_counter() - ts0) / args.batch_plain_blocks)
            continue
        nb, due = 0, 2
        while True:
            plain_block(r, nb)
            nb += 1
            if nb >= due:  # the same checking policy as Batch.render_to_rmse
                e = sbatch.relative_rmse_estimate(r, nb)
                if e <= target:
                    break
                due = sbatch.next_check(nb, e, target)
        plain.append(nb)
    torch.cuda.synchronize()
    tp = time.perf_counter() - t0
    from spectral_b200 import autotune
    results, bits, tune = {}, 0, None
    for name in engines_wanted:
        if name == "kernel":
            t0 = time.time()
            (bs, bpsm, occ), _ = autotune.tune_batch(rs, steps=1)
            tune = {"block_size": bs, "blocks_per_sm": bpsm, "occupancy": occ, "seconds": time.time() - t0}
            imgs = rs
            eng = sbatch.Batch(imgs, block_size=bs, blocks_per_sm=bpsm, occupancy=occ, use_graph=True)
            what = "all images in one persistent megakernel launch per step (CUDA graph), two-child nodes"
        elif name == "loop":
            imgs = sets[4][1]
            eng = sbatch.Batch(imgs, kernel="wavefront", use_graph=True, queue_capacity=1 << 25, trace_budget=16)
            what = "all images in one regenerating wavefront loop per step (one CUDA graph), four-child nodes"
        else:
            imgs = sets[4][1]
            eng = sbatch.StreamBatch(imgs, streams=8)
            what = "per image one regenerating wavefront loop per block, 8 streams, four-child nodes"
        with eng as b:
            b.reset()
            b.step()
            b.reset()
            blocks, secs = b.render_to_rmse(target=target, max_seconds=limit)
            bits |= b.check()
            est = [float(sbatch.relative_rmse_estimate(r, int(n))) for r, n in zip(imgs, blocks)]
        paths = sum(int(n) * B * r.config.width * r.config.height for n, r in zip(blocks, imgs))
        results[name] = {"seconds": secs, "mpaths_per_s": paths / secs / 1e6, "blocks": [int(x) for x in blocks],
                         "reached": bool(max(est) <= target), "max_estimated_rmse": max(est), "what": what}
    if args.batch_plain_blocks > 0:
        need = results[engines_wanted[0]]["blocks"]
        tp = sum(n * t for n, t in zip(need, plain_block_s))
        plain = need
    for v in results.values():
        v["speedup"] = tp / v["seconds"]
    best = min(results, key=lambda k: results[k]["seconds"])
    line = {"metric": f"seconds to {target:.0%} relative XYZ RMSE, all images", "value": results[best]["seconds"],
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "impl": "ours",
            "data": "synthetic (seeded procedural scenes)",
            "config": {"workload": f"{len(work)} scenes of seeds 100-{99 + len(work)}: box / terrain / volume, "
                                   "1k-500k triangles, 128^2-512^2, depth 4-16; a second camera (turned 20 "
                                   f"degrees) on the first {nviews}: {len(rs)} images",
                       "scene_build_seconds": build_s},
            "plain_seconds": tp, "batched_seconds": results[best]["seconds"],
            "speedup": tp / results[best]["seconds"], "engine": best,
            "plain": {"what": "one image at a time, one megakernel launch per pass (the reference's cadence), "
                              "two-child nodes",
                      "timed": ("%d blocks per image, scaled by the blocks the engines needed" % args.batch_plain_blocks
                                if args.batch_plain_blocks > 0 else "run to the target"),
                      "blocks": [int(x) for x in plain],
                      "seconds_per_block": plain_block_s or None},
            "engines": results, "batch_autotune": tune, "device_error_bits": bits,
            "images": [{"res": r.config.width, "tris": r.compiled.num_tris, "depth": r.config.max_path_length,
                        "view": k >= len(work)} for k, r in enumerate(rs)]}
    for owners, imgs in sets.values():
        for r in imgs[len(owners):]:
            r.close()
        for r in owners:
            r.close()
    print(json.dumps(line))


def bench_reference(args):
    """CPU arm: the reference's estimator (the oracle restatement, pinned to the
    reference's own code) on all host threads, traversing the reference's BVH
    algorithm in the reference's order without distance culling.  Loads no
    part of the CUDA library: the scene comes from the workload generator and
    the host-side flattening (pure Python), the tree from the oracle.  Each
    step renders a random pixel sample of every pass of one spectral block
    (the same 25 band-passes as a GPU step), sized so that the run ends in a
    few minutes."""
    import numpy as np
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from spectral_b200 import scene as sbscene
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    scene, cfg, ex, desc = workload(args.workload)
    comp = sbscene.compile_scene(scene, cfg.bands, eems=ex["eems"], cmf=ex["cmf"])
    t0 = time.perf_counter()
    bvh = reference_tree(comp)
    tree_s = time.perf_counter() - t0
    osc = orc.oracle_scene(comp, bvh, scene["camera"])
    ocfg = orc.oracle_config(cfg)
    B = cfg.bands
    npix = cfg.width * cfg.height
    rng = np.random.default_rng(7)
    pix = rng.choice(npix, 1024, replace=False).astype(np.int32)
    t = time.perf_counter()
    orc.render_pass(osc, ocfg, 0, 0, pix)
    rate = 1024 / max(time.perf_counter() - t, 1e-6)
    # pixels per pass of a step: ~150 s for the whole run, at most 2 s a step
    per_pass = int(min(npix, max(64, rate * min(2.0, 150.0 / max(1, args.steps + args.warmup)) / B)))

    def step(k):
        for b in range(B):
            px = rng.choice(npix, per_pass, replace=False).astype(np.int32)
            orc.render_pass(osc, ocfg, k * B + b, b, px)

    for w in range(args.warmup):
        step(w)
    t = time.perf_counter()
    for k in range(args.steps):
        step(args.warmup + k)
    total = time.perf_counter() - t
    mpaths = per_pass * B * args.steps / total / 1e6
    threads = os.cpu_count() or 1
    sample = (f"{per_pass} random pixels of each of the {B} band-passes of a step (of {npix} per pass); "
              f"reference BVH algorithm (full-sweep SAH, built in {tree_s:.1f} s), reference traversal order")
    line = {"impl": "reference", "metric": "Mpaths/s", "value": mpaths, "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene; no dataset)",
            "config": step_config(cfg, ex, desc, world, comp.num_tris),
            "cpu_baseline": {"value": mpaths, "unit": "Mpaths/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": mpaths, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def bench_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import spectral_b200 as sb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        # bounded wait: ranks build their scene and tune before the first barrier
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    scene, cfg, ex, desc = workload(args.workload)
    cfg.kernel = args.kernel
    cfg.traversal = args.traversal
    cfg.trace_budget = args.budget
    cfg.occupancy = args.occupancy
    cfg.queue_capacity = args.queue_capacity
    cfg.loop_host = 1 if args.loop_host else 0
    cfg.device = local
    tuned = None
    if not args.no_tune:
        # launch configuration chosen by the autotuner (megakernel candidates: BVH width,
        # traversal loop, block shape, register budget; for bundles also the regenerating
        # wavefront loop's queue capacity); every candidate renders the same paths
        from spectral_b200 import autotune
        t0 = time.time()
        bundles = args.launch == "bundle"
        best, table = autotune.tune(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], quick=True,
                                    passes=50 if bundles else 6, first_pass=1 << 26, bundles=bundles)
        cfg = best.apply(cfg)
        args.width, args.kernel, args.traversal, args.occupancy = best.width, best.kernel, best.traversal, best.occupancy
        args.quantize = best.quantize
        tuned = {"seconds": time.time() - t0, "candidates": len(table),
                 "best": {"width": best.width, "quantize": best.quantize, "traversal": best.traversal,
                          "kernel": best.kernel,
                          "block_size": best.block_size, "blocks_per_sm": best.blocks_per_sm,
                          "occupancy": best.occupancy, "queue_capacity": best.queue_capacity,
                          "trace_budget": best.trace_budget},
                 "ms_per_pass": {f"w{c.width}{'q' if c.quantize else ''}/{c.traversal}/{c.kernel}/b{c.block_size}/s{c.blocks_per_sm}"
                                 f"/o{c.occupancy}/q{c.queue_capacity}/t{c.trace_budget}": round(ms, 4)
                                 for c, ms in table}}
    comp = sb.compile_scene(scene, cfg.bands, eems=ex["eems"], cmf=ex["cmf"])
    bvh = sb._lib.build_bvh_host(comp.tris["v0"], comp.tris["v1"], comp.tris["v2"], leaf_max=args.leaf_max,
                                 cost_trav=args.cost_trav)
    r = sb.Renderer(scene, cfg, eems=ex["eems"], cmf=ex["cmf"], bvh=bvh,
                    bvh_params={"width": args.width, "quantize": args.quantize})
    B = cfg.bands
    npix = cfg.width * cfg.height
    paths_per_step = B * npix  # one step = one spectral block of B passes
    base_pass = rank * (args.warmup + args.steps + 64) * B * 4  # disjoint random streams per rank
    use_bundles = args.launch == "bundle" and (args.kernel == "mega" or cfg.sort_keys == 0)
    wave_loop = args.kernel == "wavefront" and (use_bundles or cfg.queue_capacity > 0) and cfg.sort_keys == 0

    def step(k, first_pass):
        """Step k: the B passes of one spectral block (bands 0..B-1)."""
        p0 = first_pass + k * B
        if use_bundles:
            r.cast_rays_bundle(0, B, pass_idx=p0)
        else:
            for b in range(B):
                r.cast_rays(b, pass_idx=p0 + b)

    # warm-up, then one counted pass (work counters for the roofline's algorithmic bytes)
    for w in range(args.warmup):
        step(w, base_pass)
    work = r.cast_rays_counted(12, pass_idx=base_pass + 1)
    torch.cuda.synchronize()
    info = r.scene_info()
    node_bytes = (BYTES_NODE_Q[info["node_width"]] if info["node_quantized"]
                  else BYTES_NODE * (info["node_width"] // 2))  # 2 -> 64 B, 4 -> 128 B, 8 -> 256 B
    bytes_per_path = (node_bytes * work["node_visits"] + BYTES_TRI * work["tri_tests"] + BYTES_HIT * work["hits"]
                      + BYTES_MAT_VERTEX * work["vertices"] + BYTES_DEPOSIT * work["deposits"]) / work["paths"]

    # ---- timed region: K steps, device time, max over ranks
    sampler = ClockSampler(gpu_uuid(local))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timed_first = base_pass + (args.warmup + 1) * B
    e0.record()
    for k in range(args.steps):
        step(k, timed_first)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps * paths_per_step / (ms_max * 1e-3) / 1e6
    bits = r.check_device()

    # ---- kernels launched in the timed region: the same steps again, untimed
    # (the same passes, so the same paths), reading each loop launch's iterations
    if wave_loop:
        iters = []
        for k in range(args.steps):
            if use_bundles:
                step(k, timed_first)
                iters.append(r.wave_loop_iterations())
            else:
                for b in range(B):
                    r.cast_rays(b, pass_idx=timed_first + k * B + b)
                    iters.append(r.wave_loop_iterations())
        # a loop launch: the init kernel, then trace + shade + control per iteration
        gpu_launches = sum(1 + 3 * it for it in iters)
        launches = ("one regenerating wavefront loop per %s (init kernel, then a CUDA-graph while-loop of trace, "
                    "shade, control; %.1f iterations per launch)" % ("step (25-pass bundle)" if use_bundles
                                                                     else "pass", sum(iters) / len(iters)))
    elif args.kernel == "mega":
        gpu_launches = args.steps * (1 if use_bundles else B)
        launches = "one megakernel launch per " + ("step (25-pass bundle)" if use_bundles else "pass")
    else:
        gpu_launches = args.steps * B * (2 + 2 * cfg.max_path_length)
        launches = "depth-synchronous wavefront: generate, then trace + shade per depth, per pass"
    torch.cuda.synchronize()

    # ---- end to end through the public API with host buffers, at the
    # reference's cadence (main.py:1826-1837): per step the camera in, one
    # block of B passes, the block folded into the running mean
    # (average_and_reset_block) and the resolved XYZ image out (pinned)
    out = torch.empty((cfg.height, cfg.width, 3), dtype=torch.float32, pin_memory=True).numpy()
    cam = scene["camera"]
    r.clear_pixel_space()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_first = base_pass + (args.warmup + args.steps + 8) * B
    f0.record()
    for k in range(args.steps):
        r.update_camera(cam["origin"], cam["lookat"], cam["up"])
        step(k, e2e_first)
        r.average_and_reset_block(k + 1)
        r.resolve_xyz_host(out)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    t2 = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps * paths_per_step / (float(t2.item()) * 1e-3) / 1e6

    peak, peak_src = measured_peak()
    step_s = ms_max * 1e-3 / args.steps
    achieved = bytes_per_path * paths_per_step / step_s / 1e9
    traffic = profiled_traffic(args.kernel, args.workload, f"{args.width}q" if args.quantize else args.width,
                               0 if wave_loop else args.occupancy, use_bundles)
    kernel_name = ("k_render_mega" if args.kernel == "mega" else
                   "regenerating wavefront loop (k_trace + k_shade_loop + k_loop_control per iteration)"
                   if wave_loop else "depth-synchronous wavefront pass")

    line = {"metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene; no dataset)",
            "config": step_config(cfg, ex, desc, world, comp.num_tris),
            "launch": {"kernel": args.kernel, "bvh_width": args.width, "bvh_quantized": bool(args.quantize),
                       "node_bytes": node_bytes, "traversal": args.traversal,
                       "bvh_leaf_max": args.leaf_max or 8, "bvh_cost_trav": args.cost_trav or 1.0,
                       "occupancy": args.occupancy, "queue_capacity": cfg.queue_capacity,
                       "block_size": cfg.block_size, "trace_budget": cfg.trace_budget, "launches": launches},
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 36,
                    "d2h_bytes_per_step": int(out.nbytes),
                    "what": "per step (one spectral block): Renderer.update_camera + %s + "
                            "average_and_reset_block + resolve_xyz_host (pinned host XYZ image), through the C ABI"
                            % ("cast_rays_bundle of the block's %d passes" % B if use_bundles
                               else "%d cast_rays" % B)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": None if traffic is None else traffic * B,
                         "traffic_per": "step (one 25-pass launch): DRAM bytes per pass of the committed ncu capture "
                                        "(profiles/traffic.json, its source says which case) x 25 passes",
                         "kernel": kernel_name, "bytes_per_path": bytes_per_path,
                         "bytes_per_launch": bytes_per_path * paths_per_step, "peak_source": peak_src,
                         "work_per_path": {k: v / work["paths"] for k, v in work.items() if k != "paths"}},
            "gpu_launches": int(gpu_launches),
            "autotune": tuned,
            "clocks": clocks, "device_error_bits": bits}

    line["vertices_per_s"] = value * 1e6 * work["vertices"] / work["paths"]
    # the same passes with one launch per pass (the reference's cadence), for comparison
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n1 = 2 * B
    h0.record()
    for k in range(n1):
        r.cast_rays(k % B, pass_idx=base_pass + 40000 + k)
    h1.record()
    torch.cuda.synchronize()
    line["one_launch_per_pass"] = {"value": npix / (h0.elapsed_time(h1) / n1 * 1e-3) / 1e6,
                                   "unit": "Mpaths/s", "ms_per_pass": h0.elapsed_time(h1) / n1}
    if rank == 0 and world == 1 and not args.no_extras:
        # the plain single-scene wavefront kernel on the same workload (same paths)
        r.set_launch_config(kernel="wavefront", traversal="default", block_size=128, blocks_per_sm=0, sort_keys=0,
                            trace_budget=16, occupancy=0, queue_capacity=0)
        for k in range(3):
            r.cast_rays(k % B, pass_idx=base_pass + 41000 + k)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nw = 2 * B
        g0.record()
        for k in range(nw):
            r.cast_rays(k % B, pass_idx=base_pass + 41100 + k)
        g1.record()
        torch.cuda.synchronize()
        wms = g0.elapsed_time(g1) / nw
        line["plain_wavefront"] = {"value": npix / (wms * 1e-3) / 1e6, "unit": "Mpaths/s",
                                   "ms_per_pass": wms, "bvh_width": args.width, "trace_budget": 16}
    if rank == 0 and world == 1 and not args.no_extras:
        line["rmse"] = [rmse_leg("box", 0.01, args.rmse_seconds, bundles=True),
                        rmse_leg("box", 0.01, args.rmse_seconds, bundles=False),
                        rmse_leg("terrain", 0.05, args.rmse_seconds, bundles=True),
                        rmse_leg("volume", 0.05, args.rmse_seconds, bundles=True)]
        line["adjoint"] = adjoint_leg()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, n, dt, threads, st = cpu_oracle_rate(comp, reference_tree(comp), scene, cfg, seconds=12.0)
        line["cpu_baseline"] = {"value": rate / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "port",
                                "sample": f"{n} paths of the workload's band-passes ({dt:.1f} s, FP32 oracle "
                                          f"pinned to the reference's code, reference BVH algorithm and "
                                          f"traversal order)"}
    r.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        bench_reference(a)
    elif a.workload == "batch":
        bench_batch(a)
    elif a.workload == "adjoint":
        bench_adjoint(a)
    elif a.workload == "rmse":
        bench_rmse(a)
    elif a.workload == "gradcheck":
        bench_gradcheck(a)
    elif a.workload == "inverse":
        bench_inverse(a)
    else:
        bench_ours(a)
