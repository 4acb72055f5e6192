"""Benchmark: Mpaths/s of the path-tracing hot path at 1080p.

One step = one frame of the large plain render: 1920x1080, 16 spp, depth 8,
64 instances of a 158,420-triangle displaced sphere (10.14M triangles, a
649 MB flattened BVH), 8 procedural 2048^2 textures, GGX / dielectric /
Lambert materials and an environment light with a sun lobe.  The frame is
PathTracer::execute (wavefront: generate, extend, shade, shadow, finalize)
followed by the fused reduce + accumulate + tonemap resolve.  Synthetic,
seeded inputs stand in for the reference's USD scenes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl strelka|reference]

N > 1 runs under torchrun, one rank per GPU: every rank renders its own
frames (distinct sample seeds) of the same scene, so per-GPU work is fixed
(weak scaling) and there is no collective on the data path.  Rank 0 prints
one JSON line.

--impl reference times the reference's algorithm on the host cores: the
oracle's C restatement of the shaders (the reference's HLSL cannot run here:
there is no Vulkan device or software renderer), all host threads, on a
bounded sample of each frame's paths.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mpaths/s at 1080p"
UNIT = "Mpaths/s"

# DRAM bytes (read + write) per closest-hit query of the extend kernel on the
# large scene, from one ncu capture of the five extend launches of a
# 960x540 x 4 spp frame (dram__bytes_read.sum + dram__bytes_write.sum =
# 1714.7 MB for 4,300,568 queries).  The per-query figure falls as the frame
# grows (496 B per query at 480x270 x 4 spp): more queries share the cached
# nodes.  bench.py cannot run ncu itself, so roofline.traffic is this figure
# times the queries of an average launch, an upper bound for the full frame.
EXTEND_DRAM_BYTES_PER_RAY = 398.7

# DRAM bytes (read + write) per closest-hit query of the ray-query kernel on
# the 1M-triangle soup, from one ncu capture of a timed launch with 4M rays
# (1404.8 + 122.1 MB); 380.0 B per query with 1M rays, so the figure scales
# with the number of rays.
TRACE_SOUP_DRAM_BYTES_PER_RAY = 381.7

# Bytes a traversal reads per 4-wide node it processes: the bounds of its four
# entries (6 float4) and their refs (1 float4).
WIDE_NODE_BYTES = 112


def workload_config(args):
    return {
        "workload": "large plain render: 1920x1080, 16 spp, depth 8, 64 instances x 158,420-tri displaced sphere "
                    "(10.14M tris), 8x 2048^2 RGBA8 textures, GGX/dielectric/Lambert, 1024x512 HDR env with sun lobe",
        "width": args.width, "height": args.height, "spp": args.spp, "max_depth": args.depth,
        "instances": args.instances, "triangles": None, "mode": args.mode,
        "l2": "inputs larger than L2 (649 MB BVH, 128 MB textures per frame)",
    }


def make_scene(args):
    from strelka_b200 import scenes

    return scenes.large(width=args.width, height=args.height, instances=args.instances, frequency=args.frequency,
                        num_textures=8, tex_size=2048, env_width=1024, env_height=512, max_depth=args.depth,
                        spp=args.spp, seed=0)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.strip().split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(hs, args, budget_s: float, frame_number: int = 0, per: int | None = None):
    """Times the oracle (fast build, all host threads) on 64 evenly spaced,
    non-overlapping runs of the frame's sample indices.  Calibration passes
    (64 paths per run, growing 4x until a pass takes a tenth of `budget_s`)
    give the rate; the timed pass then renders as many paths per run as fit
    `budget_s`.  `per` skips the calibration and renders that many paths per
    run.  Returns (Mpaths/s, paths, threads, seconds)."""
    import oracle

    view = oracle.SceneView(hs)
    p = hs.param(frameNumber=frame_number)
    total = args.width * args.height * args.spp
    threads = os.cpu_count() or 1
    slices = 64

    def run(per):
        t = time.perf_counter()
        for k in range(slices):
            oracle.pathtrace(view, p, threads=threads, first=(k * total) // slices, count=per, fast=True)
        return time.perf_counter() - t

    most = max(total // slices, 1)
    if per is None:
        # calibration passes grow 4x until one takes a tenth of the budget: a
        # short pass is mostly per-call overhead and would understate the rate
        per = min(64, most)
        while True:
            el = run(per)
            if el >= 0.1 * budget_s or per >= most:
                break
            per = min(per * 4, most)
        rate = slices * per / max(el, 1e-6)
        per = int(min(max(rate * budget_s / slices, 64), most))
    el = run(per)
    done = slices * per
    return done / el / 1e6, done, threads, el


def frame_parity(hs, p, sb, slices: int = 64, per: int = 1024):
    """Parity of one rendered frame: the oracle (exact build, no FMA
    contraction) renders `slices` evenly spaced runs of `per` sample indices
    of the frame with parameters `p`, and they are compared with the GPU's
    sample buffer `sb` of that frame: relMSE (mean over samples and channels
    of (x - y)^2 / (y^2 + 1e-2)) and the fraction of bit-identical values."""
    import oracle

    view = oracle.SceneView(hs)
    total = p.dimension[0] * p.dimension[1] * p.spp
    per = min(per, total // slices) if total >= slices else total
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    got, ref = [], []
    for k in range(slices if total >= slices else 1):
        first = (k * total) // slices
        ref.append(oracle.pathtrace(view, p, threads=threads, first=first, count=per))
        got.append(sb[first * 3:(first + per) * 3].cpu().numpy())
    el = time.perf_counter() - t0
    g = np.concatenate(got).astype(np.float64)
    r = np.concatenate(ref).astype(np.float64)
    rel = float(np.mean((g - r) ** 2 / (r * r + 1e-2)))
    exact = float(np.mean(np.concatenate(got).view(np.uint32) == np.concatenate(ref).view(np.uint32)))
    return {"samples": int(g.size // 3), "relmse": rel, "bit_exact_frac": exact, "frame_number": int(p.frameNumber),
            "bar": "relMSE <= 1e-4 against the oracle at the same seeds", "oracle_seconds": round(el, 2),
            "sample": f"{slices} evenly spaced runs of {per} sample indices of the frame"}


def run_reference(args):
    """--impl reference: rank 0 times the oracle on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    from strelka_b200 import scenes

    # the scene comes from the CPU-only build of the generators: this arm
    # never loads the CUDA library
    scenes.use_generator_library(oracle.workload())
    hs = make_scene(args)
    vals = []
    per = None
    for step in range(args.warmup + args.steps):
        v, n, threads, el = cpu_baseline(hs, args, budget_s=args.ref_step_seconds, per=per)
        per = n // 64  # the first step's calibrated size for every step
        if step >= args.warmup:
            vals.append((v, n, el))
    value = statistics.median(v for v, _, _ in vals)
    n = vals[-1][1]
    cfg = workload_config(args)
    cfg["triangles"] = hs.num_triangles
    sample = (f"{n} paths per step in 64 evenly spaced slices of the frame's {args.width * args.height * args.spp} "
              f"sample indices, oracle C restatement (-O3 -ffp-contract=fast), OpenMP")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(el for _, _, el in vals),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": cfg, "parallelism": f"host cores x{threads}",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def traversal_study(args, steps: int, warmup: int) -> dict:
    """The ray-query microbenchmark: the --tris-triangle soup with --rays rays,
    closest hit (tmax 1e9) and any hit (tmax uniform in [0.1, 2]), each timed
    over `steps` launches after `warmup` with CUDA events on the launching
    stream.  Algorithmic bytes per query: 112 B per 4-wide node processed,
    48 B per triangle test, 32 B ray in, 20 B hit out (counted exactly by an
    untimed counting replay)."""
    import torch

    from strelka_b200 import abi, scenes
    from strelka_b200.render import DeviceScene, PathTracer, to_device

    hs = scenes.soup(args.tris, 0)
    ds = DeviceScene(hs)
    n = args.rays
    res = {}
    stream = torch.cuda.current_stream()
    peak, peak_src = hbm_peak()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    for name, shadow, flags in (("closest", False, abi.TRACE_CLOSEST), ("any", True, abi.TRACE_ANY)):
        rays = to_device(scenes.rays_soup(n, 1 if not shadow else 2, shadow=shadow))
        hits = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
        pt = PathTracer()
        desc = ds.trace_desc(rays, hits, flags)
        for _ in range(warmup):
            pt.trace(desc, stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            pt.trace(desc, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        pt.trace(ds.trace_desc(rays, hits, flags | abi.TRACE_COUNT, cnt), stream)
        c = cnt.cpu().numpy()
        out_bytes = 20
        bytes_alg = WIDE_NODE_BYTES * int(c[0]) + 48 * int(c[1]) + (32 + out_bytes) * n
        st = pt.device_status()
        pt.close()
        if st != 0:
            raise RuntimeError(f"device status {st:#x}")
        res[name] = {"mrays_s": n / (ms * 1e-3) / 1e6, "ms_per_launch": ms, "nodes_per_ray": c[0] / n,
                     "tests_per_ray": c[1] / n, "bytes_alg_per_launch": bytes_alg,
                     "achieved_gbs": bytes_alg / (ms * 1e-3) / 1e9,
                     "frac": bytes_alg / (ms * 1e-3) / 1e9 / peak}
    clk = clocks.stop()
    return {"workload": f"traversal microbenchmark: {args.tris} soup triangles (centroids uniform in the unit cube, "
                        f"log-normal vertex offsets mu=ln 0.003 sigma=0.5), {n} rays (origins uniform in "
                        f"[-0.5,1.5]^3, directions uniform on the sphere), closest hit and any hit",
            "triangles": hs.num_triangles, "rays": n, "steps": steps, "warmup": warmup, "peak_gbs": peak,
            "peak_source": peak_src, "target_frac": 0.60, "closest": res["closest"], "any": res["any"],
            "clocks": clk, "l2": "inputs larger than L2"}


def run_traversal(args):
    """--workload traversal: traversal_study as its own JSON line."""
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    tr = traversal_study(args, args.steps, args.warmup)
    c = tr["closest"]
    line = {"metric": "Mrays/s (traversal microbenchmark)", "value": c["mrays_s"], "unit": "Mrays/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": tr["workload"], "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "achieved": c["achieved_gbs"], "peak": tr["peak_gbs"], "unit": "GB/s",
                         "frac": c["frac"],
                         "traffic": (TRACE_SOUP_DRAM_BYTES_PER_RAY * tr["rays"]
                                     if (args.tris, args.rays) == (1_000_000, 4_000_000) else None),
                         "traffic_source": "ncu DRAM bytes per query of one closest-hit launch with 4M rays x rays"},
            "detail": tr, "clocks": tr["clocks"]}
    print(json.dumps(line), flush=True)


def cornell_study(args, steps: int = 3, warmup: int = 1) -> dict:
    """The Cornell box at 512x512, 1 spp per iteration x 64 iterations, depth
    4, frameNumber = iteration, accumulated and tonemapped (ACESFitted) every
    iteration: PathTracer::execute then the fused reduce + accumulate +
    tonemap, as PtRender::drawFrame records them (ptrender.cpp:735-862).
    One step is the whole 64-iteration sequence, timed with CUDA events,
    issued call by call (mpaths_s_stream) and replayed from a CUDA graph of
    the same calls (mpaths_s).  The last step's accumulated and tonemapped
    images are compared with the oracle's same chain."""
    import torch

    import oracle
    from strelka_b200 import abi, scenes
    from strelka_b200.render import DeviceScene, PathTracer, accumulation_param, resolve, tonemap_param

    W = H = 512
    iters = 64
    s = scenes.cornell(W, H, sphere_levels=4)
    ds = DeviceScene(s)
    pt = PathTracer(mode=abi.MODE_WAVEFRONT if args.mode == "wavefront" else abi.MODE_MEGAKERNEL)
    npx = W * H
    sb = torch.empty(npx * 3, dtype=torch.float32, device="cuda")
    acc = [torch.zeros(npx * 4, dtype=torch.float32, device="cuda") for _ in range(2)]
    tm = torch.empty(npx * 4, dtype=torch.float32, device="cuda")
    tp = tonemap_param(W, H, 1)
    stream = torch.cuda.current_stream()
    params = [s.param(spp=1, maxDepth=4, frameNumber=it, iteration=it, stratifiedSamplingType=0) for it in range(iters)]
    aps = [accumulation_param(W, H, it) for it in range(iters)]

    def sequence(st):
        for it in range(iters):
            pt.execute(ds.desc(params[it], sb), npx, 1, it, st)
            resolve(params[it], sb, tp, aps[it], acc[it % 2], acc[(it + 1) % 2], tm, None, st)

    def timed(run):
        times = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)

    for _ in range(warmup):
        sequence(stream)
    torch.cuda.synchronize()
    ms_stream = timed(lambda: sequence(stream))
    stream_acc = acc[iters % 2].clone()
    # the same 64 iterations captured once into a CUDA graph (after the
    # frames above, the calls allocate nothing and never synchronise) and
    # replayed: the same kernels with the launch gaps between them removed
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(graph, stream=side):
        sequence(side)
    for _ in range(warmup):
        graph.replay()
    torch.cuda.synchronize()
    ms = timed(graph.replay)
    st = pt.device_status()
    del graph
    pt.close()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")
    if not torch.equal(acc[iters % 2].view(torch.int32), stream_acc.view(torch.int32)):
        raise RuntimeError("the graph's accumulated image differs from the stream-ordered one")
    # the oracle's chain (pathtracerMdl.hlsl, reduction, accumulation, tonemap)
    t0 = time.perf_counter()
    view = oracle.SceneView(s)
    hist = np.zeros(npx * 4, np.float32)
    threads = os.cpu_count() or 1
    for it in range(iters):
        o = oracle.reduce(params[it], oracle.pathtrace(view, params[it], threads=threads))
        hist = oracle.accumulate(aps[it], o, hist)
    o_tm = oracle.tonemap(tp, hist)
    o_s = time.perf_counter() - t0
    g_acc = acc[iters % 2].cpu().numpy()
    g_tm = tm.cpu().numpy()
    rel = float(np.mean((g_acc.astype(np.float64) - hist) ** 2 / (hist.astype(np.float64) ** 2 + 1e-2)))
    return {"workload": "Cornell box 512x512 (10,252 triangles), 1 spp x 64 iterations, depth 4, frameNumber = "
                        "iteration, accumulation + ACESFitted every iteration", "mode": args.mode,
            "launch": "the 64 iterations captured once into a CUDA graph and replayed",
            "mpaths_s": npx * iters / (ms * 1e-3) / 1e6, "ms_per_64_iterations": ms,
            "mpaths_s_stream": npx * iters / (ms_stream * 1e-3) / 1e6, "ms_per_64_iterations_stream": ms_stream,
            "steps": steps, "warmup": warmup,
            "parity": {"relmse_accumulated": rel,
                       "bit_exact_accumulated": float(np.mean(g_acc.view(np.uint32) == hist.view(np.uint32))),
                       "bit_exact_tonemapped": float(np.mean(g_tm.view(np.uint32) == o_tm.view(np.uint32))),
                       "oracle_seconds": round(o_s, 2)}}


def hbm_peak():
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        return json.load(open(peaks_path))["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def nrc_mlp_microbench(torch, RadianceCache, lo, hi, log2t, peak_tflops):
    """Throughput of the cache's fused kernels on resident random records:
    inference over 2^22 queries and one training step (forward + backward
    + Adam) over 2^16 records.  Forward FLOPs per query: 2 x (4 x 64 x 64 +
    16 x 64) = 34,816; a training record costs the forward pass plus about
    twice that backward (input and weight gradients)."""
    rng = np.random.default_rng(0)

    def records(n):
        r = np.zeros((n, 16), np.float32)
        r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
        d = rng.normal(size=(n, 3))
        r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
        nn = rng.normal(size=(n, 3))
        r[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
        r[:, 9] = rng.uniform(0.05, 1.0, n)
        r[:, 10:13] = rng.gamma(1.0, 1.0, (n, 3))
        return torch.from_numpy(r).cuda()

    cache = RadianceCache(lo, hi, seed=5, log2_table_size=log2t)
    out = {}
    n = 1 << 22
    recs = records(n)
    y = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    for _ in range(3):
        cache.infer(recs, n, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        cache.infer(recs, n, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    fl = 34816.0 * n
    out["infer"] = {"queries": n, "ms": ms, "gqueries_s": n / ms / 1e6, "tflops": fl / ms / 1e9,
                    "frac_of_sustained_peak": fl / ms / 1e9 / peak_tflops}
    n = 1 << 16
    recs = records(n)
    for _ in range(3):
        cache.train(recs, n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    for _ in range(20):
        cache.train(recs, n)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 20
    fl = 3 * 34816.0 * n
    out["train_step"] = {"records": n, "ms": ms, "tflops_mlp": fl / ms / 1e9,
                         "note": "includes the loss read-back to the host, the gradient clears and dense Adam "
                                 "over all hash-grid parameters"}
    cache.close()
    return out


def run_nrc_mlp(args):
    """--workload nrc-mlp: the radiance cache's fused kernels alone on
    resident random records (nrc_mlp_microbench), one JSON line."""
    import torch

    from strelka_b200.render import RadianceCache

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak_tf = json.load(open(peaks_path)).get("bf16_tflops_sustained", 1400.0) if os.path.exists(peaks_path) else 1400.0
    lo, hi = np.array([-20.0, -2.0, -20.0], np.float32), np.array([20.0, 8.0, 20.0], np.float32)
    mlp = nrc_mlp_microbench(torch, RadianceCache, lo, hi, args.nrc_log2t, peak_tf)
    line = {"metric": "radiance-cache inference Gqueries/s", "value": mlp["infer"]["gqueries_s"], "unit": "Gqueries/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f16 (f32 accumulation)", "data": "synthetic",
            "config": {"workload": "hash grid (16 levels x 2^%d) + 64-wide 5-layer MLP, random records" % args.nrc_log2t},
            "detail": mlp}
    print(json.dumps(line), flush=True)


def nrc_study(args, hs, ds) -> dict:
    """Wall time of the radiance-cache renderer to reach the relMSE of one
    plain frame (the large render at --spp samples per pixel), both measured
    against a --ref-spp reference of the plain renderer.

    The cached renderer starts from an untrained cache; its warm-up of
    --nrc-warmup training batches (training paths and Adam steps, no image)
    counts toward its time, and then it accumulates frames of --nrc-spp
    samples, training on every frame.  A trial reaches the target when its
    running relMSE is at or below the plain relMSE on two consecutive
    frames; its time runs to the end of the second of them.  Each trial also
    reports its relMSE at equal time: after the last frame that ends within
    the plain frame's wall time.  Every frame is timed with CUDA events on
    the launching stream; relMSE is computed between frames, outside the
    timed intervals."""
    import torch

    from strelka_b200 import abi
    from strelka_b200.render import PathTracer, RadianceCache

    W, H, S = args.width, args.height, args.spp
    npx = W * H
    stream = torch.cuda.current_stream()
    sb = torch.empty(npx * max(S, 16, args.nrc_spp) * 3, dtype=torch.float32, device="cuda")

    def render(pt, fn, spp):
        p = hs.param(spp=spp, frameNumber=fn)
        pt.execute(ds.desc(p, sb), npx * spp, 1, 0, stream)
        return sb[:npx * spp * 3].view(npx, spp, 3)

    def timed(pt, fn, spp, acc):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        img = render(pt, fn, spp)
        acc += img.sum(1, dtype=torch.float64)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    plain = PathTracer(mode=abi.MODE_WAVEFRONT)
    # reference: --ref-spp samples per pixel of the plain renderer, in 16-spp frames
    t0 = time.perf_counter()
    ref = torch.zeros(npx, 3, dtype=torch.float64, device="cuda")
    ref_frames = max(1, args.ref_spp // 16)
    for k in range(ref_frames):
        ref += render(plain, 1_000_000 + k, 16).sum(1, dtype=torch.float64)
    ref /= ref_frames * 16
    torch.cuda.synchronize()
    ref_s = time.perf_counter() - t0
    den = ref * ref + 1e-2

    def relmse(acc, n):
        return float((((acc / n) - ref) ** 2 / den).mean())

    # plain: frames of S spp, each compared with the reference on its own
    for k in range(3):
        render(plain, 10 + k, S)
    plain_ms, plain_err = [], []
    for k in range(max(args.nrc_plain_frames, 8)):
        acc = torch.zeros(npx, 3, dtype=torch.float64, device="cuda")
        plain_ms.append(timed(plain, 2000 + k, S, acc))
        plain_err.append(relmse(acc, S))
    target = statistics.mean(plain_err)
    t_plain = statistics.median(plain_ms)
    st = plain.device_status()
    plain.close()

    lo, hi = hs.bounds()
    trials = []
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    # one renderer for every trial, its buffers allocated by an untimed frame
    # with a throwaway cache (as the plain renderer had warm-up frames); it
    # records no per-kernel events, like the plain renderer
    pt = PathTracer(mode=abi.MODE_WAVEFRONT)
    scratch_cache = RadianceCache(lo, hi, learning_rate=args.nrc_lr, seed=99, log2_table_size=args.nrc_log2t)
    pt.set_nrc(scratch_cache, train_paths=args.nrc_train_paths, train_steps=args.nrc_train_steps,
               diffuse_roughness=args.nrc_diffuse_roughness)
    for k in range(2):
        render(pt, 77 + k, args.nrc_spp)
    pt.train_nrc(ds.desc(hs.param(spp=args.nrc_spp, frameNumber=79), sb), 79, args.nrc_warmup_group, stream)
    torch.cuda.synchronize()
    for trial in range(max(args.nrc_trials, 1)):
        cache = RadianceCache(lo, hi, learning_rate=args.nrc_lr, seed=1 + trial, log2_table_size=args.nrc_log2t)
        pt.set_nrc(cache, train_paths=args.nrc_train_paths, train_steps=args.nrc_train_steps,
                   diffuse_roughness=args.nrc_diffuse_roughness)
        torch.cuda.synchronize()
        base = 100_000 * (trial + 1)
        t_nrc = 0.0
        # warm-up: training only (training paths + Adam steps), no image;
        # --nrc-warmup batches, --nrc-warmup-group of them traced per launch
        for k in range(0, args.nrc_warmup, args.nrc_warmup_group):
            nb = min(args.nrc_warmup_group, args.nrc_warmup - k)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pt.train_nrc(ds.desc(hs.param(spp=args.nrc_spp, frameNumber=base + k), sb), base + k, nb, stream)
            e1.record(stream)
            torch.cuda.synchronize()
            t_nrc += e0.elapsed_time(e1)
        t_warm = t_nrc
        acc = torch.zeros(npx, 3, dtype=torch.float64, device="cuda")
        curve = []
        reached = None
        below = 0
        at_equal_time = None
        frames_ms = []
        for k in range(args.nrc_max_frames):
            ms = timed(pt, base + 50_000 + k, args.nrc_spp, acc)
            frames_ms.append(ms)
            t_nrc += ms
            e = relmse(acc, (k + 1) * args.nrc_spp)
            curve.append([(k + 1) * args.nrc_spp, round(e, 6), round(t_nrc, 3)])
            if t_nrc <= t_plain:
                at_equal_time = e
            below = below + 1 if e <= target else 0
            if below >= 2:
                reached = (k + 1) * args.nrc_spp
                break
        st |= pt.device_status()
        pt.set_nrc(None)
        cache.close()
        trials.append({"reached_at_spp": reached, "ratio": (t_nrc / t_plain) if reached else None, "ms_total": t_nrc,
                       "ms_warmup": t_warm, "ms_per_frame": statistics.median(frames_ms),
                       "relmse_at_plain_time": at_equal_time,
                       "relmse_ratio_at_plain_time": (at_equal_time / target) if at_equal_time is not None else None,
                       "curve_spp_relmse_ms": curve})
    clk = clocks.stop()
    pt.close()
    # per-kernel times of cached frames, from a separate profiling renderer
    # (untimed): the first trial's warm-up and four frames with a fresh cache
    ptp = PathTracer(mode=abi.MODE_WAVEFRONT, profile=True)
    cache = RadianceCache(lo, hi, learning_rate=args.nrc_lr, seed=1, log2_table_size=args.nrc_log2t)
    ptp.set_nrc(cache, train_paths=args.nrc_train_paths, train_steps=args.nrc_train_steps,
                diffuse_roughness=args.nrc_diffuse_roughness)
    for k in range(0, args.nrc_warmup, args.nrc_warmup_group):
        nb = min(args.nrc_warmup_group, args.nrc_warmup - k)
        ptp.train_nrc(ds.desc(hs.param(spp=args.nrc_spp, frameNumber=100_000 + k), sb), 100_000 + k, nb, stream)
    render(ptp, 99, args.nrc_spp)
    torch.cuda.synchronize()
    ptp.kernel_times(stream)
    for k in range(4):
        render(ptp, 150_000 + k, args.nrc_spp)
    times = ptp.kernel_times(stream)
    kernel_ms = {k: v[0] / 4 for k, v in times.items() if v[1]}
    st |= ptp.device_status()
    ptp.set_nrc(None)
    cache.close()
    ptp.close()
    scratch_cache.close()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")
    ratios = sorted(t["ratio"] if t["ratio"] is not None else float("inf") for t in trials)
    median_ratio = ratios[len(ratios) // 2]
    eq = sorted(t["relmse_ratio_at_plain_time"] if t["relmse_ratio_at_plain_time"] is not None else float("inf")
                for t in trials)
    return {
        "metric": "radiance-cache wall time to the plain 16-spp relMSE, relative to plain",
        "median_ratio": median_ratio if median_ratio != float("inf") else None, "unit": "x plain wall time",
        "target": 0.5, "trials_reached": sum(t["ratio"] is not None for t in trials),
        "median_relmse_ratio_at_plain_time": eq[len(eq) // 2] if eq[len(eq) // 2] != float("inf") else None,
        "rule": "reached when the running relMSE is at or below the plain relMSE on two consecutive frames; "
                "time to the end of the second",
        "config": {"workload": f"radiance cache on the large render ({W}x{H}, depth {args.depth}, "
                               f"{args.instances} instances)",
                   "reference_spp": ref_frames * 16, "plain_spp": S, "plain_frames": len(plain_err),
                   "nrc_trials": len(trials), "nrc_spp_per_frame": args.nrc_spp,
                   "nrc_warmup_batches": args.nrc_warmup, "nrc_warmup_batches_per_launch": args.nrc_warmup_group,
                   "train_paths_per_frame": args.nrc_train_paths,
                   "train_steps_per_frame": args.nrc_train_steps, "log2_table_size": args.nrc_log2t,
                   "diffuse_roughness": args.nrc_diffuse_roughness, "learning_rate": args.nrc_lr,
                   "relmse": "mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2)"},
        "plain": {"relmse": target, "relmse_frames": plain_err, "ms": t_plain},
        "trials": trials, "kernel_ms_per_frame_profiled": kernel_ms,
        "reference_seconds": ref_s, "clocks": clk,
    }


def run_nrc(args):
    """--workload nrc: nrc_study as its own JSON line, with the cache's
    fused-kernel microbenchmark."""
    import torch

    from strelka_b200.render import DeviceScene, RadianceCache

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    hs = make_scene(args)
    ds = DeviceScene(hs)
    res = nrc_study(args, hs, ds)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak_tf = json.load(open(peaks_path)).get("bf16_tflops_sustained", 1400.0) if os.path.exists(peaks_path) else 1400.0
    lo, hi = hs.bounds()
    mlp = nrc_mlp_microbench(torch, RadianceCache, lo, hi, args.nrc_log2t, peak_tf)
    line = {
        "metric": res["metric"], "value": res["median_ratio"], "unit": res["unit"], "n_gpus": 1,
        "steps": len(res["plain"]["relmse_frames"]), "warmup": 3, "ms_per_step": res["plain"]["ms"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 render, f16 network (f32 accumulation)", "data": "synthetic", "config": res["config"],
        "plain": res["plain"], "nrc": res, "clocks": res["clocks"], "mlp_microbench": mlp,
    }
    print(json.dumps(line), flush=True)


def batch_jobs(args, rng):
    """The batch workload: --batch-scenes scenes from the large-render
    generator with triangle counts log-uniform in [50k, 10M], and
    --batch-jobs jobs, each a scene with a camera on a random orbit,
    resolution log-uniform from 256x256 to 1920x1080, spp uniform in
    {1..16}, depth 6."""
    from strelka_b200 import scenes

    per_sphere_max = 20 * 89 * 89
    scene_list = []
    for k in range(args.batch_scenes):
        tris = float(np.exp(rng.uniform(np.log(5e4), np.log(1e7))))
        if tris < per_sphere_max:
            inst, freq = 1, max(8, int(round(np.sqrt(tris / 20))))
        else:
            inst, freq = min(64, max(1, int(round(tris / per_sphere_max)))), 89
        hs = scenes.large(width=256, height=256, instances=inst, frequency=freq, num_textures=8, tex_size=2048,
                          env_width=1024, env_height=512, max_depth=6, spp=1, seed=100 + k)
        scene_list.append(hs)
    jobs = []
    for j in range(args.batch_jobs):
        si = int(rng.integers(len(scene_list)))
        t = rng.uniform()
        w = int(round(256 * (1920 / 256) ** t))
        h = int(round(256 * (1080 / 256) ** t))
        spp = int(rng.integers(1, 17))
        a = rng.uniform(0, 2 * np.pi)
        eye = (30 * np.sin(a), 4 + 8 * rng.uniform(), 30 * np.cos(a))
        jobs.append((si, w, h, spp, eye, j))
    return scene_list, jobs


def run_batch(args):
    """--workload batch: the jobs of batch_jobs rendered as one batch
    (autotuned configuration, CUDA graph), timed over --steps executions
    after --warmup, each with new sample seeds; against the same jobs
    rendered one PathTracer::execute at a time (the reference's shape)."""
    import torch

    from strelka_b200 import abi
    from strelka_b200.render import Batch, DeviceScene, PathTracer

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    rng = np.random.default_rng(args.batch_seed)
    t0 = time.perf_counter()
    scene_list, jobs = batch_jobs(args, rng)
    gen_s = time.perf_counter() - t0
    dss = [DeviceScene(hs) for hs in scene_list]
    params, bufs, descs = [], [], []
    for si, w, h, spp, eye, fn in jobs:
        p = scene_list[si].look_at(w, h, eye, (0.0, 1.5, 0.0), 40.0, spp=spp, maxDepth=6, frameNumber=fn)
        sb = torch.empty(w * h * spp * 3, dtype=torch.float32, device="cuda")
        params.append(p)
        bufs.append(sb)
        descs.append(dss[si].desc(p, sb))
    paths = [w * h * spp for _, w, h, spp, _, _ in jobs]
    total = sum(paths)
    stream = torch.cuda.current_stream()
    b = Batch()
    b.set_jobs(descs, stream)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    best, entries = b.autotune(repeats=args.batch_tune_repeats, stream=stream)
    tune_s = time.perf_counter() - t1
    for k in range(args.warmup):
        b.set_frame(1000 + k, stream)
        b.execute(None, stream)
    torch.cuda.synchronize()
    st = b.device_status(stream)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    times, lats = [], []
    for k in range(args.steps):
        b.set_frame(2000 + k, stream)  # synchronises; outside the timed interval
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.execute(None, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        lats.append(b.job_latency(stream))
    clk = clocks.stop()
    st |= b.device_status(stream)
    ms = statistics.median(times)
    lat = np.median(np.array(lats), axis=0)

    # the same jobs one execute at a time (wavefront pass, whole-job chunks)
    pt = PathTracer(mode=abi.MODE_WAVEFRONT)
    for p, sb, (si, *_rest) in zip(params, bufs, jobs):
        n = p.dimension[0] * p.dimension[1] * p.spp
        pt.execute(dss[si].desc(p, sb), n, 1, 0, stream)
    torch.cuda.synchronize()
    seq = []
    for k in range(max(1, min(args.steps, 3))):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for p, sb, (si, *_rest) in zip(params, bufs, jobs):
            n = p.dimension[0] * p.dimension[1] * p.spp
            pt.execute(dss[si].desc(p, sb), n, 1, 0, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        seq.append(e0.elapsed_time(e1))
    st |= pt.device_status(stream)
    pt.close()
    b.close()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")
    seq_ms = statistics.median(seq)
    order = np.argsort(paths)
    line = {
        "metric": "batched Mpaths/s (32 jobs)", "value": total / (ms * 1e-3) / 1e6, "unit": "Mpaths/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{len(jobs)} jobs over {len(scene_list)} scenes of the large-render generator "
                               "(50k-10M triangles), resolutions log-uniform 256^2..1920x1080, 1-16 spp, depth 6",
                   "total_paths": total, "scene_triangles": [hs.num_triangles for hs in scene_list],
                   "jobs": [{"scene": si, "w": w, "h": h, "spp": spp} for si, w, h, spp, _, _ in jobs],
                   "l2": "inputs larger than L2", "seed": args.batch_seed},
        "tuned": {"mode": ["persistent", "wavefront"][best.mode], "block": best.blockSize,
                  "queue_chunk": best.queueChunk, "material_sort": bool(best.materialSort),
                  "graph": bool(best.useGraph)},
        "autotune": [{"mode": ["persistent", "wavefront"][c.mode], "block": c.blockSize, "chunk": c.queueChunk,
                      "sort": bool(c.materialSort), "ms": round(t, 3)} for c, t in entries],
        "job_latency_ms": {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
                           "max": float(lat.max()), "per_job": [round(float(v), 3) for v in lat],
                           "smallest_job": round(float(lat[order[0]]), 3),
                           "largest_job": round(float(lat[order[-1]]), 3)},
        "sequential_single_job": {"ms": seq_ms, "mpaths_s": total / (seq_ms * 1e-3) / 1e6},
        "gpu_launches": 1, "clocks": clk,
        "setup_seconds": {"scene_generation": gen_s, "autotune": tune_s},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="strelka", choices=["strelka", "reference"])
    ap.add_argument("--mode", default="wavefront", choices=["wavefront", "megakernel"])
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--frequency", type=int, default=89)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-step-seconds", type=float, default=4.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--split-frame", action="store_true",
                    help="N > 1: split every frame over the ranks (strong scaling) instead of independent frames")
    ap.add_argument("--no-studies", action="store_true",
                    help="skip the traversal microbenchmark and the radiance-cache study in the default run")
    ap.add_argument("--workload", default="large", choices=["large", "traversal", "nrc", "nrc-mlp", "batch", "cornell"])
    ap.add_argument("--batch-jobs", type=int, default=32)
    ap.add_argument("--batch-scenes", type=int, default=6)
    ap.add_argument("--batch-seed", type=int, default=0)
    ap.add_argument("--batch-tune-repeats", type=int, default=3)
    ap.add_argument("--tris", type=int, default=1_000_000)
    ap.add_argument("--rays", type=int, default=4_000_000)
    ap.add_argument("--ref-spp", type=int, default=16384)
    ap.add_argument("--nrc-spp", type=int, default=2)
    ap.add_argument("--nrc-warmup", type=int, default=16)
    ap.add_argument("--nrc-warmup-group", type=int, default=8)
    ap.add_argument("--nrc-max-frames", type=int, default=64)
    ap.add_argument("--nrc-plain-frames", type=int, default=10)
    ap.add_argument("--nrc-train-paths", type=int, default=16384)
    ap.add_argument("--nrc-train-steps", type=int, default=1)
    ap.add_argument("--nrc-trials", type=int, default=5)
    ap.add_argument("--nrc-log2t", type=int, default=19)
    ap.add_argument("--nrc-lr", type=float, default=1e-2)
    ap.add_argument("--nrc-diffuse-roughness", type=float, default=0.25)
    args = ap.parse_args()
    if args.workload == "traversal":
        run_traversal(args)
        return
    if args.workload == "nrc":
        run_nrc(args)
        return
    if args.workload == "nrc-mlp":
        run_nrc_mlp(args)
        return
    if args.workload == "cornell":
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        c = cornell_study(args, steps=args.steps, warmup=args.warmup)
        print(json.dumps({"metric": "Mpaths/s (Cornell 512^2, 64 accumulated iterations)", "value": c["mpaths_s"],
                          "unit": "Mpaths/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
                          "data": "synthetic", "config": {"workload": c["workload"]}, "detail": c}), flush=True)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "strelka" else args.warmup

    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    from strelka_b200 import abi, multigpu
    from strelka_b200.render import (Accumulation, DeviceScene, PathTracer, ReductionPass, Tonemap, accumulation_param,
                                     ptr, resolve, tonemap_param)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    hs = make_scene(args)
    ds = DeviceScene(hs)
    W, H, S = args.width, args.height, args.spp
    total = W * H * S
    # --split-frame (N > 1): every frame is split over the ranks, spp/N
    # samples per pixel each, and their reduced images are averaged by one
    # NCCL all-reduce per frame (strong scaling); otherwise every rank renders
    # its own frames (weak scaling)
    split = world > 1 and args.split_frame
    local_total = total // world if split else total
    mode = abi.MODE_WAVEFRONT if args.mode == "wavefront" else abi.MODE_MEGAKERNEL
    pt = PathTracer(mode=mode, chunk_paths=args.chunk, profile=True)
    sb = torch.empty(local_total * 3, dtype=torch.float32, device="cuda")
    hist = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    acc = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    cur = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    tmimg = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    rgba8 = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
    tp = tonemap_param(W, H, 1)
    stream = torch.cuda.current_stream()

    def frame_param(it):
        if split:
            return multigpu.split_frame_param(hs.param(frameNumber=it, iteration=it), rank, world)
        return hs.param(frameNumber=multigpu.frame_number(rank, it), iteration=it)

    def frame(it):
        # PtRender::drawFrame (src/render/ptrender.cpp:735-862) for one view
        p = frame_param(it)
        pt.execute(ds.desc(p, sb), local_total, 1, it, stream)
        ap_ = accumulation_param(W, H, it)
        if split:
            ReductionPass().execute(abi.ReductionDesc(p, ptr(sb), ptr(cur)), W * H, 1, it, stream)
            multigpu.combine_split_frame(cur, dist)
            Accumulation().execute(abi.AccumulationDesc(ap_, ptr(cur), ptr(hist), ptr(acc)), W, H, it, stream)
            Tonemap().execute(abi.TonemapDesc(tp, ptr(acc), ptr(tmimg)), W, H, it, stream)
        else:
            resolve(p, sb, tp, ap_ if it > 0 else None, hist if it > 0 else None, acc, None, rgba8, stream)
        return p

    for it in range(args.warmup):
        frame(it)
    torch.cuda.synchronize()
    st = pt.device_status()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")

    # ---- device-timed region: inputs resident in HBM -------------------------
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    pt.kernel_times(stream)  # reset the per-launch records
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ext_ms = 0.0
    launches = 0
    for k in range(args.steps):
        frame(args.warmup + k)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    el_ms = e0.elapsed_time(e1)
    # per-kernel CUDA-event times summed over every launch of the timed region
    times = pt.kernel_times(stream)
    el_ms = multigpu.max_over_ranks(el_ms, dist, device="cuda")

    frame_paths = total if split else world * total  # paths of the whole job per step
    value = frame_paths * args.steps / (el_ms * 1e-3) / 1e6

    # ---- extend-kernel roofline: replay the timed frames with counters -------
    ext_ms = times["extend"][0]
    ext_launches = times["extend"][1]
    launches = sum(c for _, c in times.values()) + args.steps  # + one resolve per frame
    pt_count = PathTracer(mode=mode, chunk_paths=args.chunk, count=True)
    for k in range(args.steps):
        pt_count.execute(ds.desc(frame_param(args.warmup + k), sb), local_total, 1, 0, stream)
    cnt = pt_count.counters(stream)
    pt_count.close()
    # algorithmic bytes of the closest-hit traversal: 112 B per 4-wide node
    # processed, 48 B per triangle test, 32 B ray in, 20 B hit out
    bytes_alg = WIDE_NODE_BYTES * cnt["extend_inner"] + 48 * cnt["extend_leaf"] + 52 * cnt["extend_rays"]
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = bytes_alg / (ext_ms * 1e-3) / 1e9 if ext_ms > 0 else None
    sh_ms, sh_launches = times["shadow"]
    sh_bytes = WIDE_NODE_BYTES * cnt["shadow_inner"] + 48 * cnt["shadow_leaf"] + 64 * cnt["shadow_rays"]
    sh_overlapped = sh_bytes / (sh_ms * 1e-3) / 1e9 if sh_ms > 0 else None
    # the shadow kernel alone: the timed frames again (same samples, so the
    # same visit counts) with each bounce's shadow queries on the frame's
    # stream after its shading, every launch timed by CUDA events
    pt_serial = PathTracer(mode=mode, chunk_paths=args.chunk, profile=True, serial_shadow=True)
    pt_serial.execute(ds.desc(frame_param(args.warmup), sb), local_total, 1, 0, stream)  # scene tables, warm-up
    torch.cuda.synchronize()
    pt_serial.kernel_times(stream)
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for k in range(args.steps):
        pt_serial.execute(ds.desc(frame_param(args.warmup + k), sb), local_total, 1, 0, stream)
    s1.record(stream)
    torch.cuda.synchronize()
    serial_frame_ms = s0.elapsed_time(s1) / args.steps
    sh_alone_ms, sh_alone_launches = pt_serial.kernel_times(stream)["shadow"]
    st = pt_serial.device_status()
    pt_serial.close()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")
    sh_achieved = sh_bytes / (sh_alone_ms * 1e-3) / 1e9 if sh_alone_ms > 0 else None

    # ---- end to end through the C ABI: host param in, tonemapped RGBA8 out ---
    out_img = tmimg if split else rgba8
    host_img = torch.empty(out_img.numel(), dtype=out_img.dtype, pin_memory=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for k in range(args.steps):
        frame(args.warmup + args.steps + k)
        host_img.copy_(out_img, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = multigpu.max_over_ranks(f0.elapsed_time(f1), dist, device="cuda")
    e2e = frame_paths * args.steps / (e2e_ms * 1e-3) / 1e6
    img = host_img.numpy()
    if not (img[3::4] == (1.0 if split else 255)).all():
        raise RuntimeError("resolve produced no image")
    st = pt.device_status()
    if st != 0:
        raise RuntimeError(f"device status {st:#x}")

    # ---- parity of the first timed frame against the oracle -------------------
    parity = None
    if rank == 0 and world == 1 and not args.no_parity:
        p_first = hs.param(frameNumber=multigpu.frame_number(rank, args.warmup), iteration=args.warmup)
        pt.execute(ds.desc(p_first, sb), total, 1, args.warmup, stream)
        torch.cuda.synchronize()
        parity = frame_parity(hs, p_first, sb)
        st = pt.device_status()
        if st != 0:
            raise RuntimeError(f"device status {st:#x}")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, n, threads, el = cpu_baseline(hs, args, budget_s=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} paths of the frame ({n / total * 100:.3f}%), 64 evenly spaced slices of the sample "
                         f"indices, {el:.1f} s, oracle C restatement -O3 -ffp-contract=fast, OpenMP"}

    # ---- the rest of the metric, one GPU: the traversal microbenchmark and
    # the radiance-cache time-to-equal-relMSE study ---------------------------
    trav = nrc_res = cornell = None
    if rank == 0 and world == 1 and not args.no_studies:
        trav = traversal_study(args, steps=10, warmup=3)
        cornell = cornell_study(args)
        nrc_res = nrc_study(args, hs, ds)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cfg = workload_config(args)
    cfg["triangles"] = hs.num_triangles
    param_bytes = 336 + 416 + 16
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el_ms / args.steps, "higher_is_better": True, "scaling": "strong" if split else "weak",
        "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded procedural scene, see config.workload)", "config": cfg,
        "parallelism": (f"one frame split over {world} GPUs (spp/{world} each, NCCL all-reduce of the image per frame)"
                        if split else f"replicas x{world} (independent frames per GPU)" if world > 1 else "single GPU"),
        "parity": parity,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": EXTEND_DRAM_BYTES_PER_RAY * cnt["extend_rays"] / max(ext_launches, 1)
                     if args.width == 1920 and args.height == 1080 and args.spp == 16 else None,
                     "traffic_source": "ncu DRAM bytes per query of a 960x540x4 frame's extend launches x queries per "
                                       "launch (an upper bound: the per-query figure falls as the frame grows)",
                     "bytes_alg_per_launch": bytes_alg / max(ext_launches, 1),
                     "kernel": "extend (closest-hit traversal)", "peak_source": peak_src,
                     "bytes_alg_timed_region": bytes_alg, "kernel_ms_timed_region": ext_ms,
                     "kernel_launches_timed_region": ext_launches, "visits": cnt},
        "roofline_shadow": {"bound": "hbm", "kernel": "shadow (any-hit traversal)",
                            "achieved": sh_achieved, "peak": peak, "unit": "GB/s",
                            "frac": (sh_achieved / peak) if sh_achieved else None,
                            "bytes_alg_per_launch": sh_bytes / max(sh_launches, 1),
                            "kernel_ms_alone": sh_alone_ms, "kernel_launches_alone": sh_alone_launches,
                            "frame_ms_serial": serial_frame_ms,
                            "frac_overlapped": (sh_overlapped / peak) if sh_overlapped else None,
                            "kernel_ms_timed_region": sh_ms, "kernel_launches_timed_region": sh_launches,
                            "note": "112 B per 4-wide node + 48 B per triangle test + 64 B request per query. frac: "
                                    "the timed frames replayed with each bounce's shadow launch alone on the "
                                    "frame's stream (frame_ms_serial per frame), CUDA events per launch; "
                                    "frac_overlapped: the timed region's event intervals, where the kernel runs on "
                                    "a second stream beside the next bounce's extend and shares its SMs"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": param_bytes,
                "d2h_bytes_per_step": out_img.numel() * out_img.element_size()},
        "traversal": trav,
        "cornell": cornell,
        "nrc": nrc_res,
        "gpu_launches": launches,
        "clocks": clk,
        "kernel_ms_per_frame": {k: v[0] / args.steps for k, v in times.items() if v[1]},
        "kernel_ms_note": "event intervals per kernel class; shadow(k) runs on a second stream beside extend(k+1), "
                          "so the shadow and sort intervals include time shared with the other stream and the "
                          "classes sum to more than ms_per_step",
    }
    print(json.dumps(line), flush=True)
    if parity is not None and not parity["relmse"] <= 1e-4:
        raise SystemExit(f"parity failed: relMSE {parity['relmse']} against the oracle exceeds 1e-4")


if __name__ == "__main__":
    main()
