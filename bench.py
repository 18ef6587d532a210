#!/usr/bin/env python
"""Benchmark of the B200 SIFT-and-stitching hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

Prints ONE JSON line on rank 0.  Workloads (synthetic, seeded inputs that
stand in for the reference's datasets; see pysift_b200/synthetic.py):

  stitch_pair_1280x960  GPUPyStitch().stitch(img1, img2) on a seeded synthetic
                    pair of 1280x960 BGR views (ratio 0.75, 2048 hypotheses,
                    4 px, the reference's gain + DP seam + 6-level multiband
                    composition) -- the default
  detect_1280x960   detectAndCompute on one 1280x960 grayscale scene
  detect_640x480    detectAndCompute on one 640x480 scene
  match_u8_8192     exact ratio-test matching of two 8192 x 128 uint8-valued
                    descriptor sets (bf16 tcgen05 GEMM, exact against int64)
  match_u8_8192_fp8 the same through the split-nibble e4m3 tcgen05 GEMM
  batch96_detect    PySIFT.detect_batch of 96 grayscale images of uneven sizes
                    (480x360 .. 4000x3000, aspect 4:3, 3:2, 16:9) over 8 streams,
                    next to the plain per-image detectAndCompute loop and the
                    same batch replayed as one CUDA graph
  batch32_stitch    GPUPyStitch.stitch_batch of 32 uneven pairs (1280x960 ..
                    3000x2000, 4096 hypotheses each) next to sequential stitch()
  grad_16x1024x768  forward + backward of the differentiable descriptors (2000
                    fixed keypoints per image) and of warp + feather blend on
                    16 float32 1024x768 images

A step is one pass of the hot path over one input.  `value` is measured
with CUDA events on the launching stream, inputs resident in HBM, L2
flushed (256 MiB write) before every step outside the timed interval;
`e2e` is the same metric through the public API with host buffers (pinned
host->device copy of the input and device->host read of all outputs inside
every timed step).  Multi-GPU runs are independent replicas (one process per
GPU, each with its own input; scaling "weak"), timed as the max over ranks.
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "stitch_pair_1280x960": dict(kind="stitch", H=960, W=1280, seed=0, ransac_iters=2048, inlier_thresh=4.0),
    "detect_1280x960": dict(kind="detect", H=960, W=1280, seed=0),
    "detect_640x480": dict(kind="detect", H=480, W=640, seed=0),
    "match_u8_8192": dict(kind="match", N=8192, M=8192, D=128, seed=0),
    "match_u8_8192_fp8": dict(kind="match", N=8192, M=8192, D=128, seed=0, variant="split_fp8"),
    "batch96_detect": dict(kind="batch_detect", n=96, seed=0, streams=8),
    "batch32_stitch": dict(kind="batch_stitch", n=32, seed=0, streams=8, ransac_iters=4096, inlier_thresh=4.0),
    "grad_16x1024x768": dict(kind="grad", n=16, H=768, W=1024, kps=2000, seed=0),
}
DEFAULT_WORKLOAD = "stitch_pair_1280x960"
METRIC = "SIFT Mpix/s + match-pairs/s on 1 B200: batched+BF16 vs plain, bit-exact"
FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload)


class ClockSampler:
    """Samples SM clock and clock-event reasons with NVML during the timed region."""
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self._h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                self.reasons |= nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
            except Exception:
                pass
            time.sleep(0.025)

    def __enter__(self):
        if self._nv is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if self._nv is None or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        names = [n for b, n in self.REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples)}


def pyramid_alg_bytes(H, W, sift):
    """Algorithmic bytes of pyramid + DoG + extrema for one image:
    H*W (u8 in) + 4*P0 (upsampled base write) + 80*sum(P_o)."""
    doubled = sift.double_image and H * W < sift._cfg.double_px_cap
    h, w = (2 * H, 2 * W) if doubled else (H, W)
    P = []
    for _ in range(sift.n_octaves):
        P.append(h * w)
        h, w = (h + 1) // 2, (w + 1) // 2
    return H * W + 4 * P[0] + 80 * sum(P)


def cpu_detect_baseline(img, budget_s=15.0):
    """The oracle (a CPU port of the reference's path, OpenMP over the host
    cores) on the same image, repeated until ~budget_s of work."""
    from oracle import oracle
    orc = oracle.OracleSIFT()
    orc.detect_and_compute(img)  # warm-up (builds tables)
    times = []
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        orc.detect_and_compute(img)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s or len(times) >= 50:
            break
    med = float(np.median(times))
    return med, len(times)


def opencv_detect_baseline(img, threads=None, runs=5):
    """OpenCV's SIFT on the host cores, the reference's own CPU comparison
    (examples/quick_test.py:71-80): cv2.SIFT_create() with its defaults,
    detectAndCompute(img, None), median of `runs` after one warm-up call."""
    try:
        import cv2
    except Exception:
        return None
    cv2.setNumThreads(threads or os.cpu_count() or 1)
    s = cv2.SIFT_create()
    s.detectAndCompute(img, None)
    t = []
    for _ in range(runs):
        t0 = time.perf_counter()
        kps, _ = s.detectAndCompute(img, None)
        t.append(time.perf_counter() - t0)
    cv2.setNumThreads(os.cpu_count() or 1)
    return float(np.median(t)), len(kps)


def opencv_stitch_once(img1, img2, ratio=0.75, thresh=4.0):
    """The two-image stitch with OpenCV on the host: SIFT on both gray views,
    BFMatcher(NORM_L2).knnMatch(k=2) with the ratio test,
    findHomography(USAC_MAGSAC, 4 px), warpPerspective of view 1 onto the
    canvas that holds both views, and a linear feather (each view weighted by
    its distance to its own border where both cover a pixel)."""
    import cv2
    sift = cv2.SIFT_create()
    k1, d1 = sift.detectAndCompute(cv2.cvtColor(img1, cv2.COLOR_BGR2GRAY), None)
    k2, d2 = sift.detectAndCompute(cv2.cvtColor(img2, cv2.COLOR_BGR2GRAY), None)
    knn = cv2.BFMatcher(cv2.NORM_L2).knnMatch(d1, d2, k=2)
    good = [p[0] for p in knn if len(p) == 2 and p[0].distance < ratio * p[1].distance]
    src = np.float32([k1[m.queryIdx].pt for m in good]).reshape(-1, 1, 2)
    dst = np.float32([k2[m.trainIdx].pt for m in good]).reshape(-1, 1, 2)
    H, inl = cv2.findHomography(src, dst, cv2.USAC_MAGSAC, thresh)
    h1, w1 = img1.shape[:2]
    h2, w2 = img2.shape[:2]
    c = cv2.perspectiveTransform(np.float32([[0, 0], [w1, 0], [w1, h1], [0, h1]]).reshape(-1, 1, 2), H).reshape(-1, 2)
    xs = np.concatenate([c[:, 0], [0, w2]])
    ys = np.concatenate([c[:, 1], [0, h2]])
    ox, oy = max(0.0, -xs.min()), max(0.0, -ys.min())
    cw, ch = int(np.ceil(xs.max() + ox)) + 1, int(np.ceil(ys.max() + oy)) + 1
    T = np.array([[1, 0, ox], [0, 1, oy], [0, 0, 1]], np.float64)
    warped = cv2.warpPerspective(img1, T @ H, (cw, ch))
    wmask = cv2.warpPerspective(np.full((h1, w1), 255, np.uint8), T @ H, (cw, ch), flags=cv2.INTER_NEAREST)
    canvas2 = np.zeros((ch, cw, 3), np.uint8)
    m2 = np.zeros((ch, cw), np.uint8)
    iox, ioy = int(round(ox)), int(round(oy))
    ye, xe = min(ioy + h2, ch), min(iox + w2, cw)
    canvas2[ioy:ye, iox:xe] = img2[:ye - ioy, :xe - iox]
    m2[ioy:ye, iox:xe] = 255
    f1 = cv2.distanceTransform(wmask, cv2.DIST_L2, 3)
    f2 = cv2.distanceTransform(m2, cv2.DIST_L2, 3)
    wsum = f1 + f2
    wsum[wsum == 0] = 1.0
    pano = (warped * (f1 / wsum)[..., None] + canvas2 * (f2 / wsum)[..., None]).clip(0, 255).astype(np.uint8)
    return pano, len(good), int(inl.sum()) if inl is not None else 0


def opencv_stitch_baseline(img1, img2, threads, runs=3):
    """Median time of opencv_stitch_once over `runs` after one warm-up, with
    OpenCV limited to `threads` threads."""
    try:
        import cv2
    except Exception:
        return None
    cv2.setNumThreads(threads)
    opencv_stitch_once(img1, img2)
    t = []
    for _ in range(runs):
        t0 = time.perf_counter()
        _, n_good, n_inl = opencv_stitch_once(img1, img2)
        t.append(time.perf_counter() - t0)
    cv2.setNumThreads(os.cpu_count() or 1)
    return float(np.median(t)), n_good, n_inl


def opencv_baselines(kind, *imgs, scale=1.0):
    """OpenCV at one thread and at every host thread: {threads_1, threads_all}
    in units per second (scale / median seconds)."""
    n = os.cpu_count() or 1
    out = {"cores": n, "kind": "opencv " + __import__("cv2").__version__}
    for key, th in (("threads_1", 1), ("threads_all", n)):
        r = opencv_detect_baseline(imgs[0], threads=th) if kind == "detect" else opencv_stitch_baseline(*imgs, th)
        out[key] = None if r is None else scale / r[0]
        if r is not None and kind == "stitch":
            out["matches_inliers"] = [r[1], r[2]]
    return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def all_ranks_max(t, world):
    """Replace `t` in place by its element-wise maximum over all ranks, so a
    step time is the slowest rank's; a no-op on one process."""
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t


REF_BUDGET_S = 90.0  # wall-time budget of the reference arm's timed steps


class RefSchedule:
    """Step indices 0 .. warmup + steps - 1 of the reference arm, ending
    early once the timed steps (index >= warmup) have used REF_BUDGET_S,
    after at least one timed step: a CPU stitch takes seconds, so the
    requested step count is a bound, not a promise, and the line reports
    the steps it timed."""

    def __init__(self, warmup, steps):
        self.warmup, self.steps, self.k, self.t0 = warmup, steps, 0, None

    def __iter__(self):
        return self

    def __next__(self):
        if self.k == self.warmup:
            self.t0 = time.perf_counter()
        if self.k >= self.warmup + self.steps or (
                self.k > self.warmup and time.perf_counter() - self.t0 > REF_BUDGET_S):
            raise StopIteration
        self.k += 1
        return self.k - 1


def run_reference(args, wl, world, rank):
    """--impl reference: the reference's path as the CPU oracle port, rank 0
    only; three warm-up steps and at most REF_BUDGET_S of timed steps."""
    if rank != 0:
        return 0
    args.warmup = min(args.warmup, 3)
    from pysift_b200 import synthetic
    if wl["kind"] == "stitch":
        return run_reference_stitch(args, wl)
    if wl["kind"] == "match":
        return run_reference_match(args, wl)
    if wl["kind"] == "batch_detect":
        return run_reference_batch(args, wl)
    if wl["kind"] == "batch_stitch":
        return run_reference_pairs(args, wl)
    if wl["kind"] == "grad":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no differentiable path"}))
        return 0
    img = synthetic.scene(wl["H"], wl["W"], seed=wl["seed"])
    times = []
    from oracle import oracle
    orc = oracle.OracleSIFT()
    for k in RefSchedule(args.warmup, args.steps):
        t0 = time.perf_counter()
        orc.detect_and_compute(img)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    sec = float(np.mean(times))
    mpix = wl["H"] * wl["W"] / 1e6
    value = mpix / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "H": wl["H"], "W": wl["W"], "seed": wl["seed"]},
        "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"one {wl['W']}x{wl['H']} image per step, full detectAndCompute"},
        "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measured_tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured (cuBLAS bf16 burst)"
    return 1590.0, "fallback"


def run_match(args, wl, world, rank, local):
    import torch
    import torch.distributed as dist
    from pysift_b200 import _lib, match, synthetic

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    N, M, D = wl["N"], wl["M"], wl["D"]
    a, b = synthetic.descriptor_sets(N, M, seed=wl["seed"] + rank, D=D)
    ga, gb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    split = wl.get("variant") == "split_fp8"
    mfn = match.match_u8_split_fp8 if split else match.match_u8_exact
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = _lib.load()
    for _ in range(args.warmup):
        out = mfn(ga, gb)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = lib.pysift_launch_count()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0.record(stream)
            out = mfn(ga, gb)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    launches = lib.pysift_launch_count() - launches0
    n_pairs = int(out["count"].item())
    t = torch.tensor([float(np.sum(step_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(t, world)
    total_ms = float(t.item())
    # end to end: pinned host sets -> device, match, pairs and count back to the host
    ha = torch.from_numpy(a).pin_memory()
    hb = torch.from_numpy(b).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        da, db = ha.to(dev, non_blocking=True), hb.to(dev, non_blocking=True)
        o = mfn(da, db)
        cnt = int(o["count"].item())
        pairs_host = o["pairs"][:cnt].cpu()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_t = torch.tensor([float(np.sum(e2e_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(e2e_t, world)
    if rank != 0:
        return None
    step_s = total_ms / args.steps / 1e3
    flops = 2.0 * N * M * D
    peak, peak_kind = measured_tensor_peak()
    # the exact path runs unsigned 8-bit MMAs (kind::i8), the split path e4m3
    # (kind::f8f6f4): both at twice the dense bf16 rate
    peak, peak_kind = 2.0 * peak, "2 x " + peak_kind + (" (dense fp8 rate)" if split else " (dense int8 rate)")
    achieved = flops / step_s / 1e12
    if args.no_cpu_baseline:
        cpu_s, cpu_n = float("nan"), 0
    else:
        from oracle import match_oracle as mo
        times = []
        t_start = time.perf_counter()
        while time.perf_counter() - t_start < 15.0 and len(times) < 5:
            t0 = time.perf_counter()
            mo.match_u8_exact(a, b)
            times.append(time.perf_counter() - t0)
        cpu_s, cpu_n = float(np.median(times)), len(times)
    line = {
        "metric": METRIC, "value": world / step_s, "unit": "match-pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp8-e4m3" if split else "u8", "data": "synthetic",
        "config": {"workload": args.workload, "N": N, "M": M, "D": D, "seed": wl["seed"], "ratio": 0.75,
                   "mutual_matches": n_pairs, "l2": "flushed (256 MiB write) before every step",
                   "parallelism": f"replicas{world}"},
        "roofline": {"bound": "tensor", "kernel": "whole match call (k_row_norms_u8 x2, "
                     + ("k_split_nibbles_u8 x2, " if split else "k_tile_rows x2, ") + "k_match_rows x2, k_match_merge_u8 x2, "
                     "k_match_mutual); flops 2*N*M*D counted once" + (" (the e4m3 GEMM does 4x that)" if split else ""),
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_flops_per_step": flops,
                     "traffic": committed_traffic(args.workload)},
        "cpu_baseline": {"value": 1.0 / cpu_s if cpu_s == cpu_s else None, "unit": "match-pairs/s",
                         "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{cpu_n} full {N}x{M} exact matches by the oracle (numpy, BLAS float64)"},
        "e2e": {"value": world * args.steps / (float(e2e_t.item()) / 1e3), "unit": "match-pairs/s",
                "h2d_bytes_per_step": int(a.nbytes + b.nbytes), "d2h_bytes_per_step": 4 + 8 * n_pairs},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return line


def run_reference_pairs(args, wl):
    """The oracle stitch of the batch's smallest pair, per step."""
    from oracle import stitch_oracle as so
    from pysift_b200 import synthetic
    sizes = synthetic.pair_sizes(wl["n"], wl["seed"])
    i = int(np.argmin([h * w for h, w in sizes]))
    a, b, _ = synthetic.stitch_pair_fast(sizes[i][0], sizes[i][1], wl["seed"] * 1000 + i)
    times = []
    for k in RefSchedule(args.warmup, args.steps):
        orc = so.OracleStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"])
        t0 = time.perf_counter()
        orc.stitch(a, b)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = 1.0 / float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "pair": list(sizes[i]), "seed": wl["seed"]},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "the batch's smallest pair per step (oracle port, OpenMP)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batch(args, wl):
    """The oracle on a bounded sample of the batch (its smallest images)."""
    from oracle import oracle
    from pysift_b200 import synthetic
    imgs = sorted(synthetic.batch_images(wl["n"], seed=wl["seed"]), key=lambda im: im.size)[:4]
    orc = oracle.OracleSIFT()
    times = []
    for i in RefSchedule(args.warmup, args.steps):
        t0 = time.perf_counter()
        for im in imgs:
            orc.detect_and_compute(im)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = sum(im.size for im in imgs) / 1e6 / float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "images": len(imgs), "seed": wl["seed"]},
        "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "the 4 smallest images of the batch per step (oracle, OpenMP)"},
        "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_match(args, wl):
    from oracle import match_oracle as mo
    from pysift_b200 import synthetic
    a, b = synthetic.descriptor_sets(wl["N"], wl["M"], seed=wl["seed"], D=wl["D"])
    times = []
    for i in RefSchedule(args.warmup, args.steps):
        t0 = time.perf_counter()
        mo.match_u8_exact(a, b)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    sec = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": 1.0 / sec, "unit": "match-pairs/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": args.workload, "N": wl["N"], "M": wl["M"], "D": wl["D"], "seed": wl["seed"]},
        "cpu_baseline": {"value": 1.0 / sec, "unit": "match-pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "one full exact match per step (oracle, numpy + BLAS)"},
        "e2e": {"value": 1.0 / sec, "unit": "match-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch_detect(args, wl, world, rank, local):
    import torch
    import torch.distributed as dist
    from pysift_b200 import PySIFT, _lib, synthetic

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    imgs = synthetic.batch_images(wl["n"], seed=wl["seed"])
    mpix_all = sum(im.size for im in imgs) / 1e6
    if world > 1:
        # the one batch dealt over the ranks by longest-processing-time greedy
        from pysift_b200 import shard
        imgs = [imgs[i] for i in shard.lpt_assign([shard.image_cost(im.shape) for im in imgs], world)[rank]]
    mpix = sum(im.size for im in imgs) / 1e6
    sift = PySIFT(device=dev)
    g = [torch.from_numpy(im).to(dev) for im in imgs]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = _lib.load()
    ns = wl["streams"]
    for _ in range(args.warmup):
        sift.detect_batch(g, n_streams=ns)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, steps):
        ms = []
        for _ in range(steps):
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = lib.pysift_launch_count()
    with ClockSampler(local) as clk:
        step_ms = timed(lambda: sift.detect_batch(g, n_streams=ns), args.steps)
    launches = lib.pysift_launch_count() - launches0
    t = torch.tensor([float(np.sum(step_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(t, world)
    total_ms = float(t.item())
    # the same images, the plain way: one detectAndCompute call per image
    # (each comparison leg runs once untimed first, as the batched one did:
    # first calls per image size capture their CUDA graphs)
    plain_steps = max(1, min(3, args.steps))
    plain_fn = lambda: [sift.detectAndCompute(x, gpu_output=True) for x in g]
    one_fn = lambda: sift.detect_batch(g, n_streams=1)
    plain_fn()
    one_fn()
    torch.cuda.synchronize(dev)
    plain_ms = timed(plain_fn, plain_steps)
    one_ms = timed(one_fn, plain_steps)
    # the same batch replayed as one CUDA graph (captured on the first call)
    for _ in range(2):
        sift.detect_batch(g, n_streams=ns, graph=True)
    torch.cuda.synchronize(dev)
    sift.detect_batch(g, n_streams=ns, graph=True)  # capture (untimed)
    torch.cuda.synchronize(dev)
    graph_ms = timed(lambda: sift.detect_batch(g, n_streams=ns, graph=True), args.steps)
    # end to end: host images in, host arrays out
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = sift.detect_batch(imgs, n_streams=ns, gpu_output=False)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_t = torch.tensor([float(np.sum(e2e_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(e2e_t, world)
    if rank != 0:
        return None
    n_kp = int(sum(r[0].shape[0] for r in res))
    out_bytes = int(sum(r[0].nbytes + r[1].nbytes for r in res))
    step_s = total_ms / args.steps / 1e3
    peak, peak_kind = measured_peaks()
    alg = sum(pyramid_alg_bytes(im.shape[0], im.shape[1], sift) for im in imgs)
    achieved = alg / step_s / 1e9
    if args.no_cpu_baseline:
        cpu_v, cpu_n = None, 0
    else:
        from oracle import oracle
        orc = oracle.OracleSIFT()
        small = sorted(imgs, key=lambda im: im.size)[:4]
        t0 = time.perf_counter()
        for im in small:
            orc.detect_and_compute(im)
        cpu_v = sum(im.size for im in small) / 1e6 / (time.perf_counter() - t0)
        cpu_n = len(small)
    line = {
        "metric": METRIC, "value": mpix_all / step_s, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "images": wl["n"], "seed": wl["seed"], "mpix_per_batch": mpix_all,
                   "streams": ns, "keypoints": n_kp, "sizes": "480x360 .. 4000x3000, aspect 4:3 / 3:2 / 16:9",
                   "l2": "flushed (256 MiB write) before every step",
                   "parallelism": f"lpt{world} (the batch dealt over the ranks)" if world > 1 else "replicas1"},
        "plain_mpix_per_s": mpix / (float(np.mean(plain_ms)) / 1e3),
        "one_stream_mpix_per_s": mpix / (float(np.mean(one_ms)) / 1e3),
        "graph_mpix_per_s": mpix / (float(np.mean(graph_ms)) / 1e3),
        "roofline": {"bound": "hbm", "kernel": "whole batched detection: pyramid-region algorithmic bytes of all "
                     "images over the whole batch time (a lower bound for the pyramid kernels)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_bytes_per_launch": alg, "traffic": None},
        "cpu_baseline": {"value": cpu_v, "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"the {cpu_n} smallest images of the batch through the oracle (OpenMP)"},
        "e2e": {"value": mpix_all / (float(e2e_t.item()) / args.steps / 1e3), "unit": "Mpix/s",
                "h2d_bytes_per_step": int(sum(im.nbytes for im in imgs)), "d2h_bytes_per_step": out_bytes},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return line


def _gen_pairs(n, seed):
    """Seeded synthetic pairs, generated in a spawned process pool (before any
    CUDA work in this process)."""
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    from pysift_b200 import synthetic
    sizes = synthetic.pair_sizes(n, seed)
    with ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        futs = [ex.submit(synthetic.stitch_pair_fast, h, w, seed * 1000 + i) for i, (h, w) in enumerate(sizes)]
        return [f.result()[:2] for f in futs]


def batch_pairs(args, wl, world, rank):
    """The pair batch (generated in a spawned process pool); with several
    ranks, this rank's share of the one batch dealt by longest-processing-time
    greedy.  Records the whole batch's pair count and Mpix in args."""
    pairs = _gen_pairs(wl["n"], wl["seed"])
    args.batch_pairs_total = len(pairs)
    args.batch_mpix_total = sum(a.shape[0] * a.shape[1] + b.shape[0] * b.shape[1] for a, b in pairs) / 1e6
    if world > 1:
        from pysift_b200 import shard
        share = shard.lpt_assign([shard.pair_cost(a.shape, b.shape) for a, b in pairs], world)[rank]
        pairs = [pairs[i] for i in share]
    return pairs


def run_batch_stitch(args, wl, world, rank, local, pairs):
    import torch
    import torch.distributed as dist
    from pysift_b200 import _lib
    from pysift_b200.stitch import GPUPyStitch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mpix = sum(a.shape[0] * a.shape[1] + b.shape[0] * b.shape[1] for a, b in pairs) / 1e6
    st = GPUPyStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"], save_output=False,
                     verbose=False, device=dev)
    g = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b in pairs]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = _lib.load()
    ns = wl["streams"]
    for _ in range(args.warmup):
        st.stitch_batch(g, n_streams=ns)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, steps):
        ms = []
        for _ in range(steps):
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = lib.pysift_launch_count()
    with ClockSampler(local) as clk:
        step_ms = timed(lambda: st.stitch_batch(g, n_streams=ns), args.steps)
    launches = lib.pysift_launch_count() - launches0
    t = torch.tensor([float(np.sum(step_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(t, world)
    total_ms = float(t.item())
    metrics = st.last_batch_metrics
    plain_fn = lambda: [st.stitch(a, b) for a, b in g]
    plain_fn()  # untimed first pass: first calls per image size capture their CUDA graphs
    torch.cuda.synchronize(dev)
    plain_ms = timed(plain_fn, max(1, min(2, args.steps)))
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        panos = st.stitch_batch(pairs, n_streams=ns)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_t = torch.tensor([float(np.sum(e2e_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(e2e_t, world)
    if rank != 0:
        return None
    P = len(pairs)
    P_all = getattr(args, "batch_pairs_total", P)
    step_s = total_ms / args.steps / 1e3
    peak, peak_kind = measured_peaks()
    sift = st._detector
    alg = sum(pyramid_alg_bytes(a.shape[0], a.shape[1], sift) + pyramid_alg_bytes(b.shape[0], b.shape[1], sift)
              for a, b in pairs)
    achieved = alg / step_s / 1e9
    if args.no_cpu_baseline:
        cpu_v, cpu_n = None, 0
    else:
        from oracle import stitch_oracle as so
        small = min(pairs, key=lambda pr: pr[0].size)
        orc = so.OracleStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"])
        t0 = time.perf_counter()
        orc.stitch(small[0], small[1])
        cpu_v, cpu_n = 1.0 / (time.perf_counter() - t0), 1
    line = {
        "metric": METRIC, "value": P_all / step_s, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "pairs": P, "seed": wl["seed"], "mpix_per_batch": mpix,
                   "streams": ns, "ransac_iters": wl["ransac_iters"], "inlier_thresh": wl["inlier_thresh"],
                   "sizes": "1280x960 .. 3000x2000", "matches": [m["matches"] for m in metrics],
                   "inliers": [m["inliers"] for m in metrics],
                   "l2": "flushed (256 MiB write) before every step",
                   "parallelism": f"lpt{world} (the batch dealt over the ranks)" if world > 1 else "replicas1"},
        "mpix_per_s": getattr(args, "batch_mpix_total", mpix) / step_s,
        "plain_pairs_per_s": P / (float(np.mean(plain_ms)) / 1e3),
        "roofline": {"bound": "hbm", "kernel": "whole batched stitch: pyramid-region algorithmic bytes of all "
                     "views over the whole batch time (a lower bound for the pyramid kernels)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_bytes_per_launch": alg, "traffic": None},
        "cpu_baseline": {"value": cpu_v, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{cpu_n} stitch of the smallest pair by the oracle port (OpenMP)"},
        "e2e": {"value": P_all / (float(e2e_t.item()) / args.steps / 1e3), "unit": "pairs/s",
                "h2d_bytes_per_step": int(sum(a.nbytes + b.nbytes for a, b in pairs)),
                "d2h_bytes_per_step": int(sum(p.nbytes for p in panos))},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return line


def run_grad(args, wl, world, rank, local):
    import cv2
    import torch
    from pysift_b200 import PySIFT, _lib, grad, synthetic

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    H, W, n = wl["H"], wl["W"], wl["n"]
    rng = np.random.default_rng(wl["seed"] + rank)
    sift = PySIFT(double_image=False, device=dev)
    sift._cfg.output_limit = wl["kps"]
    items = []
    for i in range(n):
        u8 = synthetic.scene(H, W, seed=wl["seed"] * 100 + i)
        Hm = synthetic.random_homography(rng, W, H)
        Hm[0, 2] *= 0.3  # a mild view change, as in the stitch pair
        warped = cv2.warpPerspective(u8, Hm, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
        kp, _ = sift.detectAndCompute(u8, gpu_output=True)
        octv = sift._buffers(H, W).octv[:kp.shape[0]]
        table = grad.keypoints_for_grad(sift, kp, octv)
        x = torch.from_numpy(u8.astype(np.float32) / 255.0).to(dev)
        x2 = torch.from_numpy(warped.astype(np.float32) / 255.0).to(dev)
        with torch.no_grad():
            target = grad.descriptors(x2, table, sift)
        geo = grad.canvas_geometry((H, W), (H, W), Hm)
        h8 = torch.from_numpy(Hm.ravel()[:8].copy()).to(dev)
        ptarget = torch.zeros((geo[1], geo[0], 1), dtype=torch.float32, device=dev)
        items.append((x, x2, table, target, geo, h8, ptarget))
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]

    def step():
        df, db, wf, wb = 0.0, 0.0, 0.0, 0.0
        for x, x2, table, target, geo, h8, ptarget in items:
            xi = x.clone().requires_grad_(True)
            ev[0].record(stream)
            d = grad.descriptors(xi, table, sift)
            loss = ((d - target) ** 2).sum()
            ev[1].record(stream)
            loss.backward()
            ev[2].record(stream)
            a = x.unsqueeze(-1).clone().requires_grad_(True)
            bimg = x2.unsqueeze(-1).clone().requires_grad_(True)
            hh = h8.clone().requires_grad_(True)
            out = grad.warp_blend(a, bimg, hh, geo)
            pl = ((out - ptarget) ** 2).sum()
            ev[3].record(stream)
            pl.backward()
            ev[4].record(stream)
            ev[4].synchronize()
            df += ev[0].elapsed_time(ev[1])
            db += ev[1].elapsed_time(ev[2])
            wf += ev[2].elapsed_time(ev[3])
            wb += ev[3].elapsed_time(ev[4])
        return df, db, wf, wb

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    lib = _lib.load()
    launches0 = lib.pysift_launch_count()
    tot = np.zeros(4)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            tot += np.array(step())
    launches = lib.pysift_launch_count() - launches0
    if rank != 0:
        return None
    df, db, wf, wb = (tot / args.steps).tolist()
    step_ms = df + db + wf + wb
    line = {
        "metric": METRIC, "value": world * n / ((df + db) / 1e3), "unit": "images/s (descriptor forward+backward)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "images": n, "H": H, "W": W, "keypoints_per_image": wl["kps"],
                   "loss1": "sum of squared descriptor differences to a homography-warped copy (constant target)",
                   "loss2": "photometric L2 of warp + feather blend (gradients: both images, 8 homography params)",
                   "pyramid": "recomputed in backward", "parallelism": f"replicas{world}"},
        "desc_forward_ms": df, "desc_backward_ms": db, "desc_backward_over_forward": db / df,
        "warp_forward_ms": wf, "warp_backward_ms": wb, "warp_backward_over_forward": wb / wf,
        "roofline": None,
        "cpu_baseline": None,
        "e2e": None,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return line


def run_reference_stitch(args, wl):
    from oracle import stitch_oracle as so
    from pysift_b200 import synthetic
    img1, img2, _ = synthetic.stitch_pair(wl["H"], wl["W"], seed=wl["seed"])
    times = []
    for i in RefSchedule(args.warmup, args.steps):
        orc = so.OracleStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"])
        t0 = time.perf_counter()
        orc.stitch(img1, img2)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    sec = float(np.mean(times))
    value = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "H": wl["H"], "W": wl["W"], "seed": wl["seed"],
                   "ransac_iters": wl["ransac_iters"], "inlier_thresh": wl["inlier_thresh"], "match_ratio": 0.75,
                   "blend": "multiband (gain, DP seam, 6 levels)"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "one full two-image stitch per step (oracle port: C/OpenMP detection and "
                                   "RANSAC, numpy/scipy composition)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_detect(args, wl, world, rank, local):
    import torch
    import torch.distributed as dist
    from pysift_b200 import PySIFT, synthetic

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    H, W = wl["H"], wl["W"]
    img = synthetic.scene(H, W, seed=wl["seed"] + rank)
    sift = PySIFT(device=dev)
    g = torch.from_numpy(img).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(7)]

    for _ in range(args.warmup):
        sift.run_device(g)
    torch.cuda.synchronize(dev)
    b = sift._bufs[(H, W)]
    n_kp = int(b.stats.cpu()[0])

    step_ms, pyr_ms, stage = [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    from pysift_b200 import _lib
    launches0 = _lib.load().pysift_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0.record(stream)
            sift.run_device(g)  # the detection as the API runs it (a CUDA graph replay)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    launches = _lib.load().pysift_launch_count() - launches0
    # stage split and the pyramid region: the same detection with stage events
    # (recorded between eager launches)
    for _ in range(args.steps):
        flush.zero_()
        sift.run_device(g, stage_events=ev)
        ev[6].synchronize()
        pyr_ms.append(ev[0].elapsed_time(ev[3]))
        stage.append([ev[i].elapsed_time(ev[i + 1]) for i in range(6)])
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    total_ms = float(np.sum(step_ms))
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    all_ranks_max(t, world)
    total_ms = float(t.item())

    # end to end: pinned host image -> device -> pipeline -> host arrays
    pinned = torch.from_numpy(img).pin_memory()
    e2e_ms = []
    h2d = img.nbytes
    d2h = 0
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        b.gray.copy_(pinned, non_blocking=True)
        sift.run_device(b.gray)
        b.stats_host.copy_(b.stats, non_blocking=True)
        stream.synchronize()
        n = int(b.stats_host[0])
        kp = b.kpts[:n].cpu()
        rs = b.resp[:n].cpu()
        oc = b.octv[:n].cpu()
        ds = b.desc[:n].cpu()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
            d2h = b.stats.numel() * 4 + n * (4 * 4 + 4 + 4 + 128 * 4)
    e2e_tot = torch.tensor([float(np.sum(e2e_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(e2e_tot, world)

    if rank != 0:
        return None
    mpix = H * W / 1e6
    value = world * args.steps * mpix / (total_ms / 1e3)
    e2e_value = world * args.steps * mpix / (float(e2e_tot.item()) / 1e3)
    peak, peak_kind = measured_peaks()
    alg = pyramid_alg_bytes(H, W, sift)
    pyr_s = float(np.mean(pyr_ms)) / 1e3
    achieved = alg / pyr_s / 1e9
    if args.no_cpu_baseline:
        cpu_med, cpu_n, ocv = float("nan"), 0, None
    else:
        cpu_med, cpu_n = cpu_detect_baseline(img)
        ocv = opencv_baselines("detect", img, scale=mpix)
    line = {
        "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "H": H, "W": W, "seed": wl["seed"], "keypoints": n_kp,
                   "l2": "flushed (256 MiB write) before every step", "parallelism": f"replicas{world}"},
        "roofline": {"bound": "hbm", "kernel": "pyramid+DoG+extrema (k_blur x%d + k_extrema_mask)"
                     % (1 + sift.n_octaves * (sift.n_scales + 2)),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_bytes_per_launch": alg,
                     "region_ms": pyr_s * 1e3, "traffic": committed_traffic(args.workload)},
        "cpu_baseline": {"value": mpix / cpu_med, "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{cpu_n} runs of the oracle detectAndCompute on the same {W}x{H} image"},
        "e2e": {"value": e2e_value, "unit": "Mpix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "stage_ms": dict(zip(["base_image", "pyramid", "extrema_mask", "refine_cap", "orientation", "descriptor"],
                             [round(float(x), 4) for x in np.mean(np.array(stage), 0)]),
                         total=round(float(np.mean(step_ms)), 4)),
    }
    if ocv:
        ocv.update(unit="Mpix/s", sample="cv2.SIFT_create().detectAndCompute(img, None) on the same image, "
                   "median of 5 after a warm-up (the reference's examples/quick_test.py:71-80)")
        line["opencv_cpu"] = ocv
    return line


def cpu_stitch_baseline(img1, img2, wl, budget_s=20.0):
    """The oracle port of the stitch path on the host cores (bounded sample)."""
    from oracle import stitch_oracle as so
    times = []
    t_start = time.perf_counter()
    while True:
        orc = so.OracleStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"])
        t0 = time.perf_counter()
        orc.stitch(img1, img2)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s or len(times) >= 5:
            break
    return float(np.median(times)), len(times)


def run_stitch(args, wl, world, rank, local):
    import torch
    import torch.distributed as dist
    from pysift_b200 import _lib, synthetic
    from pysift_b200.stitch import GPUPyStitch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    H, W = wl["H"], wl["W"]
    img1, img2, _ = synthetic.stitch_pair(H, W, seed=wl["seed"] + rank)
    st = GPUPyStitch(ransac_iters=wl["ransac_iters"], inlier_thresh=wl["inlier_thresh"], save_output=False,
                     verbose=False, device=dev)
    g1 = torch.from_numpy(img1).to(dev)
    g2 = torch.from_numpy(img2).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = _lib.load()
    for _ in range(args.warmup):
        st.stitch(g1, g2)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = lib.pysift_launch_count()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0.record(stream)
            pano = st.stitch(g1, g2)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    launches = lib.pysift_launch_count() - launches0
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t = torch.tensor([float(np.sum(step_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(t, world)
    total_ms = float(t.item())
    m = dict(st.last_metrics)
    # end to end through the public API with host images
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        pano = st.stitch(img1, img2)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_tot = torch.tensor([float(np.sum(e2e_ms))], dtype=torch.float64, device=dev)
    all_ranks_max(e2e_tot, world)
    # stage breakdown of one more stitch (events on the stitch's stream); the
    # events run the middle stages eagerly (not as the graph replay), so one
    # eager stitch first brings that path's allocations back to warm
    st.stage_events = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    for _ in range(2):
        st.stitch(g1, g2)
        st.stage_events[5].synchronize()
    stage_ms = {name: round(st.stage_events[i].elapsed_time(st.stage_events[i + 1]), 4)
                for i, name in enumerate(st.STAGES)}
    st.stage_events = None
    # roofline of the dominant kernel region: pyramid + DoG + extrema of one view
    sift = st._detector
    gray = st._gray_clahe(g1, "img1")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(7)]
    pyr_ms = []
    for _ in range(max(3, args.steps)):
        flush.zero_()
        sift.run_device(gray, stage_events=ev)
        ev[6].synchronize()
        pyr_ms.append(ev[0].elapsed_time(ev[3]))
    if rank != 0:
        return None
    pairs_s = world * args.steps / (total_ms / 1e3)
    e2e_pairs_s = world * args.steps / (float(e2e_tot.item()) / 1e3)
    peak, peak_kind = measured_peaks()
    alg = pyramid_alg_bytes(H, W, sift)
    pyr_s = float(np.median(pyr_ms)) / 1e3
    achieved = alg / pyr_s / 1e9
    if args.no_cpu_baseline:
        cpu_s, cpu_n, ocv = float("nan"), 0, None
    else:
        cpu_s, cpu_n = cpu_stitch_baseline(img1, img2, wl)
        ocv = opencv_baselines("stitch", img1, img2)
    mpix = 2 * H * W / 1e6
    line = {
        "metric": METRIC, "value": pairs_s, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "H": H, "W": W, "seed": wl["seed"],
                   "ransac_iters": wl["ransac_iters"], "inlier_thresh": wl["inlier_thresh"], "match_ratio": 0.75,
                   "blend": "multiband (gain, DP seam, %d levels)" % st.n_blend_levels
                   if st.blend == "multiband" else "linear feather",
                   "keypoints": [m["kp1"], m["kp2"]], "matches": m["matches"],
                   "inliers": m["inliers"], "canvas": [m["canvas_w"], m["canvas_h"]],
                   "crop_xywh": list(m["crop_box"]) if m.get("crop_box") else None,
                   "l2": "flushed (256 MiB write) before every step", "parallelism": f"replicas{world}"},
        "mpix_per_s": pairs_s * mpix,
        "roofline": {"bound": "hbm", "kernel": "pyramid+DoG+extrema of one 1280x960 view (k_blur x%d + "
                     "k_extrema_mask)" % (1 + sift.n_octaves * (sift.n_scales + 2)),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_bytes_per_launch": alg, "region_ms": pyr_s * 1e3,
                     "traffic": committed_traffic(args.workload)},
        "cpu_baseline": {"value": 1.0 / cpu_s if cpu_s == cpu_s else None, "unit": "pairs/s",
                         "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{cpu_n} full stitches of the same pair by the oracle port (OpenMP)"},
        "e2e": {"value": e2e_pairs_s, "unit": "pairs/s", "h2d_bytes_per_step": int(img1.nbytes + img2.nbytes),
                "d2h_bytes_per_step": int(pano.nbytes) + 72 + 16 + (8 if st.blend == "multiband" else 0)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "stage_ms": stage_ms,
    }
    if ocv:
        ocv.update(unit="pairs/s", sample="3 stitches of the same pair after a warm-up: cv2 SIFT on both gray "
                   "views, BFMatcher(NORM_L2).knnMatch(k=2) + ratio 0.75, findHomography(USAC_MAGSAC, 4 px), "
                   "warpPerspective, linear feather")
        line["opencv_cpu"] = ocv
    return line


EXTRA_WORKLOADS = (("detect_640x480", None), ("match_u8_8192", None), ("batch96_detect", 3),
                   ("batch32_stitch", 2))


def run_extras(args, world, rank, local):
    """The other configurations of the metric, measured after the default
    stitch line on every rank (each takes the same collective steps there):
    plain detection of one 640x480 image (Mpix/s), exact 8192 x 8192 matching
    through the bf16 tensor-core GEMM (match-pairs/s, tensor roofline), and
    the batched forms against their plain per-image / per-pair loops.
    Returns {workload: summary} on rank 0, None elsewhere."""
    out = {}
    for name, steps in EXTRA_WORKLOADS:
        wl = WORKLOADS[name]
        sub = argparse.Namespace(**vars(args))
        sub.workload = name
        if steps is not None:
            sub.steps, sub.warmup = min(args.steps, steps), 3
        if wl["kind"] == "detect":
            line = run_detect(sub, wl, world, rank, local)
        elif wl["kind"] == "match":
            line = run_match(sub, wl, world, rank, local)
        elif wl["kind"] == "batch_detect":
            line = run_batch_detect(sub, wl, world, rank, local)
        else:
            line = run_batch_stitch(sub, wl, world, rank, local, batch_pairs(sub, wl, world, rank))
        if line is None:
            continue
        keep = {k: line.get(k) for k in ("value", "unit", "ms_per_step", "steps", "dtype", "roofline",
                                           "cpu_baseline", "opencv_cpu", "e2e", "gpu_launches", "clocks")}
        keep["config"] = line["config"]
        if wl["kind"] == "batch_detect":
            keep["plain_mpix_per_s"] = line["plain_mpix_per_s"]
            keep["graph_mpix_per_s"] = line["graph_mpix_per_s"]
            keep["batched_over_plain"] = line["value"] / line["plain_mpix_per_s"]
        if wl["kind"] == "batch_stitch":
            keep["plain_pairs_per_s"] = line["plain_pairs_per_s"]
            keep["batched_over_plain"] = line["value"] / line["plain_pairs_per_s"]
        out[name] = keep
    return out if rank == 0 else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline legs (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the other configurations embedded in its line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl, world, rank)
    # inputs that take a process pool are made before any CUDA work
    pairs = batch_pairs(args, wl, world, rank) if wl["kind"] == "batch_stitch" else None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if wl["kind"] == "stitch":
            line = run_stitch(args, wl, world, rank, local)
            if args.workload == DEFAULT_WORKLOAD and not args.no_extras:
                extras = run_extras(args, world, rank, local)
                if line is not None:
                    line["workloads"] = extras
        elif wl["kind"] == "match":
            line = run_match(args, wl, world, rank, local)
        elif wl["kind"] == "batch_detect":
            line = run_batch_detect(args, wl, world, rank, local)
        elif wl["kind"] == "batch_stitch":
            line = run_batch_stitch(args, wl, world, rank, local, pairs)
        elif wl["kind"] == "grad":
            line = run_grad(args, wl, world, rank, local)
        else:
            line = run_detect(args, wl, world, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
