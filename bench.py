"""Benchmark of the B200 Block-Equivalence labeler; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload 2d8192|2d2048|3d512|batch|serve|slab2d] [--subs LIST]
                    [--algo uf|iter|runs]

Default run: the 2D 8192x8192 headline plus one sub-record per other configuration of the metric
("sub": 3D 512^3, the 4096-image uneven batch against 4096 plain launches, and the served Poisson
sweep with p50 / p99), each with its own roofline, end-to-end figure and clock record, and two
more on the headline's images: the paper's iterative scan / analyze form ("iter") and the run
equivalence form ("runs", 4-connected).

Headline (2d8192): the seven seeded 8192x8192 families (Bernoulli p = 0.1 / 0.4 / 0.6 / 0.9, 2000
disks over p = 0.05 noise, serpentine, spiral), 8-connectivity, int32 labels.  One step labels one
image (the families in turn), inputs resident in HBM.  The inputs (64 MiB) fit in L2, so a 512 MiB
buffer is written between timed steps (L2 flush) and each step is timed alone with CUDA events on
the labeling stream.

`value` is Gpx/s over the timed steps (max time over ranks for N > 1; every rank labels its own
images, weak scaling).  `e2e` is the same metric through the host-buffer C-ABI call
(be_label2d_host: pinned host image -> device -> labels -> pinned host labels, wall clock) and
through the request API.  `roofline` takes the algorithmic 5 bytes per pixel (1 B read + 4 B label
write) of the whole labeling over the device time of its launches; `roofline_kernels` splits it
per launch.  `cpu_baseline` times the reference's own CPU labeler (compiled from its sources into
oracle/_ref) on the host cores, on a bounded sample; the same leg checks every timed label map
against the oracle (`mismatched_labels`, outside the timed region).

--impl reference runs only that reference CPU labeler (all host threads) on the same workload
and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import subprocess
import sys
import threading
import time

import numpy as np

from labeling_b200 import replicas

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STAGES_2D = ["k_tile_local_2d", "k_merge_2d", "k_scan_flatten_2d", "k_tile_write_2d"]
STAGES_3D = ["k_tile_local_3d", "k_merge_3d", "k_scan_link_3d", "k_tile_write_3d"]
# Algorithmic bytes per pixel of each launch (what the launch must move at minimum):
# tile_local reads the image (1 B), tile_write writes the labels (4 B); the others move only
# per-tile / per-segment metadata and have no per-pixel algorithmic traffic.
ALGO_BYTES = {"k_tile_local_2d": 1.0, "k_tile_write_2d": 4.0, "k_tile_local_3d": 1.0,
              "k_tile_write_3d": 4.0}

# Bytes the union-find pipeline itself moves per pixel / voxel, by array (reads and writes of the
# pipeline's launches, counted from the kernels' loads and stores; node records of border components,
# at most a few bytes per border pixel, are left out).  2D tile 64 x 256 px, 3D tile 16 x 32 x 64.
IMPL_BYTES = {
    "2d": {"input read": 1.0, "labels written": 4.0,
           "block entries written + read (uint16 per 2x2 block)": 2 * 0.5,
           "root bitmap written + read (1 bit per pixel)": 2 * 0.125,
           "border entries written + read twice": 3 * 640 / 16384,
           "segment counts + prefix": (1 + 1 + 4 + 4) / 256},
    "3d": {"input read": 1.0, "labels written": 4.0,
           "block entries written + read (uint32 per 2x2x2 block)": 2 * 0.5,
           "root bitmap written + read (1 bit per voxel)": 2 * 0.125,
           "border entries written + read twice": 3 * 2 * (8 * 16 + 8 * 32 + 16 * 32) * 2 / 32768,
           "segment counts + prefix": (1 + 1 + 4 + 4) / 64},
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def host_info() -> dict:
    """The host's CPU model, core count and OpenMP setting (for the CPU baseline records)."""
    model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count(),
            "omp_num_threads": os.environ.get("OMP_NUM_THREADS", "unset (OpenMP default: all)")}


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region: NVML every
    millisecond from a helper thread (the timed regions are tens of milliseconds long), with
    nvidia-smi as the fallback.  Read-only: no GPU setting is changed."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.samples = []       # (sm_mhz, max_mhz, set of reasons)
        self.nvml = None
        self.stop = threading.Event()
        self.t = None

    def _nvml_sample(self):
        n = self.nvml
        sm = n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
        r = n.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        bits = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        self.samples.append((float(sm), float(mx), {nm for nm, b in zip(self.NAMES, bits) if r & b}))

    def _nvml_loop(self):
        while not self.stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            self.stop.wait(0.001)

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self._nvml_sample()
            self.t = threading.Thread(target=self._nvml_loop, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.nvml is not None:
            self.stop.set()
            if self.t:
                self.t.join(timeout=2)
            try:
                self._nvml_sample()
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for s_, m_, r_ in self.samples:
            sm.append(s_)
            mx = m_
            reasons |= r_
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


# ------------------------------------------------------------------------------------------
# Workloads
# ------------------------------------------------------------------------------------------

def make_2d_inputs(side: int, families, seed: int):
    from labeling_b200 import workloads as W
    return [(f, W.family_8192(f, seed=seed + i, side=side)) for i, f in enumerate(families)]


def make_3d_inputs(side: int, seed: int, only: str = ""):
    import torch
    from labeling_b200 import workloads as W
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    keep = set(only.split(",")) if only else None
    out = []
    for i, p in enumerate([0.1, 0.3, 0.5]):
        if keep is None or f"bern{p}" in keep:
            out.append((f"bern{p}", W.bernoulli((side, side, side), p, seed + i)))
    for pct in (50, 80):
        if keep is None or f"grf{pct}" in keep:
            out.append((f"grf{pct}", W.grf((side, side, side), 4.0, pct, seed + pct, device=dev)))
    return out


def make_batch_inputs(n: int, rank: int, dev):
    """The uneven batch: n images, height and width log-uniform in [64, 2048] independently,
    Bernoulli density per image U[0.2, 0.8] (generated on the device, seeded)."""
    import torch
    from labeling_b200 import workloads as W
    sides = W.log_uniform_sides(n, 64, 2048, seed=1000 + rank)
    rng = np.random.default_rng(2000 + rank)
    dens = rng.uniform(0.2, 0.8, n)
    g = torch.Generator(device=dev).manual_seed(3000 + rank)
    d_in = [((torch.rand((h, w), generator=g, device=dev) < float(p)).to(torch.uint8) * 255)
            for (h, w), p in zip(sides, dens)]
    return sides, d_in


def headline_config(workload: str, names, shape, world: int) -> dict:
    """The `config` of a plain-labeling line; the reference arm prints the same dict."""
    return {"workload": workload, "images": list(names), "shape": list(shape),
            "connectivity": 26 if len(shape) == 3 else 8, "labels": "int32 canonical",
            "l2": "flushed between steps (512 MiB write)", "parallelism": f"replicas x{world}"}


# ------------------------------------------------------------------------------------------
# Reference CPU labelers (oracle/_ref), bounded samples; parity of the timed label maps
# ------------------------------------------------------------------------------------------

CPU_ALGS_2D = {
    "bleq": "TLabelEquivalenceX2, block equivalence, OpenMP, one background row and column appended",
    "runeq": "TRunEqivLabeling, run equivalence, OpenMP",
    "gr-block": "TBlockGranaLabeling, Grana blocks, 1 thread",
}


def _time_cpu_alg(O, alg, images, budget_s):
    px, t_total, n = 0, 0.0, 0
    t_start = time.perf_counter()
    while True:
        name, img = images[n % len(images)]
        t_total += (O.ref_cpu_bleq(img)[1] if alg == "bleq" else O.ref_cpu_label2d(img, alg)[1]) * 1e-6
        px += img.size
        n += 1
        if time.perf_counter() - t_start > budget_s or n >= 3 * len(images):
            break
    return px / t_total / 1e9, n, t_total


def cpu_reference_2d(images, budget_s: float, main_alg: str = "bleq"):
    """Times the reference's CPU labelers (its main.cpp registry's CPU slots, compiled from its
    sources) on whole images, each by the reference's own stopwatch around DoLabel, all host
    threads for the OpenMP ones.  The block-equivalence labeler (the bleq CPU slot) is the
    reported baseline; run equivalence and Grana are listed beside it."""
    from oracle import oracle as O
    lib = O.cpu_lib()
    if lib is None:
        if O.grana_lib() is None:
            return None
        t0 = time.perf_counter()
        n = min(len(images), 2)
        for _, img in images[:n]:
            O.ref_grana(img)
        t = time.perf_counter() - t0
        return {"value": sum(im.size for _, im in images[:n]) / t / 1e9, "unit": "Gpx/s", "cores": 1,
                "kind": "reference", "sample": f"{n} whole images (gr-block, Grana, 1 thread), {t:.2f} s",
                **host_info()}
    cores = int(lib.ref_cpu_max_threads())
    res = {}
    for alg in CPU_ALGS_2D:
        v, n, t = _time_cpu_alg(O, alg, images, budget_s / len(CPU_ALGS_2D))
        res[alg] = {"value": round(v, 4), "cores": 1 if alg == "gr-block" else cores,
                    "sample": f"{n} whole images, {t:.2f} s", "what": CPU_ALGS_2D[alg]}
    main = res[main_alg]
    return {"value": main["value"], "unit": "Gpx/s", "cores": main["cores"], "kind": "reference",
            "sample": f"{main_alg} CPU slot ({CPU_ALGS_2D[main_alg]}), {main['sample']}, reference stopwatch",
            "others": {k: v for k, v in res.items() if k != main_alg}, **host_info()}


def cpu_reference_3d(volumes, budget_s: float):
    """Times the reference's 3D block-equivalence path (its TOCLBlockEquivalence3D kernels,
    LabelingAlgs.cl, compiled as C++ and run over all host threads; the reference has no CPU 3D
    labeler of its own) on whole volumes until budget_s is spent, by the span of its kernel
    sequence."""
    from oracle import oracle as O
    lib = O.ref_lib()
    if lib is None:
        return None
    cores = int(lib.ref_set_threads(0))
    lib.ref_set_threads(1)
    px, t_total, n = 0, 0.0, 0
    t_start = time.perf_counter()
    i = 0
    while True:
        name, vol = volumes[i % len(volumes)]
        t_total += O.ref_be3d_timed(vol, 0, 0)[1] * 1e-6
        px += vol.size
        n += 1
        i += 1
        if time.perf_counter() - t_start > budget_s or n >= len(volumes):
            break
    return {"value": px / t_total / 1e9, "unit": "Gvox/s", "cores": cores, "kind": "reference",
            "sample": f"{n} whole volumes (reference bleq -3 kernels on the host, OpenMP), {t_total:.2f} s",
            **host_info()}


def check_against_oracle(items, threads: int = 8, conn8: bool = True) -> dict:
    """Parity of timed label maps, part of the cpu_baseline leg (outside every timed region):
    items are (name, image, labels as numpy, count); each is compared with the oracle's canonical
    labels (oracle/be_oracle.c, union-find restatement) in a thread pool.  Returns the number of
    differing labels and the names of the images that differ."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O

    def one(it):
        name, img, lab, n = it
        ref, k = O.ccl2d(img, 0, conn8) if img.ndim == 2 else O.ccl3d(img)
        d = int(np.count_nonzero(lab != ref))
        return name, d, int(n) != int(k)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(one, items))
    return {"mismatched_labels": int(sum(d for _, d, _ in res)),
            "images_checked": len(res),
            "count_mismatches": [nm for nm, _, c in res if c],
            "mismatched_images": [nm for nm, d, _ in res if d],
            "checker": f"oracle (CPU union-find restatement, {'8' if conn8 else '4'}-connectivity in 2D), every timed image once",
            "check_s": round(time.perf_counter() - t0, 2)}


# ------------------------------------------------------------------------------------------
# Our arm: plain per-image calls (2D 8192^2 / 2048^2, 3D 512^3)
# ------------------------------------------------------------------------------------------

def bench_plain(args, rank, world, local_rank, workload):
    import torch
    import labeling_b200 as be

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    is3d = workload == "3d512"
    algo = {"uf": be.ALGO_UF, "iter": be.ALGO_ITER, "runs": be.ALGO_RUNS}[args.algo]
    form = {"uf": "union-find", "iter": "iterative scan/analyze", "runs": "run equivalence (4-connected)"}[args.algo]
    if is3d and algo == be.ALGO_RUNS:
        raise SystemExit("run equivalence is 2D only")
    if is3d:
        inputs = make_3d_inputs(512, seed=replicas.replica_seed(100, rank),
                                only=args.families if args.workload == "3d512" else "")
        stages = STAGES_3D
        metric, unit = "Gvox/s labeled (3D 512^3 BE, 26-conn)", "Gvox/s"
    else:
        side = 2048 if workload == "2d2048" else 8192
        fams = ["bern0.5"] if side == 2048 else None
        if args.families and args.workload == workload:
            fams = args.families.split(",")
        from labeling_b200 import workloads as W
        inputs = make_2d_inputs(side, fams or W.FAMILIES_8192, seed=replicas.replica_seed(10, rank))
        stages = STAGES_2D
        metric, unit = f"Gpx/s labeled (2D {side}^2 BE, 8-conn)", "Gpx/s"
    if algo == be.ALGO_ITER:
        metric = metric.replace("BE,", "BE iterative,")
    if algo == be.ALGO_RUNS:
        metric = metric.replace("BE, 8-conn", "run equivalence, 4-conn")

    ctx = be.Context(local_rank)
    stream = torch.cuda.Stream(device=dev)
    d_in = [torch.from_numpy(a).to(dev) for _, a in inputs]
    d_out = [torch.empty(a.shape, dtype=torch.int32, device=dev) for _, a in inputs]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    npx = [a.size for _, a in inputs]

    def label(i, want=False):
        if is3d:
            return be.label3d(ctx, d_in[i], d_out[i], want_count=want, stream=stream, algo=algo)
        coh = be.COH_4 if algo == be.ALGO_RUNS else be.COH_DEFAULT
        return be.label2d(ctx, d_in[i], d_out[i], want_count=want, stream=stream, algo=algo, coh=coh)

    with torch.cuda.stream(stream):
        for i in range(max(args.warmup, 3)):
            label(i % len(inputs))
        stream.synchronize()
        counts = [label(i, want=True) for i in range(len(inputs))]

        # Timed steps: no events between the launches of a step (they would serialize the
        # launches' overlapped starts); the per-launch split comes from a second pass below.
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        px_done = 0
        with ClockSampler(local_rank) as clk:
            for s in range(args.steps):
                i = s % len(inputs)
                flush.fill_(s & 0xFF)
                ev0[s].record(stream)
                label(i)
                ev1[s].record(stream)
                px_done += npx[i]
            torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]

        # Per-launch device times (CUDA events between the launches), same steps again.
        stage_ms = np.zeros(len(stages))
        per_stage = {}
        if algo == be.ALGO_UF:
            ctx.set_stage_timing(True)
            for s in range(args.steps):
                i = s % len(inputs)
                flush.fill_(s & 0xFF)
                label(i)
                st = ctx.stage_times()
                stage_ms += np.array(st[:len(stages)])
                per_stage.setdefault(inputs[i][0], []).append(st[:len(stages)])
            torch.cuda.synchronize()
            ctx.set_stage_timing(False)
        # Every timed image labeled once more; its map is kept for the parity check.
        for i in range(len(inputs)):
            label(i)
        torch.cuda.synchronize()
    per_image = {}
    for s_, ms_ in enumerate(step_ms):
        per_image.setdefault(inputs[s_ % len(inputs)][0], []).append(ms_)
    per_image = {k: round(float(np.mean(v)), 4) for k, v in per_image.items()}
    t_ms, px_total = replicas.combine(float(sum(step_ms)), float(px_done), device=dev)
    value = px_total / (t_ms / 1e3) / 1e9

    # End to end through the host-buffer C-ABI call, pinned host memory.
    h_in = [torch.from_numpy(a).pin_memory() for _, a in inputs]
    h_out = [torch.empty(a.shape, dtype=torch.int32).pin_memory() for _, a in inputs]
    host_call = be.label3d_host if is3d else be.label2d_host
    host_kw = {"coh": be.COH_4} if algo == be.ALGO_RUNS else {}
    for i in range(min(2, len(inputs))):
        host_call(ctx, h_in[i].numpy(), out=h_out[i].numpy(), algo=algo, **host_kw)
    t0 = time.perf_counter()
    e2e_px = 0
    e2e_steps = max(1, min(args.steps, 2 * len(inputs)))
    h2d = d2h = 0
    for s in range(e2e_steps):
        i = s % len(inputs)
        host_call(ctx, h_in[i].numpy(), out=h_out[i].numpy(), algo=algo, **host_kw)
        e2e_px += npx[i]
        h2d += npx[i]
        d2h += 4 * npx[i] + 8
    e2e_s = time.perf_counter() - t0
    e2e_sync = e2e_px / e2e_s / 1e9
    e2e = {"value": round(e2e_sync, 4), "unit": unit, "h2d_bytes_per_step": int(h2d / e2e_steps),
           "d2h_bytes_per_step": int(d2h / e2e_steps), "per_call": round(e2e_sync, 4),
           "how": "pinned host image -> device -> labels -> pinned host, every step"}
    if algo == be.ALGO_UF:
        # The same host buffers through the request API (be_server_*: two lanes, so one image's
        # upload overlaps the previous image's download -- PCIe carries both directions at once).
        srv = be.Server(device=local_rank, lanes=2, max_batch=1)
        for i in range(min(2, len(inputs))):
            srv.wait(srv.submit(h_in[i].numpy(), h_out[i].numpy()))
        t0 = time.perf_counter()
        ids = [srv.submit(h_in[s % len(inputs)].numpy(), h_out[s % len(inputs)].numpy()) for s in range(e2e_steps)]
        for i in ids:
            srv.wait(i)
        e2e_srv_s = time.perf_counter() - t0
        srv.close()
        e2e_srv = e2e_px / e2e_srv_s / 1e9
        e2e.update({"value": round(max(e2e_sync, e2e_srv), 4), "pipelined": round(e2e_srv, 4),
                    "how": ("pinned host image -> device -> labels -> pinned host, every step; 'per_call' = "
                            "synchronous be_label*_host calls, 'pipelined' = be_server requests on two lanes "
                            "(uploads overlap downloads); value = the better")})

    peak, peak_kind = load_peaks()
    steps = args.steps
    px_step = px_done / steps
    ms_step = t_ms / steps
    impl = IMPL_BYTES["3d" if is3d else "2d"]
    impl_bpp = float(sum(impl.values()))
    roofline = {"bound": "hbm", "achieved": round(5.0 * px_step / (ms_step / 1e3) / 1e9, 1), "peak": peak,
                "unit": "GB/s", "peak_kind": peak_kind,
                "scope": "whole labeling (all launches of one call), 5 B/px over the timed ms_per_step",
                "algorithmic_bytes_per_labeling": int(5 * px_step),
                "traffic": int(impl_bpp * px_step),
                "traffic_source": ("analytic: bytes the pipeline's kernels load and store per labeling "
                                   f"({impl_bpp:.3f} B/px = {impl_bpp / 5:.2f}x the algorithmic 5 B/px)"),
                "traffic_by_array_bytes_per_px": {k: round(v, 4) for k, v in impl.items()}}
    roofline["frac"] = round(roofline["achieved"] / peak, 4)
    roofline["frac_of_8tbs"] = round(roofline["achieved"] / 8000.0, 4)
    kernels = []
    if algo == be.ALGO_UF:
        pipe_ms = float(stage_ms.sum()) / steps
        for name, ms in zip(stages, stage_ms / steps):
            ab = ALGO_BYTES.get(name, 0.0) * px_step
            kernels.append({"kernel": name, "ms": round(float(ms), 4),
                            "share": round(float(ms) / pipe_ms, 4) if pipe_ms else None,
                            "algorithmic_bytes": int(ab),
                            "achieved_gbs": round(ab / (ms / 1e3) / 1e9, 1) if ab and ms else None})
        roofline["dominant_kernel"] = max(kernels, key=lambda k: k["ms"])["kernel"]
        roofline["stage_sum_ms"] = round(pipe_ms, 4)
        # DRAM bytes of the launches that have a committed ncu capture (profiles/traffic.json):
        # a lower bound, since lines still dirty in L2 when a launch ends are written back later.
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        tr = None
        if os.path.exists(tp):
            try:
                tr = json.load(open(tp)).get("3d512" if is3d else "2d8192")
            except Exception:
                tr = None
        if tr:
            for k in kernels:
                k["ncu_dram_bytes"] = tr["per_kernel"].get(k["kernel"])
    clocks = clk.summary()

    result = {
        "metric": metric, "value": round(value, 3), "unit": unit, "n_gpus": world,
        "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded)",
        "config": {**headline_config(workload, [n for n, _ in inputs], inputs[0][1].shape, world),
                   "form": form},
        "e2e": e2e, "roofline": roofline, "roofline_kernels": kernels,
        "gpu_launches": (len(stages) * steps) if algo == be.ALGO_UF else None, "clocks": clocks,
        "components": {n: c for (n, _), c in zip(inputs, counts)},
        "per_image_ms": per_image,
        "per_image_stage_ms": {k: [round(float(x), 4) for x in np.mean(v, axis=0)] for k, v in per_stage.items()},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        budget = 20.0
        if not getattr(args, "cpu_leg", True):
            pass   # a sub-record of the headline run: its CPU baseline is the headline's
        elif is3d:
            result["cpu_baseline"] = cpu_reference_3d(inputs, budget)
        else:
            result["cpu_baseline"] = cpu_reference_2d(inputs, budget, "runeq" if algo == be.ALGO_RUNS else "bleq")
        items = [(n, a, o.cpu().numpy(), c) for (n, a), o, c in zip(inputs, d_out, counts)]
        result["parity"] = check_against_oracle(items, conn8=algo != be.ALGO_RUNS)
        result["mismatched_labels"] = result["parity"]["mismatched_labels"]
    ctx.close()
    return result


# ------------------------------------------------------------------------------------------
# Batched and served forms
# ------------------------------------------------------------------------------------------

def bench_batch(args, rank, world, local_rank):
    """4096 2D images, sides log-uniform in [64, 2048], Bernoulli density U[0.2, 0.8]: one batched
    CUDA-graph launch (autotuned) against 4096 plain per-image calls, both on one stream."""
    import torch
    import labeling_b200 as be

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.batch_images
    sides, d_in = make_batch_inputs(n, rank, dev)
    d_out = [torch.empty((h, w), dtype=torch.int32, device=dev) for h, w in sides]
    p_out = [torch.empty((h, w), dtype=torch.int32, device=dev) for h, w in sides]
    npx = sum(h * w for h, w in sides)
    ctx = be.Context(local_rank)
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        batch = be.Batch(ctx, list(zip(d_in, d_out)))
        choice = batch.tune(stream)
        for _ in range(max(args.warmup, 3)):
            batch.run(stream)
        stream.synchronize()
        counts = batch.counts(stream)
        if world > 1:
            torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            for a, b in ev:
                a.record(stream)
                batch.run(stream)
                b.record(stream)
            torch.cuda.synchronize()
        t_ms = sum(a.elapsed_time(b) for a, b in ev)
        # 4096 plain per-image calls (the C entry point called directly, no count read-back)
        f = be.lib().be_label2d
        sp = stream.cuda_stream
        args_list = [(ctx.handle, x.data_ptr(), int(x.stride(0)), int(x.shape[0]), int(x.shape[1]), 0,
                      be.COH_DEFAULT, be.ALGO_UF, y.data_ptr(), int(y.stride(0)), None, sp)
                     for x, y in zip(d_in, p_out)]
        for a_ in args_list[:64]:
            f(*a_)
        stream.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for a_ in args_list:
            f(*a_)
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1)
        # every batched result against its plain call (on the device, outside the timed regions)
        differ = [i for i in range(n) if not torch.equal(d_out[i], p_out[i])]
    t_ms, px_all = replicas.combine(t_ms, float(npx * args.steps), device=dev)
    value = px_all / (t_ms / 1e3) / 1e9
    plain = npx / (plain_ms / 1e3) / 1e9
    # end to end: pinned host images -> device -> batch graph -> labels back to pinned host
    h_in = [x.cpu().pin_memory() for x in d_in]
    h_out = [torch.empty(x.shape, dtype=torch.int32).pin_memory() for x in d_in]
    e2e_steps = 2
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for _ in range(e2e_steps):
            for hi, di in zip(h_in, d_in):
                di.copy_(hi, non_blocking=True)
            batch.run(stream)
            for ho, do in zip(h_out, d_out):
                ho.copy_(do, non_blocking=True)
            stream.synchronize()
    e2e_s = time.perf_counter() - t0
    peak, peak_kind = load_peaks()
    achieved = 5.0 * npx / (t_ms / args.steps / 1e3) / 1e9
    batch.close()
    ctx.close()
    res = {
        "metric": "Gpx/s labeled (batched 2D BE, 4096 uneven images, one CUDA graph)",
        "value": round(value, 3), "unit": "Gpx/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(t_ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded)",
        "config": {"workload": "batch", "images": n, "side": "log-uniform [64, 2048]",
                   "density": "U[0.2, 0.8]", "pixels": npx, "l2": "inputs 1.3 GB > L2",
                   "tuned_choice": choice, "parallelism": f"replicas x{world}"},
        "plain_per_image": {"value": round(plain, 3), "unit": "Gpx/s", "ms": round(plain_ms, 3),
                            "launches": len(STAGES_2D) * n},
        "batched_vs_plain": round(value / world / plain, 2),
        "e2e": {"value": round(npx * e2e_steps / e2e_s / 1e9, 3), "unit": "Gpx/s",
                "h2d_bytes_per_step": int(npx), "d2h_bytes_per_step": int(4 * npx)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": int(sum(IMPL_BYTES["2d"].values()) * npx),
                     "traffic_source": "analytic (as the 2D headline, per pixel)", "peak_kind": peak_kind,
                     "scope": "whole batch (one graph), 5 B/px"},
        "gpu_launches": len(STAGES_2D) * args.steps, "clocks": clk.summary(),
        "components_total": int(sum(counts)),
        "batched_differs_from_plain": len(differ),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        pick = np.random.default_rng(77).choice(n, min(64, n), replace=False)
        items = [(int(i), d_in[i].cpu().numpy(), d_out[i].cpu().numpy(), counts[i]) for i in pick]
        res["parity"] = check_against_oracle(items)
        res["parity"]["checker"] = ("every batched image against its plain call (device compare); a seeded "
                                    "sample of 64 against the oracle")
        res["mismatched_labels"] = res["parity"]["mismatched_labels"]
    return res


def bench_serve(args, rank, world, local_rank):
    """Served mixed stream: Poisson arrivals at each rate of --rates; 80% 2D images (side
    log-uniform [256, 8192], Bernoulli p U[0.2, 0.8]) and 20% 3D volumes (side log-uniform
    [64, 384], Gaussian random field sigma 4 thresholded at its 60th percentile).  Requests are
    drawn from a pool of pre-generated pinned host inputs; each rate runs about 2 s of arrivals
    (at most 400 requests).  Reports sustained throughput and p50 / p99 latency per rate."""
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    rng = np.random.default_rng(500 + rank)
    pool = []
    g = torch.Generator(device=dev).manual_seed(600 + rank)
    for i in range(args.pool):
        if rng.random() < 0.8:
            side = int(np.exp(rng.uniform(np.log(256), np.log(8192))))
            p = float(rng.uniform(0.2, 0.8))
            img = ((torch.rand((side, side), generator=g, device=dev) < p).to(torch.uint8) * 255).cpu()
        else:
            side = int(np.exp(rng.uniform(np.log(64), np.log(384))))
            img = torch.from_numpy(W.grf((side, side, side), 4.0, 60, int(rng.integers(1 << 30)), device="cuda"))
        h_in = img.pin_memory()
        h_out = torch.empty(img.shape, dtype=torch.int32).pin_memory()
        pool.append((h_in.numpy(), h_out.numpy()))
    srv = be.Server(device=local_rank, lanes=2, max_batch=64)
    # Warm-up: single requests (first launches), then the whole pool at once, twice, so the
    # device memory pool and the pinned descriptor staging reach their largest sizes before any
    # rate is timed (growing them stalls the device once).
    for i in range(min(4, len(pool))):
        srv.wait(srv.submit(*pool[i]))
    for _ in range(2):
        for i in [srv.submit(*pool[k]) for k in range(len(pool))]:
            srv.wait(i)
    pool_counts = [None] * len(pool)
    for k in range(len(pool)):
        pool_counts[k] = srv.wait(srv.submit(*pool[k]))[1]
    sweep = []
    h2d = d2h = n_req = 0
    with ClockSampler(local_rank) as clk:
        for rate in [float(r) for r in args.rates.split(",")]:
            srv.reset_stats()
            n = int(min(400, max(20, rate * 2.0)))
            gaps = rng.exponential(1.0 / rate, n)
            picks = rng.integers(0, len(pool), n)
            ids, px = [], 0
            t0 = time.perf_counter()
            t_next = t0
            for gap, k in zip(gaps, picks):
                t_next += gap
                while time.perf_counter() < t_next:
                    pass
                ids.append(srv.submit(*pool[k]))
                px += pool[k][0].size
                h2d += pool[k][0].size
                d2h += 4 * pool[k][0].size
                n_req += 1
            sts = [srv.wait(i)[0] for i in ids]
            st = srv.stats()
            sweep.append({"rate_req_s": rate, "requests": n, "ok": int(sum(1 for x in sts if x == 0)),
                          "throughput_req_s": round(st["completed"] / max(st["wall_s"], 1e-9), 1),
                          "throughput_gpx_s": round(st["pixels"] / max(st["wall_s"], 1e-9) / 1e9, 3),
                          "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3),
                          "batches": int(st["batches"])})
    srv.close()
    best = max(sweep, key=lambda r: r["throughput_gpx_s"])
    res = {
        "metric": "served mixed 2D/3D stream: sustained Gpx/s with p50/p99 latency (Poisson sweep)",
        "value": best["throughput_gpx_s"], "unit": "Gpx/s", "n_gpus": world, "steps": len(sweep),
        "warmup": 4 + 3 * len(pool), "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": "serve", "mix": "80% 2D side 256-8192, 20% 3D side 64-384 (GRF 60th pct)",
                   "pool": len(pool), "lanes": 2, "max_batch": 64, "host_buffers": "pinned",
                   "rates_req_s": [r["rate_req_s"] for r in sweep]},
        "e2e": {"value": best["throughput_gpx_s"], "unit": "Gpx/s",
                "h2d_bytes_per_step": int(h2d / max(n_req, 1)), "d2h_bytes_per_step": int(d2h / max(n_req, 1)),
                "how": "every request: pinned host image in, labels back to pinned host; a step = one request"},
        "sweep": sweep, "clocks": clk.summary(),
        "p50_p99_ms_by_rate": {str(int(r["rate_req_s"])): [r["p50_ms"], r["p99_ms"]] for r in sweep},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        items = [(k, a, o.copy(), c) for k, ((a, o), c) in enumerate(zip(pool, pool_counts))]
        res["parity"] = check_against_oracle(items)
        res["parity"]["checker"] = "every pool request's served result against the oracle"
        res["mismatched_labels"] = res["parity"]["mismatched_labels"]
    return res


def bench_slab(args, rank, world, local_rank):
    """One 8192^2 image labeled as slabs joined by one exchange of border rows.  Under torchrun each
    rank labels one slab (rows split evenly) and the ranks all_gather the border rows over NCCL; on
    one GPU the image is cut into --parts slabs labeled in turn.  A step is one whole image; the
    time is CUDA events around the call on each rank (host merge and border copies included), max
    over ranks.  After timing, every rank checks its rows against the whole-image labeling."""
    import torch
    import labeling_b200 as be
    from labeling_b200 import slabs
    from labeling_b200 import workloads as W
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    fams = args.families.split(",") if args.families else list(W.FAMILIES_8192)
    imgs = [(f, W.family_8192(f, seed=10 + i, side=8192)) for i, f in enumerate(fams)]
    ctx = be.Context(local_rank)
    parts = world if world > 1 else args.parts
    lo, hi = slabs.slab_bounds(8192, world)[rank] if world > 1 else (0, 8192)
    d_in = [torch.from_numpy(a[lo:hi]).to(dev) for _, a in imgs]
    d_out = [torch.empty((hi - lo, 8192), dtype=torch.int32, device=dev) for _ in imgs]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(i):
        if world > 1:
            return slabs.label_distributed(ctx, d_in[i], d_out[i])
        return slabs.label_slabs(ctx, d_in[i], d_out[i], parts)

    for i in range(max(args.warmup, 3)):
        step(i % len(imgs))
    torch.cuda.synchronize()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    px = 0
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local_rank) as clk:
        for s_ in range(args.steps):
            flush.fill_(s_ & 0xFF)
            ev0[s_].record(stream)
            step(s_ % len(imgs))
            ev1[s_].record(stream)
            px += (hi - lo) * 8192
        torch.cuda.synchronize()
    t_ms, px_total = replicas.combine(float(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))), float(px), device=dev)
    # Parity: this rank's rows against the whole image labeled at once.
    bad = 0
    for i, (_, a) in enumerate(imgs):
        step(i)
        whole = torch.empty((8192, 8192), dtype=torch.int32, device=dev)
        be.label2d(ctx, torch.from_numpy(a).to(dev), whole)
        bad += int((whole[lo:hi] != d_out[i]).sum().item())
    if world > 1:
        t = torch.tensor([bad], dtype=torch.int64, device=dev)
        torch.distributed.all_reduce(t)
        bad = int(t.item())
    value = px_total / (t_ms / 1e3) / 1e9
    return {
        "metric": "Gpx/s labeled (2D 8192^2 BE, 8-conn, slab split)", "value": round(value, 3), "unit": "Gpx/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(t_ms / args.steps, 4), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": "slab2d", "images": [n for n, _ in imgs], "shape": [8192, 8192],
                   "slabs": parts, "exchange": "nccl all_gather of border rows" if world > 1 else "slabs in turn on one GPU",
                   "l2": "flushed between steps (512 MiB write)", "parallelism": f"slabs x{parts}"},
        "e2e": None, "mismatched_labels": bad, "clocks": clk.summary(),
        "gpu_launches": 7 * parts * args.steps,
    }


# ------------------------------------------------------------------------------------------
# Reference arm
# ------------------------------------------------------------------------------------------

def bench_reference(args, rank, world):
    """The reference's own CPU implementation of the path on the host cores, bounded samples of
    the same workload (rank 0 only), with the same `config` as our arm's line."""
    if rank != 0:
        return None

    def one(workload, budget):
        if workload == "3d512":
            inputs = make_3d_inputs(512, seed=100)
            cb = cpu_reference_3d(inputs, budget_s=budget)
            metric, unit = "Gvox/s labeled (3D 512^3 BE, 26-conn)", "Gvox/s"
        else:
            side = 2048 if workload == "2d2048" else 8192
            from labeling_b200 import workloads as W
            names = ["bern0.5"] if side == 2048 else W.FAMILIES_8192
            if args.families and args.workload == workload:
                names = args.families.split(",")
            inputs = make_2d_inputs(side, names, seed=10)
            cb = cpu_reference_2d(inputs, budget_s=budget, main_alg="runeq" if args.algo == "runs" else "bleq")
            metric, unit = f"Gpx/s labeled (2D {side}^2 BE, 8-conn)", "Gpx/s"
        if cb is None:
            return None
        form = {"uf": "union-find", "iter": "iterative scan/analyze", "runs": "run equivalence (4-connected)"}[args.algo]
        if args.algo == "iter":
            metric = metric.replace("BE,", "BE iterative,")
        if args.algo == "runs":
            metric = metric.replace("BE, 8-conn", "run equivalence, 4-conn")
        return {"impl": "reference", "metric": metric, "value": round(cb["value"], 4),
                "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic (seeded)",
                "config": {**headline_config(workload, [n for n, _ in inputs], inputs[0][1].shape, world),
                           "form": form},
                "cpu_baseline": cb, "e2e": {"value": round(cb["value"], 4), "unit": unit,
                                            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}

    if args.workload not in ("2d8192", "2d2048", "3d512"):
        return {"impl": "reference", "unavailable": f"the reference has no {args.workload} form "
                "(batching, serving and slab splits are this project's additions)"}
    res = one(args.workload, 40.0 if args.workload == "3d512" else 30.0)
    if res is None:
        return {"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent at build time)"}
    subs = [s for s in args.subs.split(",") if s] if (args.workload == "2d8192" and args.algo == "uf") else []
    if "3d512" in subs:
        r3 = one("3d512", 30.0)
        if r3 is not None:
            res["sub"] = {"3d512": r3}
    return res


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=28)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="2d8192", choices=["2d8192", "2d2048", "3d512", "batch", "serve", "slab2d"])
    ap.add_argument("--subs", default="3d512,batch,serve,iter,runs",
                    help="with the 2d8192 headline: the other configurations measured in the same run, "
                         "as sub-records (empty string: none)")
    ap.add_argument("--algo", default="uf", choices=["uf", "iter", "runs"],
                    help="plain workloads: union-find form (default), the iterative scan/analyze form, or "
                         "2D run equivalence (the runeq path, 4-connected)")
    ap.add_argument("--parts", type=int, default=4, help="slab2d on one GPU: number of slabs")
    ap.add_argument("--rates", default="100,300,1000,3000,5000", help="serve: Poisson rates (req/s)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg (and its parity check)")
    ap.add_argument("--families", default="", help="comma-separated subset of the workload's images "
                    "(2D families, or 3D bern0.1,bern0.3,bern0.5,grf50,grf80), for profiling captures")
    ap.add_argument("--batch-images", type=int, default=4096)
    ap.add_argument("--pool", type=int, default=40, help="serve: pre-generated requests")
    return ap.parse_args(argv)


def main():
    args = parse_args()
    rank, world, local_rank = replicas.rank_info()
    if args.impl == "reference":
        res = bench_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload == "batch":
        res = bench_batch(args, rank, world, local_rank)
    elif args.workload == "serve":
        res = bench_serve(args, rank, world, local_rank)
    elif args.workload == "slab2d":
        res = bench_slab(args, rank, world, local_rank)
    else:
        res = bench_plain(args, rank, world, local_rank, args.workload)
        subs = [s for s in args.subs.split(",") if s] if (args.workload == "2d8192" and args.algo == "uf") else []
        if subs:
            import torch
            res["sub"] = {}
            for s in subs:
                torch.cuda.empty_cache()
                if s == "3d512":
                    r = bench_plain(args, rank, world, local_rank, "3d512")
                elif s == "batch":
                    r = bench_batch(args, rank, world, local_rank)
                elif s == "serve":
                    r = bench_serve(args, rank, world, local_rank)
                elif s in ("iter", "runs"):
                    # the paper's iterative form / run equivalence on the headline's images
                    a2 = argparse.Namespace(**vars(args))
                    a2.algo, a2.cpu_leg = s, False
                    r = bench_plain(a2, rank, world, local_rank, "2d8192")
                else:
                    raise SystemExit(f"unknown sub-record {s}")
                for k in ("higher_is_better", "scaling", "vs_baseline", "dtype", "data", "n_gpus"):
                    r.pop(k, None)
                res["sub"][s] = r
            launches = [res.get("gpu_launches") or 0] + [r.get("gpu_launches") or 0 for r in res["sub"].values()]
            res["gpu_launches_all_records"] = int(sum(launches))
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
