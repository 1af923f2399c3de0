"""Benchmark: symmetric-mode affine registration of a 256x256x128 float32 pair.

Workload (one "step" = one full registration, the reference's
`mirorr --reg-mode symmetric -t affine --blockwidth 4 --nhoodwidth 9
--nhoodgap 3 -n 10 --pyr-num 3 --pyr-end 0`):
  synthetic phantom pair of 256x256x128 voxels (80 Gaussians, non-monotone
  intensity map on the moving image, known affine transform), 3 pyramid
  levels, block side 4, search radius +-4 (729 candidates), block spacing 3,
  LTS keep 0.5, up to 10 iterations per level, FP32 plain GPU path.

Arms:
  default       the CUDA path.  `value` = registrations/s with the inputs
                already in HBM (device-timed with CUDA events on the library's
                stream, max over ranks); `e2e` = the same through the C ABI
                from pinned host buffers (uploads inside the timed step,
                result read back).
  --impl reference
                the reference's CPU block matcher, restated in C
                (oracle/mirorr_oracle.c, threaded with the reference's slab
                split) on all host cores, on a bounded sample of the workload;
                registrations/s extrapolated from its block-NCC rate.

Multi-GPU: registrations are independent, so N ranks run N replicas, each its
own pair (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (256, 256, 128)
N_GAUSS = 80
LEVELS = 3
ITERS = 10
BW, NW, G = 4, 9, 3
LTS_KEEP = 0.5
METRIC = "registrations/s"
BASELINE_METRIC = ("registrations/s & p50/p99 latency at ≤1e-4 matrix err; "
                   "G block-NCC/s vs roofline")
WORKLOAD = ("symmetric affine registration, 256x256x128 float32 phantom pair (80 Gaussians), "
            "3 pyramid levels, block 4, radius 4 (729 candidates), block spacing 3, "
            "LTS keep 0.5, 10 iterations/level")


def traffic_bytes_per_candidate():
    """DRAM bytes per scored candidate of the search kernel, from the committed
    ncu summary (line 'bytes_per_candidate: X'); None when absent."""
    p = os.path.join(ROOT, "profiles", "ncc_xlane_kernel_256x256x128.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.strip().startswith("bytes_per_candidate:"):
                return float(line.split(":", 1)[1])
    return None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_pair(seed):
    from mirorr_b200.phantom import make_phantom
    return make_phantom(SHAPE, n_gauss=N_GAUSS, kind="affine", seed=seed, max_angle_deg=8.0,
                        max_shift_vox=12.0)


def reg_params(mb):
    return mb.reg_params(symmetric=True, kind="affine", levels=LEVELS, iterations=ITERS,
                         block_width=BW, nhood_width=NW, nhood_gap=G, block_keep=1.0,
                         lts_keep=LTS_KEEP)


def dist_setup(n):
    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), dist


def run_cuda(args):
    import torch
    import mirorr_b200 as mb
    from mirorr_b200.phantom import tre

    rank, world, dist = dist_setup(args.gpus)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    ph = make_pair(seed=1000 + rank)
    ctx = mb.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    p = reg_params(mb)
    # device-resident inputs
    fixed_d = torch.from_numpy(ph.fixed).to(f"cuda:{dev}")
    moving_d = torch.from_numpy(ph.moving).to(f"cuda:{dev}")
    geom = mb.Geometry.of(ph.fixed, ph.spacing, ph.origin)
    # pinned host inputs for the e2e arm
    fixed_h = torch.from_numpy(ph.fixed).pin_memory()
    moving_h = torch.from_numpy(ph.moving).pin_memory()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    torch.cuda.synchronize()

    def step_device():
        return mb.register_device(ctx, fixed_d.data_ptr(), geom, moving_d.data_ptr(), geom, p)

    def step_e2e():
        return mb.register(ctx, fixed_h.numpy(), moving_h.numpy(), p, geom, geom)

    for _ in range(args.warmup):
        step_device()
        step_e2e()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(fn, profile):
        times, stats, res = [], [], None
        ctx.set_profiling(profile)
        ctx.stage_times()
        if profile:
            ctx.search_kernel_times()
        l0 = ctx.kernel_launches()
        for _ in range(args.steps):
            flush.fill_(1.0)  # L2 flush between steps, outside the events
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res, st = fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
        launches = ctx.kernel_launches() - l0
        stage_ms, calls = ctx.stage_times()
        kern = ctx.search_kernel_times() if profile else (0.0, 0, 0)
        ctx.set_profiling(False)
        return times, stats, res, launches, (stage_ms, kern), calls

    sampler = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    t_dev, st_dev, res_dev, launches, (stage_ms, kern), calls = timed(step_device, True)
    t_e2e, st_e2e, res_e2e, _, _, _ = timed(step_e2e, False)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier()

    total_dev = sum(t_dev)
    total_e2e = sum(t_e2e)
    if dist is not None:
        tt = torch.tensor([total_dev, total_e2e], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_dev, total_e2e = float(tt[0]), float(tt[1])
    regs = args.steps * world
    value = regs / (total_dev / 1e3)
    e2e_value = regs / (total_e2e / 1e3)
    ncc = st_dev[-1].block_ncc_evaluated
    peaks, peak_src = load_peaks()
    # Roofline of the dominant kernel, the per-x-lane FP32 NCC search: FP32 FMA
    # bound, 2*B algorithmic flops per block-NCC (the cross term; mean and sum
    # of squares come from box_stats).  Its launches are bracketed by CUDA
    # events on the context's stream and a device counter adds up the
    # candidates it scores.
    flops_per_ncc = 2 * BW ** 3
    k_ms, k_launches, k_cands = kern
    k_avg_ms = k_ms / max(k_launches, 1)
    k_cands_per_launch = k_cands / max(k_launches, 1)
    achieved = flops_per_ncc * k_cands / (k_ms / 1e3) / 1e12 if k_ms > 0 else 0.0
    fma_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    bpc = traffic_bytes_per_candidate()
    traffic = round(bpc * k_cands_per_launch) if bpc else None
    ncc_ms_per_call = stage_ms[2] / max(calls, 1)
    ncc_per_call = sum(s.block_ncc_evaluated for s in st_dev) / max(
        sum(s.matcher_calls for s in st_dev), 1)
    err = tre(res_dev.M, res_dev.off, ph.true_matrix, ph.true_offset, SHAPE, ph.spacing)
    d_e2e = np.max(np.abs(res_e2e.M - res_dev.M))
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": "registrations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_dev / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "shape": list(SHAPE), "levels": LEVELS,
                   "iterations_per_level": ITERS, "block_width": BW, "nhood_width": NW,
                   "nhood_gap": G, "lts_keep": LTS_KEEP, "mode": "symmetric", "transform": "affine",
                   "parallelism": f"replicas{world}", "l2": "flushed (256 MB write) between steps",
                   "baseline_metric": BASELINE_METRIC},
        "latency_ms": {"p50": round(float(np.percentile(t_dev, 50)), 3),
                       "p99": round(float(np.percentile(t_dev, 99)), 3)},
        "gblock_ncc_per_s": round(ncc * args.steps * world / (total_dev / 1e3) / 1e9, 3),
        "block_ncc_per_registration": int(ncc),
        "tre_mm": round(err, 4),
        "e2e_vs_device_max_matrix_diff": float(d_e2e),
        "e2e": {"value": round(e2e_value, 4), "unit": "registrations/s",
                "h2d_bytes_per_step": int(st_e2e[-1].h2d_bytes),
                "d2h_bytes_per_step": int(st_e2e[-1].d2h_bytes),
                "latency_ms": {"p50": round(float(np.percentile(t_e2e, 50)), 3),
                               "p99": round(float(np.percentile(t_e2e, 99)), 3)}},
        "roofline": {"kernel": f"ncc_xlane_kernel<{NW}> (FP32 NCC search)", "bound": "fma",
                     "achieved": round(achieved, 3), "peak": round(fma_peak, 2),
                     "unit": "TFLOP/s", "frac": round(achieved / fma_peak, 4), "traffic": traffic,
                     "peak_source": "nominal FP32 FMA: 148 SMs x 128 lanes x 2 x sm_max_mhz "
                                    f"from MEASURED_PEAKS.json ({peak_src}); that file has no "
                                    "FP32 figure",
                     "flops_per_block_ncc": flops_per_ncc,
                     "launches": int(k_launches),
                     "avg_launch_ms": round(k_avg_ms, 4),
                     "candidates_per_launch": round(k_cands_per_launch),
                     "traffic_source": "dram bytes read+written per candidate from the ncu "
                                       "capture in profiles/ncc_xlane_kernel_256x256x128.md, "
                                       "times this run's candidates per launch",
                     "ncc_stage_ms_per_call": round(ncc_ms_per_call, 4),
                     "ncc_stage_block_ncc_per_call": round(ncc_per_call)},
        "stage_ms_per_registration": {k: round(v / args.steps, 3) for k, v in
                                      zip(["box_stats", "selection", "ncc", "postfilter"], stage_ms)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, sample_only=True)
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def registration_ncc_counts():
    """Block-NCC evaluations per matcher call at each level (all blocks)."""
    from oracle import oracle as O
    out = []
    ms, _ = O.pyramid_schedule(SHAPE, SHAPE, np.ones(3), np.ones(3), 32, LEVELS)
    for f in ms:
        size = tuple(int(s // fi) for s, fi in zip(SHAPE, f))
        nb, st = O.block_grid(size, BW, G)
        per_axis = []
        for d in range(3):
            tot = 0
            for b in range(nb[d]):
                o = st[d] + b * G
                lo = max(0, o - NW // 2)
                hi = min(size[d] - BW, o + NW // 2)
                tot += hi - lo + 1
            per_axis.append(tot)
        out.append(per_axis[0] * per_axis[1] * per_axis[2])
    return out


def cpu_baseline(args, sample_only=False):
    """The reference CPU matcher (oracle/mirorr_oracle.c restatement, threaded
    as itkBlockMatcherThreaded) timed on a bounded sample: the finest level's
    matcher on a 16-slice slab of the pair.  Registrations/s are extrapolated
    from the measured block-NCC rate (10 iterations x 2 matcher calls per level)."""
    from oracle import oracle as O
    ph = make_pair(seed=1000)
    threads = os.cpu_count() or 1
    slab = slice(56, 72)
    base = np.ascontiguousarray(ph.moving[slab])
    search = np.ascontiguousarray(ph.fixed[slab])
    p = O.BMParams(BW, 1, G, NW, 1.0)
    O.lib()
    t0 = time.perf_counter()
    r = O.match_blocks(base, search, None, None, p, threads=threads)
    dt = time.perf_counter() - t0
    nb = r.best.size
    # candidates evaluated in the sample
    size = (base.shape[2], base.shape[1], base.shape[0])
    per_axis = []
    for d in range(3):
        tot = 0
        for b in range(r.nblocks[d]):
            o = r.start[d] + b * G
            tot += min(size[d] - BW, o + NW // 2) - max(0, o - NW // 2) + 1
        per_axis.append(tot)
    sample_ncc = per_axis[0] * per_axis[1] * per_axis[2]
    rate = sample_ncc / dt
    per_reg = sum(registration_ncc_counts()) * ITERS * 2
    value = rate / per_reg
    return {"value": round(value, 6), "unit": "registrations/s", "cores": threads, "kind": "port",
            "sample": f"finest-level matcher on a 16-slice slab ({nb} blocks, {sample_ncc} "
                      f"block-NCCs) in {dt:.2f} s; extrapolated to {per_reg} block-NCCs per "
                      "registration (3 levels x 10 iterations x 2 calls)",
            "block_ncc_per_s": round(rate, 1)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    samples = []
    for _ in range(max(args.warmup, 0)):
        cpu_baseline(args)
    for _ in range(args.steps):
        samples.append(cpu_baseline(args))
    v = statistics.median([s["value"] for s in samples])
    out = {"metric": METRIC, "value": v, "unit": "registrations/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1e3 / v, 1) if v else None, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "shape": list(SHAPE), "levels": LEVELS,
                      "iterations_per_level": ITERS, "block_width": BW, "nhood_width": NW,
                      "nhood_gap": G, "parallelism": "cpu threads"},
           "cpu_baseline": dict(samples[-1], value=v),
           "e2e": {"value": v, "unit": "registrations/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
