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
                stream, max over ranks, in-library profiling off); `e2e` = the
                same through the C ABI from pinned host buffers (uploads inside
                the timed step, result read back).  After the timed steps: a
                profiled pass (kernel rooflines), the selector leg, and on
                rank 0 at N=1 the FP64 oracle's registration of the same pair
                (matrix error, TRE, argmax agreement; its time is the CPU
                baseline).
  --impl reference
                the reference's CPU path restated (oracle/: the C block
                matcher threaded with the reference's slab split, FP64 LTS,
                resampler and loop) running full registrations of the same pair
                on all host cores, as many as fit a time budget.

Profiling legs (`--leg ...`), for ncu captures on one GPU:
  matcher        one finest-level matcher call (--masked, --base-masked add
                 field-of-view masks);
  matcher16      the same call with 16-bit storage beside float32;
  registration   whole registrations of the benchmark workload;
  selector       the variance selection stage (block keep 0.5);
  resample-pass  one finest-level image + mask resampling pass;
  resample       the final-resampling interpolators through host buffers;
  batched, large the batched/served and large-configuration legs alone.

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
# seconds of full CPU registrations the reference arm times at most (at least one)
REFERENCE_BUDGET_S = 240.0


def config():
    """The workload description both arms print (identical by construction)."""
    return {"workload": WORKLOAD, "shape": list(SHAPE), "levels": LEVELS,
            "iterations_per_level": ITERS, "block_width": BW, "nhood_width": NW,
            "nhood_gap": G, "block_keep": 1.0, "lts_keep": LTS_KEEP, "mode": "symmetric",
            "transform": "affine", "baseline_metric": BASELINE_METRIC}


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


def oracle_params(O):
    return O.RegParams("symmetric", "affine", ITERS, O.BMParams(BW, 1, G, NW, 1.0), LTS_KEEP)


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


def cpu_info():
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return os.cpu_count() or 1, model


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

    def timed(fn, steps, profile):
        times, stats, res = [], [], None
        ctx.set_profiling(profile)
        ctx.stage_times()
        if profile:
            ctx.search_kernel_times()
            ctx.resample_times()
        l0 = ctx.kernel_launches()
        for _ in range(steps):
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
        rs = ctx.resample_times() if profile else (0.0, 0, 0)
        ctx.set_profiling(False)
        return times, stats, res, launches, (stage_ms, kern, rs), calls

    sampler = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    t_dev, st_dev, res_dev, launches, _, _ = timed(step_device, args.steps, False)
    t_e2e, st_e2e, res_e2e, _, _, _ = timed(step_e2e, args.steps, False)
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

    # ---- profiled pass (not part of `value`): kernel rooflines ----------------
    n_prof = max(1, min(3, args.steps))
    _, _, _, _, (stage_ms, kern, rs), calls = timed(step_device, n_prof, True)
    peaks, peak_src = load_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    # The dominant kernel, the per-x-lane FP32 NCC search: FP32 FMA bound, 2*B
    # algorithmic flops per block-NCC (the cross term; mean and sum of squares
    # come from box_stats).  Its launches are bracketed by CUDA events on the
    # context's stream and a device counter adds up the candidates it scores.
    flops_per_ncc = 2 * BW ** 3
    k_ms, k_launches, k_cands = kern
    k_avg_ms = k_ms / max(k_launches, 1)
    k_cands_per_launch = k_cands / max(k_launches, 1)
    achieved = flops_per_ncc * k_cands / (k_ms / 1e3) / 1e12 if k_ms > 0 else 0.0
    fma_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    bpc = traffic_bytes_per_candidate()
    traffic = round(bpc * k_cands_per_launch) if bpc else None
    ncc_ms_per_call = stage_ms[2] / max(calls, 1)
    # resampler: 10 algorithmic bytes per output voxel of an image + mask pass
    # (float32 image 4 B read + 4 B written, uint8 mask 1 B + 1 B)
    rs_ms, rs_passes, rs_vox = rs
    # image 4 B read + 4 B written, mask 1 B written per output voxel; the
    # workload gives no masks, so the default all-255 mask is not read
    rs_gbs = 9.0 * rs_vox / (rs_ms / 1e3) / 1e9 if rs_ms > 0 else 0.0

    out = {
        "metric": METRIC, "value": round(value, 4), "unit": "registrations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_dev / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config(),
        "parallelism": f"replicas{world}", "l2": "flushed (256 MB write) between steps",
        "latency_ms": {"p50": round(float(np.percentile(t_dev, 50)), 3),
                       "p99": round(float(np.percentile(t_dev, 99)), 3)},
        "gblock_ncc_per_s": round(ncc * args.steps * world / (total_dev / 1e3) / 1e9, 3),
        "block_ncc_per_registration": int(ncc),
        "tre_mm": round(tre(res_dev.M, res_dev.off, ph.true_matrix, ph.true_offset, SHAPE,
                            ph.spacing), 4),
        "e2e_vs_device_max_matrix_diff": float(np.max(np.abs(res_e2e.M - res_dev.M))),
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
                     "timed_in": f"a separate profiled pass of {n_prof} registrations"},
        "roofline_secondary": [
            {"kernel": "resample_kernel (image + mask pass, all levels)", "bound": "hbm",
             "achieved": round(rs_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
             "frac": round(rs_gbs / hbm_peak, 4), "passes": int(rs_passes),
             "avg_pass_ms": round(rs_ms / max(rs_passes, 1), 4),
             "voxels_per_pass": round(rs_vox / max(rs_passes, 1)),
             "bytes_per_voxel": 9, "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_src})"},
        ],
        "stage_ms_per_registration": {k: round(v / n_prof, 3) for k, v in
                                      zip(["box_stats", "selection", "ncc", "postfilter"], stage_ms)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0:
        sel = selector_leg(mb, ctx, ph, hbm_peak, peak_src)
        if sel:
            out["roofline_secondary"].append(sel)
        out["roofline_secondary"].append(resample_finest_leg(mb, ctx, ph, dev, hbm_peak,
                                                             peak_src))
    if rank == 0 and world == 1 and not args.no_parity:
        par, cpu = parity_leg(mb, ctx, ph, res_dev, args)
        out["parity"] = par
        out["cpu_baseline"] = cpu
    if rank == 0 and world == 1 and not args.no_batched:
        pairs = c2_pairs()
        out["batched"] = c2_leg(mb, ctx, dev, pairs)
        out["served"] = c3_leg(mb, ctx, pairs)
        del pairs
        out["large"] = c4_leg(mb, ctx)
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def selector_leg(mb, ctx, ph, hbm_peak, peak_src, calls=5):
    """Block-variance selection (keep the top half of the blocks by variance)
    on the 256x256x128 pair at block 4, spacing 3: the selection stage's
    CUDA-event time per call.  Algorithmic bytes: 4 per base voxel read + 8 per
    block key."""
    m = mb.BlockMatcher(ctx)
    m.SetBlockWidth(BW)
    m.SetNhoodWidth(NW)
    m.SetNhoodGap(G)
    m.SetBlockKeep(0.5)
    m.SetBaseImage(ph.moving, ph.spacing, ph.origin)
    m.SetSearchImage(ph.fixed, ph.spacing, ph.origin)
    ts = []
    for i in range(calls + 1):
        m.GetOffsets()
        if i:
            ts.append(float(m.LastTimings()[1]))
    nb = int(np.prod(m.Grid()[0]))
    m.close()
    ms = statistics.median(ts)
    nbytes = 4 * ph.moving.size + 8 * nb
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"kernel": "variance selection (select_kernel: variances, radix select and flags in one cooperative launch)",
            "bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(gbs / hbm_peak, 4), "ms_per_call": round(ms, 4), "blocks": nb,
            "algorithmic_bytes": int(nbytes), "block_keep": 0.5,
            "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_src})"}


def resample_finest_leg(mb, ctx, ph, dev, hbm_peak, peak_src, reps=10):
    """One image + mask resampling pass at the finest level's size (the pass a
    symmetric iteration makes twice): 256x256x128 float32 image and uint8 mask
    through an affine map, device buffers, CUDA events; 10 algorithmic bytes
    per output voxel."""
    import torch
    from mirorr_b200.phantom import random_rotation
    rng = np.random.default_rng(5)
    g = mb.Geometry.of(ph.moving, ph.spacing, ph.origin)
    C, e = mb.resample_map(g, g, random_rotation(rng, 4.0) @ np.diag([1.02, 0.98, 1.0]),
                           rng.uniform(-3, 3, 3))
    img = torch.from_numpy(ph.moving).to(f"cuda:{dev}")
    msk = torch.full(ph.moving.shape, 255, dtype=torch.uint8, device=f"cuda:{dev}")
    out = torch.empty_like(img)
    outm = torch.empty_like(msk)
    size = (SHAPE[0], SHAPE[1], SHAPE[2])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    ts = []
    for i in range(reps + 2):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mb.resample_device(ctx, img.data_ptr(), msk.data_ptr(), size, size, C, e,
                           out.data_ptr(), outm.data_ptr())
        e1.record(stream)
        e1.synchronize()
        if i >= 2:
            ts.append(e0.elapsed_time(e1))
    ms = statistics.median(ts)
    nbytes = 10 * ph.moving.size
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"kernel": "resample_kernel, image + mask in one launch, 256x256x128 (finest level)",
            "bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(gbs / hbm_peak, 4), "ms_per_launch": round(ms, 4),
            "voxels": int(ph.moving.size), "bytes_per_voxel": 10, "l2": "flushed before each",
            "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_src})"}


def parity_leg(mb, ctx, ph, res_dev, args):
    """The FP64 oracle's registration of the same pair on all host cores
    (outside every timed region): final matrix and offset error of the GPU
    result against it, both TREs, and the argmax agreement of one
    finest-size matcher call.  The oracle's wall time is the CPU baseline."""
    from oracle import oracle as O
    from mirorr_b200.phantom import tre
    threads, model = cpu_info()
    fixed = O.Image(ph.fixed, ph.spacing, ph.origin)
    moving = O.Image(ph.moving, ph.spacing, ph.origin)
    t0 = time.perf_counter()
    to = O.register(fixed, moving, oracle_params(O), LEVELS, threads=threads)
    dt = time.perf_counter() - t0
    dM = float(np.max(np.abs(res_dev.M - to.M)))
    doff = float(np.max(np.abs(res_dev.off - to.off)))
    # argmax agreement on a finest-size call (base = moving, search = fixed)
    m = mb.BlockMatcher(ctx)
    m.SetBlockWidth(BW)
    m.SetNhoodWidth(NW)
    m.SetNhoodGap(G)
    m.SetBaseImage(ph.moving, ph.spacing, ph.origin)
    m.SetSearchImage(ph.fixed, ph.spacing, ph.origin)
    m.GetOffsets()
    mi, best, second, status = m.BlockResults()
    m.close()
    ref = O.match_blocks(ph.moving, ph.fixed, None, None, O.BMParams(BW, 1, G, NW, 1.0),
                         threads=threads)
    s = ref.status == 1
    same = np.all(mi == ref.match, axis=1)[s]
    gap = (ref.best.astype(np.float64) - ref.second)[s]
    clear = gap > 1e-4
    par = {"oracle": "FP64 CPU restatement (oracle/), same inputs and parameters",
           "max_abs_dM_vs_oracle": dM, "max_abs_doffset_mm_vs_oracle": doff,
           "within_1e-4": bool(dM <= 1e-4),
           "tre_mm_gpu": round(tre(res_dev.M, res_dev.off, ph.true_matrix, ph.true_offset, SHAPE,
                                   ph.spacing), 5),
           "tre_mm_oracle": round(tre(to.M, to.off, ph.true_matrix, ph.true_offset, SHAPE,
                                      ph.spacing), 5),
           "finest_call_blocks": int(s.sum()),
           "finest_call_argmax_agreement": round(float(same.mean()), 6),
           "finest_call_argmax_agreement_gap_gt_1e-4": round(float(same[clear].mean()), 6),
           "finest_call_scores_bit_identical": bool(np.array_equal(best[s], ref.best[s]) and
                                                    np.array_equal(second[s], ref.second[s]))}
    cpu = {"value": round(1.0 / dt, 6), "unit": "registrations/s", "cores": threads,
           "kind": "port", "cpu_model": model,
           "sample": f"one full registration of the same pair by the FP64 oracle in {dt:.1f} s "
                     f"({threads} threads in the block matcher)"}
    return par, cpu


# ---- batched and served configurations ----------------------------------------
C2_PAIRS = 64
C2_LEVELS, C2_ITERS, C2_NW, C2_G = 3, 10, 7, 3
C2_WORKLOAD = ("64 phantom pairs of uneven sizes, per axis U{96..320} x U{96..320} x "
               "U{48..160}, 40 Gaussians each (per-pair seed), rigid/affine 50/50, classic "
               "method, 3 pyramid levels, block 4, radius 3 (343 candidates), block spacing 3, "
               "LTS keep 0.5, 10 iterations/level")


def _gen_pair(spec):
    shape, kind, seed = spec
    from mirorr_b200.phantom import make_phantom
    return make_phantom(shape, n_gauss=40, kind=kind, seed=seed, max_angle_deg=5.0,
                        max_shift_vox=8.0)


def c2_pairs(n=C2_PAIRS, seed0=2000):
    """The batched configuration's pairs, generated on the host cores in a
    spawn pool (input preparation, outside every timed region)."""
    import multiprocessing as mp
    rng = np.random.default_rng(seed0)
    specs = []
    for i in range(n):
        shape = (int(rng.integers(96, 321)), int(rng.integers(96, 321)), int(rng.integers(48, 161)))
        specs.append((shape, "rigid" if i % 2 == 0 else "affine", seed0 + i))
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        phs = pool.map(_gen_pair, specs)
    return specs, phs


def c2_leg(mb, ctx, dev, pairs, oracle_pairs=2):
    """Serial per-pair loop (float32 plain path, then the 16-bit path) against
    the batched form (all pairs in one batch, BF16 and FP16), each through
    the C ABI from host buffers with the copies inside; registrations/s of
    each, agreement of the batch with the serial 16-bit loop, and the FP64
    oracle's registration (same stored inputs) of the smallest pairs."""
    import torch
    from oracle import oracle as O
    specs, phs = pairs

    def params(kind, storage):
        return mb.reg_params(symmetric=False, kind=kind, levels=C2_LEVELS, iterations=C2_ITERS,
                             block_width=4, nhood_width=C2_NW, nhood_gap=C2_G, block_keep=1.0,
                             lts_keep=0.5, storage=storage)

    out = {"workload": C2_WORKLOAD, "pairs": len(phs),
           "voxels_mean": round(float(np.mean([ph.fixed.size for ph in phs]))), "legs": {}}
    host16 = {st: [(mb.to_storage(ph.fixed, st), mb.to_storage(ph.moving, st)) for ph in phs]
              for st in ("bf16", "f16")}
    # untimed warm-up: the first call of each path loads its kernels
    (shape0, kind0, _), ph0 = specs[0], phs[0]
    mb.register(ctx, ph0.fixed, ph0.moving, params(kind0, "f32"))
    for st in ("bf16", "f16"):
        mb.register(ctx, host16[st][0][0], host16[st][0][1], params(kind0, st))
        wb = mb.Batch(ctx, max_slots=2, hbm_budget=150e9)
        rid = wb.submit(host16[st][0][0], host16[st][0][1], params(kind0, st))
        wb.run()
        wb.result(rid)
        wb.close()
    res = {}
    for name, storage in [("serial_f32", "f32"), ("serial_bf16", "bf16")]:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rs = []
        for (shape, kind, seed), ph in zip(specs, phs):
            if storage == "f32":
                r, _ = mb.register(ctx, ph.fixed, ph.moving, params(kind, storage))
            else:
                f, m = host16[storage][len(rs)]
                r, _ = mb.register(ctx, f, m, params(kind, storage))
            rs.append(r)
        dt = time.perf_counter() - t0
        res[name] = rs
        out["legs"][name] = {"seconds": round(dt, 3), "registrations_per_s": round(len(phs) / dt, 3)}
    for name, storage in [("batch_bf16", "bf16"), ("batch_f16", "f16")]:
        # two passes through one batch: the first allocates the requests'
        # device arenas (cold), the second reuses them as a running service
        # does (warm, the figure reported)
        b = mb.Batch(ctx, max_slots=len(phs), hbm_budget=150e9)
        passes = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ids = [b.submit(f, m, params(kind, storage))
                   for (shape, kind, seed), (f, m) in zip(specs, host16[storage])]
            t1 = time.perf_counter()
            b.run()
            t2 = time.perf_counter()
            rs = [b.result(i)[0] for i in ids]
            dt = time.perf_counter() - t0
            passes.append((dt, {"submit_s": round(t1 - t0, 4), "run_s": round(t2 - t1, 4),
                                "results_s": round(t0 + dt - t2, 4)}))
        info = b.info()
        tm = b.times()
        b.close()
        res[name] = rs
        dt, phases = passes[1]
        out["legs"][name] = {"seconds": round(dt, 3), "registrations_per_s": round(len(phs) / dt, 3),
                             "cold_first_pass": {"seconds": round(passes[0][0], 3),
                                                 "registrations_per_s": round(len(phs) / passes[0][0], 3),
                                                 "phases": passes[0][1]},
                             "steps_both_passes": info["steps"], "graph_replays": info["replays"],
                             "graph_instantiations": info["captures"],
                             "graph_updates": info["updates"], "phases": phases,
                             "host_seconds_both_passes": {k: round(v, 4) for k, v in tm.items()}}
    f32 = out["legs"]["serial_f32"]["registrations_per_s"]
    for k in ("serial_bf16", "batch_bf16", "batch_f16"):
        out["legs"][k]["speedup_vs_serial_f32"] = round(out["legs"][k]["registrations_per_s"] / f32, 3)
    out["batch_vs_serial_bf16_max_abs_dM"] = float(max(
        np.max(np.abs(a.M - b.M)) for a, b in zip(res["batch_bf16"], res["serial_bf16"])))
    # FP64 oracle on the same stored inputs for the smallest pairs
    order = np.argsort([ph.fixed.size for ph in phs])[:oracle_pairs]
    checks = []
    for i in order:
        (shape, kind, seed), ph = specs[i], phs[i]
        rp = O.RegParams("classic", kind, C2_ITERS, O.BMParams(4, 1, C2_G, C2_NW, 1.0), 0.5, "bf16")
        to = O.register(O.Image(ph.fixed, ph.spacing, ph.origin),
                        O.Image(ph.moving, ph.spacing, ph.origin), rp, C2_LEVELS,
                        threads=os.cpu_count() or 1)
        checks.append({"pair": int(i), "shape": list(shape),
                       "max_abs_dM_batch_bf16_vs_oracle": float(np.max(np.abs(res["batch_bf16"][i].M - to.M))),
                       "max_abs_dM_serial_f32_vs_oracle_bf16_inputs": float(np.max(np.abs(res["serial_f32"][i].M - to.M)))})
    out["oracle_checks"] = checks
    return out


C4_SHAPE = (512, 512, 256)
C4_WORKLOAD = ("symmetric affine registration, 512x512x256 phantoms stored as FP16 (200 Gaussians, "
               "quadratic +-20 % bias field), 4 pyramid levels, block 5, radius 5 (1331 candidates), "
               "block spacing 3, 30 % of the blocks kept, LTS keep 0.5, 10 iterations/level")


def c4_leg(mb, ctx, n_batch=8, seed0=4000):
    """Large stress form: one registration, then a batch of n_batch such
    requests (different phantoms) through one batch (a cold pass, then a warm
    one), each through the C ABI from host FP16 buffers with the copies
    inside; registrations/s and the target registration error of each."""
    import torch
    from mirorr_b200.phantom import make_phantom, make_phantom_gpu, tre

    def params():
        return mb.reg_params(symmetric=True, kind="affine", levels=4, iterations=10, block_width=5,
                             nhood_width=11, nhood_gap=3, block_keep=0.3, lts_keep=0.5,
                             storage="f16")

    phs = [make_phantom_gpu(C4_SHAPE, n_gauss=200, kind="affine", seed=seed0 + i, bias=0.2,
                            max_angle_deg=8.0, max_shift_vox=12.0) for i in range(n_batch)]
    host = [(mb.to_storage(ph.fixed, "f16"), mb.to_storage(ph.moving, "f16")) for ph in phs]
    # untimed warm-up on a small volume (loads the block-width-5 kernels)
    w = make_phantom((64, 64, 48), n_gauss=10, kind="affine", seed=1)
    mb.register(ctx, mb.to_storage(w.fixed, "f16"), mb.to_storage(w.moving, "f16"), params())
    out = {"workload": C4_WORKLOAD, "data": "synthetic (GPU-generated phantoms, seeded)"}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r, st = mb.register(ctx, host[0][0], host[0][1], params())
    dt = time.perf_counter() - t0
    out["single"] = {"seconds": round(dt, 3), "registrations_per_s": round(1.0 / dt, 4),
                     "tre_mm": round(tre(r.M, r.off, phs[0].true_matrix, phs[0].true_offset,
                                         C4_SHAPE, phs[0].spacing), 3),
                     "h2d_bytes": int(st.h2d_bytes), "matcher_calls": int(st.matcher_calls),
                     "block_ncc_evaluated": int(st.block_ncc_evaluated)}
    # roofline of the search stage: the same registration again with the
    # per-stage CUDA events on (outside the timed region); the block-width-5
    # search is the direct FP32 kernel (2 * 5^3 flops per block-candidate,
    # the cross term) plus its preparation kernels, against the nominal FP32
    # FMA peak
    peaks, peak_src = load_peaks()
    ctx.set_profiling(True)
    ctx.stage_times()
    _, st_p = mb.register(ctx, host[0][0], host[0][1], params())
    stage_ms, _ = ctx.stage_times()
    ctx.set_profiling(False)
    fp32_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    flops = 2.0 * 125 * float(st_p.block_ncc_evaluated)
    tflops = flops / (float(stage_ms[2]) * 1e-3) / 1e12 if stage_ms[2] > 0 else 0.0
    out["roofline_search_stage"] = {
        "kernels": "search stage of every matcher call (box statistics, window-AND, block "
                   "preparation and the direct FP32 search ncc_fb16_kernel<__half, 5>)",
        "bound": "fma", "achieved": round(tflops, 3), "peak": round(fp32_peak, 2),
        "unit": "TFLOP/s", "frac": round(tflops / fp32_peak, 4),
        "flops_per_block_ncc": 250, "block_ncc": int(st_p.block_ncc_evaluated),
        "search_stage_ms": round(float(stage_ms[2]), 3),
        "stage_ms": {k: round(float(v), 3) for k, v in
                     zip(["box_stats", "selection", "ncc", "postfilter"], stage_ms)},
        "peak_source": "nominal FP32 FMA: 148 SMs x 128 lanes x 2 x sm_max_mhz from "
                       f"MEASURED_PEAKS.json ({peak_src})"}
    b = mb.Batch(ctx, max_slots=n_batch, hbm_budget=150e9)
    passes = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ids = [b.submit(f, m, params()) for f, m in host]
        b.run()
        rs = [b.result(i)[0] for i in ids]
        passes.append(time.perf_counter() - t0)
    b.close()
    out["batch"] = {"requests": n_batch, "seconds": round(passes[1], 3),
                    "registrations_per_s": round(n_batch / passes[1], 4),
                    "cold_first_pass_seconds": round(passes[0], 3),
                    "tre_mm": [round(tre(x.M, x.off, ph.true_matrix, ph.true_offset, C4_SHAPE,
                                         ph.spacing), 3) for x, ph in zip(rs, phs)],
                    "max_abs_dM_vs_single_request_0": float(np.max(np.abs(rs[0].M - r.M)))}
    return out


def c3_leg(mb, ctx, pairs, rates=(5, 10, 20, 50, 100, 200), per_rate=24, seed=3000):
    """Served form: Poisson arrivals at each rate, requests drawn from the
    batched configuration's pairs with 2-4 levels, classic or symmetric and
    rigid or affine (uniform), admitted into a batch against a 150 GB budget
    between steps; latency from arrival to result, by the host clock."""
    specs, phs = pairs
    rng = np.random.default_rng(seed)
    host16 = [(mb.to_storage(ph.fixed, "bf16"), mb.to_storage(ph.moving, "bf16")) for ph in phs]
    table = []
    # one serving batch for the whole sweep (its device arenas are reused by
    # later requests, as in a long-running server)
    b = mb.Batch(ctx, max_slots=64, hbm_budget=150e9)
    for rate in rates:
        reqs = []
        t = 0.0
        for _ in range(per_rate):
            t += rng.exponential(1.0 / rate)
            i = int(rng.integers(len(phs)))
            p = mb.reg_params(symmetric=bool(rng.integers(2)),
                              kind="rigid" if rng.integers(2) else "affine",
                              levels=int(rng.integers(2, 5)), iterations=C2_ITERS, block_width=4,
                              nhood_width=C2_NW, nhood_gap=C2_G, block_keep=1.0, lts_keep=0.5,
                              storage="bf16")
            reqs.append((t, i, p))
        lat, inflight = [], {}
        q = 0
        t0 = time.perf_counter()
        done_t = []
        while q < len(reqs) or inflight:
            now = time.perf_counter() - t0
            while q < len(reqs) and reqs[q][0] <= now:
                at, i, p = reqs[q]
                try:
                    rid = b.submit(host16[i][0], host16[i][1], p)
                except mb.MirorrError as e:
                    if e.name != "EBUSY":
                        raise
                    break
                inflight[rid] = at
                q += 1
            if inflight:
                b.step()
                for rid in b.poll():
                    b.result(rid)
                    end = time.perf_counter() - t0
                    lat.append(end - inflight.pop(rid))
                    done_t.append(end)
            elif q < len(reqs):
                time.sleep(max(0.0, reqs[q][0] - (time.perf_counter() - t0)))
        span = max(done_t) - reqs[0][0]
        table.append({"rate_per_s": rate, "requests": len(reqs),
                      "p50_ms": round(1e3 * float(np.percentile(lat, 50)), 2),
                      "p99_ms": round(1e3 * float(np.percentile(lat, 99)), 2),
                      "throughput_per_s": round(len(reqs) / span, 3)})
    b.close()
    return {"workload": "Poisson arrivals, requests drawn from the 64 batched pairs with 2-4 "
                        "levels, classic or symmetric, rigid or affine (uniform), BF16 storage, "
                        "150 GB budget, up to 64 in flight", "rates": table}


def run_reference(args):
    """Full CPU registrations of the workload by the reference's path restated
    (oracle/), as many as fit REFERENCE_BUDGET_S (at least one, at most
    --steps); the warm-up is one small registration that loads the code."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from mirorr_b200.phantom import make_phantom
    threads, model = cpu_info()
    O.lib()
    if args.warmup > 0:
        w = make_phantom((48, 48, 32), n_gauss=10, kind="affine", seed=1)
        O.register(O.Image(w.fixed), O.Image(w.moving), oracle_params(O), 1, threads=threads)
    ph = make_pair(seed=1000)
    fixed = O.Image(ph.fixed, ph.spacing, ph.origin)
    moving = O.Image(ph.moving, ph.spacing, ph.origin)
    times = []
    t_start = time.perf_counter()
    while len(times) < max(args.steps, 1):
        t0 = time.perf_counter()
        O.register(fixed, moving, oracle_params(O), LEVELS, threads=threads)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start + times[-1] > REFERENCE_BUDGET_S:
            break
    total = sum(times)
    v = len(times) / total
    out = {"metric": METRIC, "value": round(v, 6), "unit": "registrations/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": len(times), "steps_requested": args.steps,
           "warmup": args.warmup, "ms_per_step": round(1e3 * total / len(times), 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config(), "parallelism": f"cpu threads ({threads})",
           "latency_ms": {"p50": round(1e3 * float(np.percentile(times, 50)), 1),
                          "p99": round(1e3 * float(np.percentile(times, 99)), 1)},
           "cpu_baseline": {"value": round(v, 6), "unit": "registrations/s", "cores": threads,
                            "kind": "port", "cpu_model": model,
                            "sample": f"{len(times)} full registrations of the workload "
                                      f"({total:.1f} s); the steps that fit "
                                      f"{REFERENCE_BUDGET_S:.0f} s of the {args.steps} asked for"},
           "e2e": {"value": round(v, 6), "unit": "registrations/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_leg(args):
    """Profiling legs for ncu captures (one GPU, small and bounded)."""
    import mirorr_b200 as mb
    from mirorr_b200.phantom import make_phantom
    shape = tuple(int(v) for v in args.shape.split(","))
    ph = make_phantom(shape, n_gauss=80, kind="affine", seed=1000, max_angle_deg=8.0,
                      max_shift_vox=12.0)
    ctx = mb.Context(0)
    if args.leg == "matcher":
        # one finest-level matcher call of the benchmark (block 4, radius 4,
        # spacing 3); --masked gives the search image a 10-voxel field-of-view
        # shell of mask 0, --base-masked the base image a 12-voxel one
        m = mb.BlockMatcher(ctx)
        m.SetBlockWidth(BW)
        m.SetNhoodWidth(NW)
        m.SetNhoodGap(G)
        m.SetBlockKeep(args.block_keep)
        m.SetBaseImage(ph.moving)
        m.SetSearchImage(ph.fixed)
        if args.masked:
            sm = np.zeros(ph.fixed.shape, np.uint8)
            sm[10:-10, 10:-10, 10:-10] = 255
            m.SetSearchMask(sm)
        if args.base_masked:
            bm = np.zeros(ph.moving.shape, np.uint8)
            bm[12:-12, 12:-12, 12:-12] = 255
            m.SetBaseMask(bm)
        res = None
        for _ in range(args.calls):
            bp, _ = m.GetOffsets()
            t = m.LastTimings()
            d = m.LastDiagnostics()
            res = {"kept": int(bp.shape[0]), "ms_box_stats": float(t[0]),
                   "ms_selection": float(t[1]), "ms_ncc": float(t[2]),
                   "ms_postfilter": float(t[3]), "refined": d[0], "fallback_blocks": d[1],
                   "fast_blocks": d[4], "basemask_blocks": d[5], "blocks": d[3]}
        print(json.dumps(res))
        m.close()
    elif args.leg == "matcher16":
        # one matcher call with 16-bit storage (tensor-core search at block 4,
        # the direct search at block 5) beside the same call with float32
        # storage: block --bw, radius --radius, spacing 3
        res = {}
        for store in ["f32", args.store]:
            m = mb.BlockMatcher(ctx)
            m.SetStorage(store)
            m.SetBlockWidth(args.bw)
            m.SetNhoodWidth(2 * args.radius + 1)
            m.SetNhoodGap(G)
            m.SetBaseImage(ph.moving)
            m.SetSearchImage(ph.fixed)
            if args.masked:
                sm = np.zeros(ph.fixed.shape, np.uint8)
                sm[10:-10, 10:-10, 10:-10] = 255
                m.SetSearchMask(sm)
            ts = []
            for _ in range(args.calls):
                bp, _ = m.GetOffsets()
                ts.append([float(v) for v in m.LastTimings()])
            d = m.LastDiagnostics()
            res[store] = {"kept": int(bp.shape[0]), "ms_box_stats": ts[-1][0],
                          "ms_selection": ts[-1][1], "ms_ncc": ts[-1][2],
                          "ms_postfilter": ts[-1][3], "diag": [int(v) for v in d]}
            m.close()
        print(json.dumps(res))
    elif args.leg == "registration":
        # --calls registrations of the benchmark workload (its pair, seed
        # 1000, at --shape), host buffers in and out, for a launch list of the
        # whole path
        wp = ph
        p = reg_params(mb)
        out = []
        for _ in range(args.calls):
            r, st = mb.register(ctx, wp.fixed, wp.moving, p)
            out.append({"iterations": list(st.iterations_run)[:LEVELS],
                        "matcher_calls": int(st.matcher_calls)})
        print(json.dumps({"registrations": out, "kernel_launches": ctx.kernel_launches()}))
    elif args.leg in ("selector", "resample-pass"):
        # the variance selection stage (keep 0.5) or one finest-level image +
        # mask resampling pass, with their HBM rooflines
        import torch
        peaks, peak_src = load_peaks()
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        if args.leg == "selector":
            print(json.dumps(selector_leg(mb, ctx, ph, hbm_peak, peak_src, calls=args.calls)))
        else:
            print(json.dumps(resample_finest_leg(mb, ctx, ph, torch.cuda.current_device(),
                                                 hbm_peak, peak_src, reps=args.calls)))
    elif args.leg == "batched":
        pairs = c2_pairs(n=args.calls)
        out = {"batched": c2_leg(mb, ctx, 0, pairs, oracle_pairs=1)}
        out["served"] = c3_leg(mb, ctx, pairs, per_rate=8)
        print(json.dumps(out))
    elif args.leg == "large":
        print(json.dumps({"large": c4_leg(mb, ctx, n_batch=args.calls)}))
    elif args.leg == "resample":
        # final resampling through a small rigid transform with each
        # interpolator, host buffers (upload and read-back included)
        from mirorr_b200.phantom import random_rotation
        img = ph.moving
        rng = np.random.default_rng(3)
        M = random_rotation(rng, 6.0)
        geom = mb.Geometry.of(img, ph.spacing, ph.origin)
        C, e = mb.resample_map(geom, geom, M, rng.uniform(-3, 3, 3))
        size = (img.shape[2], img.shape[1], img.shape[0])
        calls = {
            "nn": lambda: mb.resample(ctx, img, None, size, C, e, nearest=True),
            "linear": lambda: mb.resample(ctx, img, None, size, C, e),
            "bspline": lambda: mb.resample_final(ctx, img, size, C, e, "bspline"),
            "sinc": lambda: mb.resample_final(ctx, img, size, C, e, "sinc"),
        }
        out = {"shape_xyz": list(size), "voxels": int(img.size)}
        for name, fn in calls.items():
            fn()
            ts = []
            for _ in range(args.calls):
                t0 = time.perf_counter()
                fn()
                ts.append(time.perf_counter() - t0)
            ms = float(np.median(ts) * 1e3)
            out[name] = {"ms_per_call": round(ms, 3), "voxels_per_s": float(img.size / (ms * 1e-3))}
        print(json.dumps(out))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the FP64 oracle registration (parity and CPU baseline)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched (64 uneven pairs) and served (Poisson) legs")
    ap.add_argument("--leg", choices=["matcher", "matcher16", "resample", "resample-pass",
                                      "selector", "registration", "batched", "large"],
                    default=None)
    ap.add_argument("--store", default="bf16")
    ap.add_argument("--radius", type=int, default=3)
    ap.add_argument("--bw", type=int, default=BW, help="block width of the matcher16 leg")
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--shape", default="256,256,128")
    ap.add_argument("--masked", action="store_true")
    ap.add_argument("--base-masked", action="store_true")
    ap.add_argument("--block-keep", type=float, default=1.0)
    args = ap.parse_args()
    if args.leg:
        run_leg(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
