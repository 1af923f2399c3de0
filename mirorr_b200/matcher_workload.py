"""One block-matching call (GetOffsets) on the benchmark's 256x256x128
phantom pair, for kernel profiling.

    python -m mirorr_b200.matcher_workload [--calls N] [--masked] [--base-masked]

Block width 4, search radius 4 (9^3 = 729 candidates), block spacing 3: the
finest-level matcher call of the symmetric affine benchmark.  --masked gives
the search image a field-of-view border (mask 0 on a 10-voxel shell), as a
resampled image has.  Prints the per-stage CUDA-event timings and the
fast/general path split.  --base-masked gives the base image a 12-voxel
shell (blocks across its edge take the general search kernel).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--masked", action="store_true")
    ap.add_argument("--base-masked", action="store_true")
    ap.add_argument("--shape", default="256,256,128")
    args = ap.parse_args()
    shape = tuple(int(v) for v in args.shape.split(","))
    ph = make_phantom(shape, n_gauss=80, kind="affine", seed=1000, max_angle_deg=8.0,
                      max_shift_vox=12.0)
    ctx = mb.Context(0)
    m = mb.BlockMatcher(ctx)
    m.SetBlockWidth(4)
    m.SetNhoodWidth(9)
    m.SetNhoodGap(3)
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
    out = []
    for _ in range(args.calls):
        bp, _ = m.GetOffsets()
        t = m.LastTimings()
        d = m.LastDiagnostics()
        out.append({"kept": int(bp.shape[0]), "ms_box_stats": float(t[0]),
                    "ms_selection": float(t[1]), "ms_ncc": float(t[2]),
                    "ms_postfilter": float(t[3]), "refined": d[0], "fallback_blocks": d[1],
                    "fast_blocks": d[4], "basemask_blocks": d[5], "blocks": d[3]})
    print(json.dumps(out[-1]))
    m.close()
    ctx.close()


if __name__ == "__main__":
    main()
