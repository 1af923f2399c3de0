"""Final resampling of the benchmark's 256x256x128 phantom through a small
rigid transform with each interpolator of GetResampledImage, timed through
the C ABI with host buffers (the upload and the read-back included).

    python -m mirorr_b200.resample_workload [--reps N]

Prints one JSON object: milliseconds per call (median of N) per interpolator
and the output voxels per second.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom, random_rotation


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--shape", default="256,256,128")
    args = ap.parse_args()
    shape = tuple(int(v) for v in args.shape.split(","))
    ph = make_phantom(shape, n_gauss=80, kind="rigid", seed=1000)
    img = ph.moving
    rng = np.random.default_rng(3)
    M = random_rotation(rng, 6.0)
    geom = mb.Geometry.of(img, ph.spacing, ph.origin)
    C, e = mb.resample_map(geom, geom, M, rng.uniform(-3, 3, 3))
    size = (img.shape[2], img.shape[1], img.shape[0])
    ctx = mb.Context(0)
    calls = {
        "nn": lambda: mb.resample(ctx, img, None, size, C, e, nearest=True),
        "linear": lambda: mb.resample(ctx, img, None, size, C, e),
        "bspline": lambda: mb.resample_final(ctx, img, size, C, e, "bspline"),
        "sinc": lambda: mb.resample_final(ctx, img, size, C, e, "sinc"),
    }
    out = {"shape_xyz": list(size), "voxels": int(img.size)}
    for name, fn in calls.items():
        fn()  # warm-up
        ts = []
        for _ in range(args.reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        ms = float(np.median(ts) * 1e3)
        out[name] = {"ms_per_call": round(ms, 3), "voxels_per_s": float(img.size / (ms * 1e-3))}
    print(json.dumps(out))
    ctx.close()


if __name__ == "__main__":
    main()
