"""Generates tests/golden/optkmatch_cases.npz from the reference's own OpenCL
block-matching kernel (src/mirorr/kernels/optKmatchMask.cl), compiled for the
CPU by oracle/build_ref.sh into oracle/_ref/liboptkmatch_ref.so.

Run here (where the reference tree exists):  python tests/golden/make_golden.py
Each case stores the inputs (base/search images and masks, block parameters)
and the kernel's outputs per block in grid raster order: the linear voxel
index of the best match origin, the best and the second-best squared NCC.

Cases use block width 4 (64 work-items) or 2: the kernel's tree reduction
(optKmatchMask.cl:46-59) is only exact for power-of-two work-group sizes.
Block gap 1 only: for a gap > 1 the OpenCL and CPU matchers clip the upper end
of the search window differently (optKmatchMask.cl:199-209 vs
itkBlockMatcher.txx:746-756).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mirorr_b200.phantom import make_phantom  # noqa: E402

REF_SO = os.path.join(ROOT, "oracle", "_ref", "liboptkmatch_ref.so")


def ref_lib():
    if not os.path.exists(REF_SO):
        subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh")])
    L = ctypes.CDLL(REF_SO)
    L.ref_optkmatch.restype = ctypes.c_long
    return L


def run_ref(L, base, search, bmask, smask, bw, nw, bgap, ngap):
    d, h, w = base.shape
    nb = ((w - bw) // ngap + 1) * ((h - bw) // ngap + 1) * ((d - bw) // ngap + 1)
    km = np.zeros(nb, np.uint32)
    sc = np.zeros(nb, np.float32)
    s2 = np.zeros(nb, np.float32)
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    n = L.ref_optkmatch(P(base, ctypes.c_float), P(search, ctypes.c_float),
                        P(bmask, ctypes.c_uint8), P(smask, ctypes.c_uint8), w, h, d, bw, nw, bgap,
                        ngap, P(km, ctypes.c_uint32), P(sc, ctypes.c_float), P(s2, ctypes.c_float),
                        os.cpu_count() or 1)
    assert n == nb
    return km, sc, s2


def cases():
    out = []
    ph = make_phantom((22, 20, 16), n_gauss=10, seed=11)
    full = np.full(ph.fixed.shape, 255, np.uint8)
    out.append(dict(name="plain_bw4_w7_g3", base=ph.moving, search=ph.fixed, bmask=full,
                    smask=full, bw=4, nw=7, bgap=1, ngap=3))
    sm = full.copy()
    sm[:, :, :4] = 0
    sm[:3] = 0
    bm = full.copy()
    bm[:, 15:, :] = 0
    out.append(dict(name="masked_bw4_w7_g3", base=ph.moving, search=ph.fixed, bmask=bm,
                    smask=sm, bw=4, nw=7, bgap=1, ngap=3))
    ph2 = make_phantom((20, 18, 14), n_gauss=8, kind="affine", seed=12)
    full2 = np.full(ph2.fixed.shape, 255, np.uint8)
    out.append(dict(name="plain_bw4_w5_g2", base=ph2.fixed, search=ph2.moving, bmask=full2,
                    smask=full2, bw=4, nw=5, bgap=1, ngap=2))
    out.append(dict(name="plain_bw2_w5_g2", base=ph2.moving, search=ph2.fixed, bmask=full2,
                    smask=full2, bw=2, nw=5, bgap=1, ngap=2))
    out.append(dict(name="plain_bw4_w9_g3", base=ph.moving, search=ph.fixed, bmask=full,
                    smask=full, bw=4, nw=9, bgap=1, ngap=3))
    flat = ph2.fixed.copy()
    flat[:, :, :8] = 0.25  # constant slab: degenerate (score -2) candidates
    out.append(dict(name="flat_bw4_w5_g2", base=flat, search=ph2.moving, bmask=full2,
                    smask=full2, bw=4, nw=5, bgap=1, ngap=2))
    return out


def main():
    L = ref_lib()
    arrays = {}
    names = []
    for c in cases():
        km, sc, s2 = run_ref(L, np.ascontiguousarray(c["base"], np.float32),
                             np.ascontiguousarray(c["search"], np.float32),
                             np.ascontiguousarray(c["bmask"], np.uint8),
                             np.ascontiguousarray(c["smask"], np.uint8),
                             c["bw"], c["nw"], c["bgap"], c["ngap"])
        n = c["name"]
        names.append(n)
        arrays[f"{n}/base"] = np.asarray(c["base"], np.float32)
        arrays[f"{n}/search"] = np.asarray(c["search"], np.float32)
        arrays[f"{n}/bmask"] = np.asarray(c["bmask"], np.uint8)
        arrays[f"{n}/smask"] = np.asarray(c["smask"], np.uint8)
        arrays[f"{n}/params"] = np.array([c["bw"], c["nw"], c["bgap"], c["ngap"]], np.int32)
        arrays[f"{n}/ref_match"] = km
        arrays[f"{n}/ref_best"] = sc
        arrays[f"{n}/ref_second"] = s2
        print(n, km.size, "blocks")
    arrays["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "optkmatch_cases.npz"), **arrays)


if __name__ == "__main__":
    main()
