"""CPU oracle for Mirorr's block-matching registration hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker of the CUDA product in
``mirorr_b200``: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it.  The product never imports it.

It is a restatement, in numpy (FP64) plus the C core in ``mirorr_oracle.c``,
of the reference's algorithm:

* block matching (grid, variance selection, masked NCC search, post-filter,
  thread split)            -- mirorr_oracle.c (see its header for citations)
* ITK transform semantics  -- MatrixOffsetTransformBase / Euler3DTransform /
  AffineTransform as used throughout src/mirorr/itkMirorrRegistrationMethod.txx
  and itkSymMirorrRegistrationMethod.txx (ITK itself is absent; its documented
  behaviour is restated: T(x) = M (x - c) + c + t, offset = t + c - M c,
  Compose(other, pre), GetInverse keeps the centre, Euler3D uses Z*X*Y)
* classic LTS              -- itkMirorrRegistrationMethod.txx:758-1106
* symmetric LTS            -- itkSymMirorrRegistrationMethod.txx:729-1442
* half-space transforms    -- itkSymMirorrRegistrationMethod.txx:139-201 and
  the Denman-Beavers square root of src/mirorr/vnl_utils.h:46-119
* classic / symmetric loop -- itkMirorrRegistrationMethod.txx:422-659,
  itkSymMirorrRegistrationMethod.txx:238-720
* level loop               -- itkMirorrPyramidImplement.txx:71-158
* pyramid schedule         -- itkPyramidScheduleTuner.txx:250-414 (UpdateSymmetric)
* vnl quaternion helpers   -- vnl_quaternion's published conventions: (x,y,z,r)
  storage, rotation_euler_angles for R = Rz*Ry*Rx, axis()/angle().

Parity status: the NCC search is pinned against the reference's own OpenCL
kernel compiled on the CPU (``oracle/build_ref.sh``, golden vectors in
``tests/golden``).  Everything else here is PARITY UNPINNED: the reference
ships no tests or fixtures and cannot be built (ITK, VXL and Boost are
absent), so the ITK/vnl pieces are restatements of their published behaviour.

The image pyramid is NOT the reference's (ITK's recursive Gaussian); it is this
project's own documented Gaussian + decimation, shared by the oracle and the
product so that it is not a parity variable.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile mirorr_oracle.c into oracle/_build/liboracle.so."""
    src = os.path.join(_HERE, "mirorr_oracle.c")
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(src)):
        return _LIB_PATH
    os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
    tmp = _LIB_PATH + f".tmp{os.getpid()}"
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                           "-shared", "-pthread", "-o", tmp, src, "-lm"])
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        i3 = ctypes.POINTER(ctypes.c_int)
        _lib.orc_match.restype = ctypes.c_int
        _lib.orc_emit_points.restype = ctypes.c_long
        _lib.orc_block_grid.restype = ctypes.c_int
        _lib.orc_variance_cutoff.restype = ctypes.c_int
        del i3
    return _lib


def _p(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


# ---------------------------------------------------------------------------
# Images
# ---------------------------------------------------------------------------
@dataclass
class Image:
    """A 3D volume in ITK layout: data[z, y, x] (x fastest in memory)."""
    data: np.ndarray
    spacing: np.ndarray = field(default_factory=lambda: np.ones(3))
    origin: np.ndarray = field(default_factory=lambda: np.zeros(3))
    direction: np.ndarray = field(default_factory=lambda: np.eye(3))

    @property
    def size(self):  # (nx, ny, nz)
        return (self.data.shape[2], self.data.shape[1], self.data.shape[0])

    def index_to_physical(self):
        return self.direction * self.spacing[None, :]

    def center(self):
        """ComputeImageCenter (itkMirorrRegistrationMethod.txx): physical point of
        continuous index (size - 1) / 2."""
        ci = (np.array(self.size, dtype=np.float64) - 1.0) / 2.0
        return self.origin + self.index_to_physical() @ ci


def geometry_like(img: Image, data):
    return Image(data, img.spacing.copy(), img.origin.copy(), img.direction.copy())


# ---------------------------------------------------------------------------
# Block matching (C core)
# ---------------------------------------------------------------------------
@dataclass
class BMParams:
    block_width: int = 4
    block_gap: int = 1
    nhood_gap: int = 2
    nhood_width: int = 5
    block_keep: float = 1.0


def block_grid(size, bw, gap):
    nb = (ctypes.c_int * 3)()
    st = (ctypes.c_int * 3)()
    if lib().orc_block_grid(_i3(size), int(bw), int(gap), nb, st):
        raise ValueError("image smaller than a block")
    return tuple(nb), tuple(st)


def block_variances(img: np.ndarray, bw: int, gap: int) -> np.ndarray:
    img = np.ascontiguousarray(img, dtype=np.float32)
    size = (img.shape[2], img.shape[1], img.shape[0])
    nb, _ = block_grid(size, bw, gap)
    out = np.zeros(nb[0] * nb[1] * nb[2], dtype=np.float64)
    lib().orc_block_variances(_p(img, ctypes.c_float), _i3(size), int(bw), int(gap),
                              _p(out, ctypes.c_double))
    return out


def variance_selection(var: np.ndarray, keep: float):
    """Returns (selected uint8 mask or None, cutoff or None)."""
    cut = ctypes.c_double(0.0)
    on = lib().orc_variance_cutoff(_p(np.ascontiguousarray(var), ctypes.c_double),
                                   ctypes.c_long(var.size), ctypes.c_double(keep),
                                   ctypes.byref(cut))
    if not on:
        return None, None
    return (var > cut.value).astype(np.uint8), cut.value


@dataclass
class MatchResult:
    nblocks: tuple
    start: tuple
    match: np.ndarray      # (N, 3) int32 match origins (x, y, z)
    best: np.ndarray       # (N,) float32
    second: np.ndarray     # (N,) float32
    status: np.ndarray     # (N,) uint8: 0 = skipped by selection
    selected: np.ndarray | None


def match_blocks(base, search, base_mask, search_mask, p: BMParams, threads: int = 0) -> MatchResult:
    """Per-block best/second/argmax over the grid (raster order)."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    search = np.ascontiguousarray(search, dtype=np.float32)
    if base_mask is None:
        base_mask = np.full(base.shape, 255, np.uint8)
    if search_mask is None:
        search_mask = np.full(base.shape, 255, np.uint8)
    base_mask = np.ascontiguousarray(base_mask, dtype=np.uint8)
    search_mask = np.ascontiguousarray(search_mask, dtype=np.uint8)
    size = (base.shape[2], base.shape[1], base.shape[0])
    nb, st = block_grid(size, p.block_width, p.nhood_gap)
    n = nb[0] * nb[1] * nb[2]
    selected = None
    if p.block_keep < 1.0:
        var = block_variances(base, p.block_width, p.nhood_gap)
        selected, _ = variance_selection(var, p.block_keep)
    match = np.zeros((n, 3), np.int32)
    best = np.zeros(n, np.float32)
    second = np.zeros(n, np.float32)
    status = np.zeros(n, np.uint8)
    if threads <= 0:
        threads = os.cpu_count() or 1
    sel_p = _p(selected, ctypes.c_uint8) if selected is not None else None
    lib().orc_match(_p(base, ctypes.c_float), _p(search, ctypes.c_float),
                    _p(base_mask, ctypes.c_uint8), _p(search_mask, ctypes.c_uint8), _i3(size),
                    int(p.block_width), int(p.block_gap), int(p.nhood_gap), int(p.nhood_width),
                    sel_p, int(threads), _p(match, ctypes.c_int32), _p(best, ctypes.c_float),
                    _p(second, ctypes.c_float), _p(status, ctypes.c_uint8))
    return MatchResult(nb, st, match, best, second, status, selected)


def emit_points(res: MatchResult, geom: Image, p: BMParams, order: int = 0):
    """Post-filter + block->mm conversion.  order=0: raster (GPU matcher order);
    order=T: the threaded CPU matcher's order with T threads."""
    n = res.best.size
    size = geom.size
    bp = np.zeros((n, 3), np.float64)
    mp = np.zeros((n, 3), np.float64)
    kept = np.zeros(n, np.int64)
    direction = np.ascontiguousarray(geom.direction, dtype=np.float64)
    k = lib().orc_emit_points(_i3(size), int(p.block_width), int(p.nhood_gap),
                              _p(res.match, ctypes.c_int32), _p(res.best, ctypes.c_float),
                              _p(res.second, ctypes.c_float), _p(res.status, ctypes.c_uint8),
                              _p(np.ascontiguousarray(geom.origin, dtype=np.float64), ctypes.c_double),
                              _p(np.ascontiguousarray(geom.spacing, dtype=np.float64), ctypes.c_double),
                              _p(direction, ctypes.c_double), int(order),
                              _p(bp, ctypes.c_double), _p(mp, ctypes.c_double),
                              _p(kept, ctypes.c_int64))
    return bp[:k], mp[:k], kept[:k]


def get_offsets(base: Image, search: Image, base_mask, search_mask, p: BMParams, threads=0, order=0):
    """AbstractBlockMatcher::GetOffsets: (block positions, match positions) in mm."""
    res = match_blocks(base.data, search.data, base_mask, search_mask, p, threads)
    if not np.any(res.status):
        raise RuntimeError("no block matches occurred")
    bp, mp, _ = emit_points(res, base, p, order)
    return bp, mp


# ---------------------------------------------------------------------------
# Resampling
# ---------------------------------------------------------------------------
def resample_map(out_geom: Image, in_geom: Image, tfm_matrix, tfm_offset):
    """Affine map from output voxel index to input continuous index:
    c = e + C @ idx, composed from index->physical (output), the transform
    (y = M x + offset) and physical->index (input).  Evaluated in FP64."""
    a_out = out_geom.index_to_physical()
    a_in_inv = np.linalg.inv(in_geom.index_to_physical())
    C = a_in_inv @ (np.asarray(tfm_matrix) @ a_out)
    e = a_in_inv @ (np.asarray(tfm_matrix) @ out_geom.origin + np.asarray(tfm_offset) - in_geom.origin)
    return np.ascontiguousarray(C, dtype=np.float64), np.ascontiguousarray(e, dtype=np.float64)


def resample(in_data, in_mask, out_size, C, e):
    """Linear resampling on an explicit index map (see mirorr_oracle.c)."""
    in_size = (in_data.shape[2], in_data.shape[1], in_data.shape[0]) if in_data is not None else \
        (in_mask.shape[2], in_mask.shape[1], in_mask.shape[0])
    out = None
    outm = None
    shape = (out_size[2], out_size[1], out_size[0])
    fp = None
    mp = None
    if in_data is not None:
        in_data = np.ascontiguousarray(in_data, dtype=np.float32)
        out = np.zeros(shape, np.float32)
        fp = _p(in_data, ctypes.c_float)
    if in_mask is not None:
        in_mask = np.ascontiguousarray(in_mask, dtype=np.uint8)
        outm = np.zeros(shape, np.uint8)
        mp = _p(in_mask, ctypes.c_uint8)
    lib().orc_resample(fp, mp, _i3(in_size), _i3(out_size),
                       _p(np.ascontiguousarray(C), ctypes.c_double),
                       _p(np.ascontiguousarray(e), ctypes.c_double),
                       _p(out, ctypes.c_float) if out is not None else None,
                       _p(outm, ctypes.c_uint8) if outm is not None else None)
    return out, outm


def resample_nearest(in_data, in_mask, out_size, C, e):
    """Nearest-neighbour resampling on an explicit index map, as
    itk::NearestNeighborInterpolateImageFunction inside ResampleImageFilter:
    c = e + C idx evaluated left to right in FP64, inside test
    -0.5 <= c < n - 0.5 (otherwise 0), index floor(c + 0.5)."""
    ref = in_data if in_data is not None else in_mask
    n = (ref.shape[2], ref.shape[1], ref.shape[0])
    k, j, i = np.meshgrid(np.arange(out_size[2], dtype=np.float64),
                          np.arange(out_size[1], dtype=np.float64),
                          np.arange(out_size[0], dtype=np.float64), indexing="ij")
    C = np.asarray(C, np.float64).reshape(3, 3)
    c = [((e[r] + C[r, 0] * i) + C[r, 1] * j) + C[r, 2] * k for r in range(3)]
    inside = np.ones(k.shape, bool)
    idx = []
    for r in range(3):
        inside &= (c[r] >= -0.5) & (c[r] < n[r] - 0.5)
        idx.append(np.clip(np.floor(c[r] + 0.5), 0, n[r] - 1).astype(np.int64))
    out = outm = None
    if in_data is not None:
        out = np.where(inside, np.asarray(in_data, np.float32)[idx[2], idx[1], idx[0]], 0).astype(np.float32)
    if in_mask is not None:
        outm = np.where(inside, np.asarray(in_mask, np.uint8)[idx[2], idx[1], idx[0]], 0).astype(np.uint8)
    return out, outm


def _index_map(out_size, C, e, n):
    """c = e + C idx (FP64, left to right) and the buffer test
    -0.5 <= c < n - 0.5, for every output voxel (arrays in z, y, x order)."""
    k, j, i = np.meshgrid(np.arange(out_size[2], dtype=np.float64),
                          np.arange(out_size[1], dtype=np.float64),
                          np.arange(out_size[0], dtype=np.float64), indexing="ij")
    C = np.asarray(C, np.float64).reshape(3, 3)
    c = [((e[r] + C[r, 0] * i) + C[r, 1] * j) + C[r, 2] * k for r in range(3)]
    inside = np.ones(k.shape, bool)
    for r in range(3):
        inside &= (c[r] >= -0.5) & (c[r] < n[r] - 0.5)
    return c, inside


def bspline_coefficients(data):
    """Cubic B-spline coefficients of a (z, y, x) volume in FP64, restating
    itk::BSplineDecompositionImageFilter of order 3 (Unser's recursive
    prefilter, pole z = sqrt(3) - 2, mirror boundaries, tolerance 1e-10), as
    used by BSplineInterpolateImageFunction for GetResampledImage's
    "bspline" interpolator (itkMirorrPyramidImplement.txx:409-415).  Axes x,
    y, z in turn; per line c[0 .. N): c *= lambda; causal initial value
    (truncated sum over the horizon, or the mirror-symmetric full sum when
    the line is shorter, z^(N-1) as a product); c[n] += z c[n-1];
    c[N-1] = z / (z^2 - 1) (z c[N-2] + c[N-1]); c[n] = z (c[n+1] - c[n])."""
    c = np.array(data, np.float64)
    z = math.sqrt(3.0) - 2.0
    lam = (1.0 - z) * (1.0 - 1.0 / z)
    iz = 1.0 / z
    anti = z / (z * z - 1.0)
    horizon = int(math.ceil(math.log(1e-10) / math.log(abs(z))))
    for axis in (2, 1, 0):
        a = np.moveaxis(c, axis, 0)
        N = a.shape[0]
        if N == 1:
            continue
        a *= lam
        zn = z
        if horizon < N:
            s = a[0].copy()
            for n in range(1, horizon):
                s = s + zn * a[n]
                zn = zn * z
            a[0] = s
        else:
            z2n = 1.0
            for _ in range(N - 1):
                z2n = z2n * z
            s = a[0] + z2n * a[N - 1]
            z2n = z2n * (z2n * iz)
            for n in range(1, N - 1):
                s = s + (zn + z2n) * a[n]
                zn = zn * z
                z2n = z2n * iz
            a[0] = s / (1.0 - zn * zn)
        for n in range(1, N):
            a[n] = a[n] + z * a[n - 1]
        a[N - 1] = anti * (z * a[N - 2] + a[N - 1])
        for n in range(N - 2, -1, -1):
            a[n] = z * (a[n + 1] - a[n])
    return c


def _mirror(idx, n):
    """Mirror boundary of the B-spline evaluation (period 2N - 2; 0 for N = 1)."""
    if n == 1:
        return np.zeros_like(idx)
    l2 = 2 * n - 2
    idx = np.where(idx < 0, -idx - l2 * ((-idx) // l2), idx - l2 * (idx // l2))
    return np.where(n <= idx, l2 - idx, idx)


def resample_bspline(in_data, out_size, C, e):
    """Final resampling with BSplineInterpolateImageFunction of order 3
    (itkMirorrPyramidImplement.txx:365-479): per axis the support starts at
    floor(c) - 1 with weights, for w = c - floor(c),
    w3 = w^3/6, w0 = 1/6 + w (w - 1)/2 - w3, w2 = w + w0 - 2 w3,
    w1 = 1 - w0 - w2 - w3; the 64 products ((wx wy) wz) coef summed with x
    fastest; 0 outside the buffer; float output."""
    coef = bspline_coefficients(in_data)
    n = (coef.shape[2], coef.shape[1], coef.shape[0])
    c, inside = _index_map(out_size, C, e, n)
    sixth = 1.0 / 6.0
    wt, ix = [], []
    for r in range(3):
        b = np.floor(c[r])
        w = c[r] - b
        b = b.astype(np.int64)
        w3 = ((sixth * w) * w) * w
        w0 = (sixth + (0.5 * w) * (w - 1.0)) - w3
        w2 = (w + w0) - 2.0 * w3
        w1 = ((1.0 - w0) - w2) - w3
        wt.append([w0, w1, w2, w3])
        ix.append([_mirror(b - 1 + k, n[r]) for k in range(4)])
    v = np.zeros(inside.shape, np.float64)
    for kz in range(4):
        for ky in range(4):
            for kx in range(4):
                w = (wt[0][kx] * wt[1][ky]) * wt[2][kz]
                v = v + w * coef[ix[2][kz], ix[1][ky], ix[0][kx]]
    return np.where(inside, v, 0.0).astype(np.float32)


def resample_sinc(in_data, out_size, C, e, radius=5):
    """Final resampling with WindowedSincInterpolateImageFunction (radius 5,
    Welch window, zero-flux Neumann boundary: indices clamp to the image),
    GetInterpolatorFromString's "sinc" (itkMirorrPyramidImplement.txx:416-425).
    Per axis, base floor(c), d = c - floor(c); the 2R taps at offsets
    1-R .. R weigh (1 - x^2/R^2) sin(pi x)/(pi x) for x = d + R - 1 - i
    (a delta at offset 0 when d = 0); the products (((p wx) wy) wz) summed with
    x fastest; 0 outside the buffer; float output."""
    data = np.asarray(in_data, np.float32)
    n = (data.shape[2], data.shape[1], data.shape[0])
    c, inside = _index_map(out_size, C, e, n)
    R, T = radius, 2 * radius
    f = 1.0 / (R * R)
    wt, ix = [], []
    for r in range(3):
        b = np.floor(c[r])
        d = c[r] - b
        b = b.astype(np.int64)
        x = d + float(R)
        ws, xs = [], []
        for i in range(T):
            xs.append(np.clip(b + i - (R - 1), 0, n[r] - 1))
            x = x - 1.0
            welch = 1.0 - (x * f) * x
            px = math.pi * x
            with np.errstate(invalid="ignore", divide="ignore"):
                tap = np.where(x == 0.0, welch, welch * (np.sin(px) / px))
            ws.append(np.where(d == 0.0, 1.0 if i == R - 1 else 0.0, tap))
        wt.append(ws)
        ix.append(xs)
    v = np.zeros(inside.shape, np.float64)
    for kz in range(T):
        for ky in range(T):
            for kx in range(T):
                p = data[ix[2][kz], ix[1][ky], ix[0][kx]].astype(np.float64)
                v = v + ((p * wt[0][kx]) * wt[1][ky]) * wt[2][kz]
    return np.where(inside, v, 0.0).astype(np.float32)


# ---------------------------------------------------------------------------
# ITK transform semantics (restated)
# ---------------------------------------------------------------------------
def euler_zxy_matrix(ax, ay, az):
    """Euler3DTransform::ComputeMatrix with ComputeZYX off: R = Rz * Rx * Ry."""
    cx, sx = math.cos(ax), math.sin(ax)
    cy, sy = math.cos(ay), math.sin(ay)
    cz, sz = math.cos(az), math.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]], dtype=np.float64)
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]], dtype=np.float64)
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]], dtype=np.float64)
    return rz @ rx @ ry


def euler_zxy_angles(m):
    """Euler3DTransform::ComputeMatrixParameters (ComputeZYX off)."""
    ax = math.asin(max(-1.0, min(1.0, m[2, 1])))
    a = math.cos(ax)
    if abs(a) > 0.00005:
        ay = math.atan2(-m[2, 0] / a, m[2, 2] / a)
        az = math.atan2(-m[0, 1] / a, m[1, 1] / a)
    else:
        az = 0.0
        ay = math.atan2(m[1, 0], m[0, 0])
    return ax, ay, az


class NonOrthogonalError(ValueError):
    pass


class Tfm:
    """MatrixOffsetTransformBase restated.  kind: 'rigid' (Euler3DTransform) or
    'affine' (AffineTransform)."""

    def __init__(self, kind="affine"):
        assert kind in ("rigid", "affine")
        self.kind = kind
        self.M = np.eye(3)
        self.off = np.zeros(3)
        self.c = np.zeros(3)
        self.t = np.zeros(3)
        self.angles = np.zeros(3)

    def copy(self):
        o = Tfm(self.kind)
        o.M, o.off, o.c, o.t, o.angles = (self.M.copy(), self.off.copy(), self.c.copy(),
                                           self.t.copy(), self.angles.copy())
        return o

    def create_another(self):
        return Tfm(self.kind)

    # internals ------------------------------------------------------------
    def _compute_offset(self):
        self.off = self.t + self.c - self.M @ self.c

    def _compute_translation(self):
        self.t = self.off - self.c + self.M @ self.c

    def _compute_matrix_parameters(self):
        if self.kind == "rigid":
            self.angles = np.array(euler_zxy_angles(self.M))
            self.M = euler_zxy_matrix(*self.angles)

    # public ---------------------------------------------------------------
    def set_identity(self):
        self.M = np.eye(3)
        self.off = np.zeros(3)
        self.c = np.zeros(3)
        self.t = np.zeros(3)
        self.angles = np.zeros(3)

    def set_center(self, c):
        self.c = np.array(c, dtype=np.float64)
        self._compute_offset()

    def set_translation(self, t):
        self.t = np.array(t, dtype=np.float64)
        self._compute_offset()

    def set_matrix(self, m):
        m = np.array(m, dtype=np.float64)
        if self.kind == "rigid":
            test = m @ m.T
            if np.max(np.abs(test - np.eye(3))) > 1e-10:
                raise NonOrthogonalError("non-orthogonal rotation matrix")
        self.M = m
        self._compute_offset()
        self._compute_matrix_parameters()

    def params(self):
        if self.kind == "rigid":
            return np.concatenate([self.angles, self.t])
        return np.concatenate([self.M.reshape(-1), self.t])

    def set_params(self, p):
        p = np.asarray(p, dtype=np.float64)
        if self.kind == "rigid":
            self.angles = p[:3].copy()
            self.M = euler_zxy_matrix(*self.angles)
            self.t = p[3:6].copy()
        else:
            self.M = p[:9].reshape(3, 3).copy()
            self.t = p[9:12].copy()
        self._compute_offset()

    def compose(self, other: "Tfm", pre: bool = False):
        if pre:
            self.off = self.M @ other.off + self.off
            self.M = self.M @ other.M
        else:
            self.off = other.M @ self.off + other.off
            self.M = other.M @ self.M
        self._compute_translation()
        self._compute_matrix_parameters()

    def inverse(self) -> "Tfm":
        inv = Tfm(self.kind)
        inv.c = self.c.copy()
        mi = np.linalg.inv(self.M)
        inv.M = mi
        inv.off = -(mi @ self.off)
        inv._compute_translation()
        inv._compute_matrix_parameters()
        return inv

    def transform_points(self, pts):
        return pts @ self.M.T + self.off


def set_center_to_origin(t: Tfm):
    """itkTransformUtils.h:22-35."""
    off = t.off.copy()
    t.set_center(np.zeros(3))
    t.set_translation(off)


def update_center(t: Tfm, c2):
    """itkTransformUtils.h:42-57."""
    set_center_to_origin(t)
    t.set_center(-np.asarray(c2))
    off = t.off.copy()
    t.set_center(np.asarray(c2))
    t.set_translation(off)


# ---------------------------------------------------------------------------
# vnl helpers (restated)
# ---------------------------------------------------------------------------
def matrix_sqrt(m, eps=1e-14, max_iter=50):
    """Denman-Beavers iteration, src/mirorr/vnl_utils.h:46-95."""
    y = m.copy()
    z = np.eye(m.shape[0])
    d = np.finfo(np.float64).max
    i = 0
    while d > eps and i < max_iter:
        ny = 0.5 * (y + np.linalg.inv(z))
        nz = 0.5 * (z + np.linalg.inv(y))
        y, z = ny, nz
        i += 1
        d = np.max(np.abs(y @ y - m))
    return y


def orthogonalize(m):
    """U * V^T of the SVD, src/mirorr/vnl_utils.h:124-135."""
    u, _, vt = np.linalg.svd(m)
    return u @ vt


def quat_rotation(q):
    """vnl_quaternion (x, y, z, r): rotation_matrix_transpose().transpose()."""
    x, y, z, r = q
    rt = np.empty((3, 3))
    x2, y2, z2, r2 = x * x, y * y, z * z, r * r
    xy, yz, zx = x * y, y * z, z * x
    rx, ry, rz = r * x, r * y, r * z
    rt[0, 0] = r2 + x2 - y2 - z2
    rt[1, 1] = r2 - x2 + y2 - z2
    rt[2, 2] = r2 - x2 - y2 + z2
    rt[0, 1] = 2 * (xy + rz)
    rt[0, 2] = 2 * (zx - ry)
    rt[1, 2] = 2 * (yz + rx)
    rt[1, 0] = 2 * (xy - rz)
    rt[2, 0] = 2 * (zx + ry)
    rt[2, 1] = 2 * (yz - rx)
    return rt.T


def quat_euler_angles(q):
    """vnl_quaternion::rotation_euler_angles (angles for R = Rz * Ry * Rx)."""
    rt = quat_rotation(q).T  # rotation_matrix_transpose
    xy = math.sqrt(rt[0, 0] ** 2 + rt[0, 1] ** 2)
    if xy > np.finfo(np.float64).eps * 8.0:
        a0 = math.atan2(rt[1, 2], rt[2, 2])
        a1 = math.atan2(-rt[0, 2], xy)
        a2 = math.atan2(rt[0, 1], rt[0, 0])
    else:
        a0 = math.atan2(-rt[2, 1], rt[1, 1])
        a1 = math.atan2(-rt[0, 2], xy)
        a2 = 0.0
    return np.array([a0, a1, a2])


def quat_axis_angle(q):
    imag = np.array(q[:3], dtype=np.float64)
    mag = math.sqrt(float(imag @ imag))
    angle = 2.0 * math.atan2(mag, q[3])
    axis = np.array([0.0, 0.0, 1.0]) if mag == 0.0 else imag / mag
    return axis, angle


def quat_from_axis_angle(axis, angle):
    a = angle * 0.5
    s = math.sin(a)
    return np.array([s * axis[0], s * axis[1], s * axis[2], math.cos(a)])


def horn_quaternion(init_c, moved_c):
    """CalculateRigidQuaternion, itkMirorrRegistrationMethod.txx:1063-1106:
    eigenvector of the smallest eigenvalue of sum Q^T Q, as (x, y, z, r)."""
    a, b = init_c, moved_c
    n = a.shape[0]
    q = np.zeros((n, 4, 4))
    q[:, 0, 1:4] = a - b
    q[:, 1, 2] = -a[:, 2] - b[:, 2]
    q[:, 1, 3] = a[:, 1] + b[:, 1]
    q[:, 2, 3] = -a[:, 0] - b[:, 0]
    q = q - np.transpose(q, (0, 2, 1))
    total = np.einsum("nij,nik->jk", q, q)
    w, v = np.linalg.eigh(total)
    e = v[:, 0]
    return np.array([e[1], e[2], e[3], e[0]])


def covariance(a, b):
    """CovarianceOfPoints(a, b): cov[r][c] = sum b[r] * a[c] / n ... restated with
    the reference's argument naming: first argument is 'initialSubset'."""
    # reference: covariance[row][col] += initialSubset[point][row] * movedSubset[point][col]
    # where (initialSubset, movedSubset) are its two arguments in order.
    return (a.T @ b) / a.shape[0]


def _nth(res, fraction):
    if fraction > 0.99999:
        return float(np.max(res))
    n = res.size
    k = int(fraction * n)
    k = min(k, n - 1)
    return float(np.partition(res, k)[k])


# ---------------------------------------------------------------------------
# LTS fits
# ---------------------------------------------------------------------------
def lts_classic(tfm: Tfm, init_pts, moved_pts, lts_keep=0.5):
    """OptimizeTransform, itkMirorrRegistrationMethod.txx:758-1003.  Updates tfm
    in place (m_Transform->Compose(final, true)); returns inner iterations."""
    final = tfm.create_another()
    rc = tfm.c.copy()
    final.set_identity()
    final.set_center(rc)
    last_params = final.params()
    fraction = 1.0
    last_delta, delta = 0.0, 1.0
    it = -1
    while delta > 1e-3 and it < 100 and abs(delta - last_delta) > 1e-3:
        it += 1
        if init_pts.shape[0] == 0:
            break
        tp = final.transform_points(init_pts)
        res = np.sum((tp - moved_pts) ** 2, axis=1)
        nth = _nth(res, fraction)
        sel = res <= nth
        isub = init_pts[sel]
        msub = moved_pts[sel]
        fraction = lts_keep
        imean = isub.mean(axis=0) if isub.shape[0] else np.zeros(3)
        mmean = msub.mean(axis=0) if msub.shape[0] else np.zeros(3)
        ic = isub - imean
        mc = msub - mmean
        new_params = last_params.copy()
        if tfm.kind == "affine":
            outer_xy = covariance(mc, ic)
            outer_xx = covariance(ic, ic)
            rot = outer_xy.copy()
            if abs(np.linalg.det(outer_xx)) >= 1e-4:
                rot = rot @ np.linalg.inv(outer_xx)
            trans = (mmean - rc) - rot @ (imean - rc)
            new_params[:9] = rot.reshape(-1)
            new_params[9:12] = trans
        else:
            q = horn_quaternion(ic, mc)
            rot = quat_rotation(q)
            trans = (mmean - rc) - rot @ (imean - rc)
            ang = quat_euler_angles(q)
            new_params[:3] = ang
            new_params[3:6] = trans
        last_delta = delta
        delta = float(np.sum((last_params - new_params) ** 2))
        rc = imean.copy()
        final.set_center(rc)
        final.set_params(new_params)
    tfm.compose(final, pre=True)
    return it + 1


def compute_half_space(t: Tfm):
    """ComputeHalfSpaceTransforms, itkSymMirorrRegistrationMethod.txx:139-201."""
    m = np.eye(4)
    m[:3, :3] = t.M
    m[:3, 3] = t.t
    m12 = matrix_sqrt(m)
    im12 = matrix_sqrt(np.linalg.inv(m))
    f = t.create_another()
    b = t.create_another()
    f.set_matrix(m12[:3, :3])
    b.set_matrix(im12[:3, :3])
    f.set_translation(m12[:3, 3])
    b.set_translation(im12[:3, 3])
    return f, b


def _half_step(K, trans):
    m = np.eye(4)
    m[:3, :3] = K
    m[:3, 3] = trans
    return matrix_sqrt(m)


def lts_symmetric(tfm: Tfm, t12f: Tfm, t12b: Tfm, init_pts, moved_pts, lts_keep=0.5):
    """OptimizeTransform(t12F, t12B), itkSymMirorrRegistrationMethod.txx:729-1442.
    Updates t12f, t12b and tfm in place."""
    rc = tfm.c.copy()
    ff = tfm.create_another()
    fb = tfm.create_another()
    ff.set_identity(); ff.set_center(rc)
    fb.set_identity(); fb.set_center(rc)
    last_params = ff.params()
    fraction = 1.0
    last_delta, delta = 0.0, 1.0
    it = -1
    while delta > 1e-3 and it < 100 and abs(delta - last_delta) > 1e-3:
        it += 1
        if init_pts.shape[0] == 0:
            break
        res = np.sum((ff.transform_points(init_pts) - fb.transform_points(moved_pts)) ** 2, axis=1)
        nth = _nth(res, fraction)
        sel = res <= nth
        isub = init_pts[sel]
        msub = moved_pts[sel]
        fraction = lts_keep
        imean = isub.mean(axis=0)
        mmean = msub.mean(axis=0)
        ic = isub - imean
        mc = msub - mmean
        new_params = last_params.copy()
        if tfm.kind == "affine":
            outer_xy = covariance(mc, ic)
            outer_xx = covariance(ic, ic)
            rot_f = outer_xy.copy()
            if abs(np.linalg.det(outer_xx)) >= 1e-4:
                rot_f = rot_f @ np.linalg.inv(outer_xx)
            outer_xy = covariance(ic, mc)
            outer_xx = covariance(mc, mc)
            rot_b = outer_xy.copy()
            if abs(np.linalg.det(outer_xx)) >= 1e-4:
                rot_b = rot_b @ np.linalg.inv(outer_xx)
            translation = mmean - imean
            new_params[:9] = rot_f.reshape(-1)
            new_params[9:12] = translation
            pf = np.concatenate([rot_f.reshape(-1), translation])
            pb = np.concatenate([rot_b.reshape(-1), -translation])
            ff.set_center(imean); ff.set_params(pf)
            fb.set_center(mmean); fb.set_params(pb)
            K = (ff.M + np.linalg.inv(fb.M)) / 2.0
            Mb = (np.linalg.inv(ff.M) + fb.M) / 2.0
            ff.set_matrix(K)
            fb.set_matrix(Mb)
        else:
            q = horn_quaternion(ic, mc)
            ang = quat_euler_angles(q)
            axis, angle = quat_axis_angle(q)
            ang_f = quat_euler_angles(quat_from_axis_angle(axis, angle))
            ang_b = quat_euler_angles(quat_from_axis_angle(axis, -angle))
            translation = mmean - imean
            new_params[:3] = ang
            new_params[3:6] = translation
            ff.set_center(imean); ff.set_params(np.concatenate([ang_f, translation]))
            fb.set_center(mmean); fb.set_params(np.concatenate([ang_b, -translation]))
            K = orthogonalize((ff.M + np.linalg.inv(fb.M)) / 2.0)
            ff.set_matrix(K)
            fb.set_matrix(K.T)
        off_f = ff.off.copy()
        off_b = fb.off.copy()
        ff.set_center(np.zeros(3)); fb.set_center(np.zeros(3))
        ff.set_translation(off_f); fb.set_translation(off_b)
        i_f = ff.inverse()
        i_b = fb.inverse()
        Kf = (ff.M + i_b.M) / 2.0
        Kb = (i_f.M + fb.M) / 2.0
        if tfm.kind == "rigid":
            Kf = orthogonalize(Kf)
            Kb = orthogonalize(Kb)
        m12 = _half_step(Kf, (ff.t + i_b.t) / 2.0)
        im12 = _half_step(Kb, (i_f.t + fb.t) / 2.0)
        try:
            ff.set_matrix(m12[:3, :3])
            fb.set_matrix(im12[:3, :3])
        except NonOrthogonalError:
            ff.set_matrix(orthogonalize(m12[:3, :3]))
            fb.set_matrix(orthogonalize(im12[:3, :3]))
        ff.set_translation(m12[:3, 3])
        fb.set_translation(im12[:3, 3])
        last_delta = delta
        delta = float(np.sum((last_params - new_params) ** 2))
        last_params = new_params.copy()
    t12f.compose(ff, pre=True)
    t12b.compose(fb, pre=True)
    inv_b = t12b.inverse()
    tfm.set_identity()
    tfm.compose(inv_b, pre=True)
    tfm.compose(t12f, pre=False)
    return it + 1


# ---------------------------------------------------------------------------
# Middle space
# ---------------------------------------------------------------------------
def middle_space_classic(fixed: Image, moving: Image):
    """itkMirorrRegistrationMethod.txx:496-514 (EResamplingMiddle)."""
    cf, cm = fixed.center(), moving.center()
    origin = cm + ((fixed.origin - cf) + (moving.origin - cm)) / 2.0
    spacing = (fixed.spacing + moving.spacing) / 2.0
    size = tuple(int((a + b + 0.5) / 2) for a, b in zip(fixed.size, moving.size))
    return origin, spacing, size


def middle_space_symmetric(fixed: Image, moving: Image):
    """itkSymMirorrRegistrationMethod.txx:264-284 (EResamplingMiddle)."""
    cf, cm = fixed.center(), moving.center()
    origin = ((fixed.origin - cf) + (moving.origin - cm)) / 2.0
    spacing = (fixed.spacing + moving.spacing) / 2.0
    size = tuple(int((a + b + 0.5) / 2) for a, b in zip(fixed.size, moving.size))
    return origin, spacing, size


def _grid_image(origin, spacing, direction, size):
    return Image(np.zeros((size[2], size[1], size[0]), np.float32), np.array(spacing, np.float64),
                 np.array(origin, np.float64), np.array(direction, np.float64))


def round_storage(a, store):
    """float32 values as a 16-bit storage type keeps them: round to nearest
    even into bfloat16 ('bf16') or IEEE half ('f16') and back to float32;
    None or 'f32' returns the array unchanged."""
    if store is None or store == "f32":
        return a
    a = np.ascontiguousarray(a, np.float32)
    if store == "f16":
        return a.astype(np.float16).astype(np.float32)
    if store == "bf16":
        u = a.view(np.uint32).astype(np.uint64)
        r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
        return r.astype(np.uint32).view(np.float32)
    raise ValueError(f"unknown storage type {store!r}")


def _resample_through(src: Image, src_mask, grid: Image, t: Tfm, mask_geom: Image | None,
                      store=None):
    C, e = resample_map(grid, src, t.M, t.off)
    img, _ = resample(src.data, None, grid.size, C, e)
    img = round_storage(img, store)
    mg = mask_geom if mask_geom is not None else src
    if src_mask is None:
        src_mask = np.full(mg.data.shape, 255, np.uint8)
    Cm, em = resample_map(grid, mg, t.M, t.off)
    _, m = resample(None, src_mask, grid.size, Cm, em)
    return img, m


# ---------------------------------------------------------------------------
# Registration drivers
# ---------------------------------------------------------------------------
@dataclass
class RegParams:
    mode: str = "symmetric"          # 'classic' | 'symmetric'
    kind: str = "rigid"              # 'rigid' | 'affine'
    iterations: int = 5
    bm: BMParams = field(default_factory=lambda: BMParams(4, 1, 3, 7, 1.0))
    lts_keep: float = 0.5
    store: str | None = None         # None/'f32' or the 16-bit storage 'bf16' | 'f16'


def classic_level(fixed: Image, moving: Image, fmask, mmask, fmask_geom, mmask_geom,
                  tfm: Tfm, rp: RegParams, threads=0, trace=None):
    """StartOptimization, itkMirorrRegistrationMethod.txx:422-659 (middle space)."""
    origin, spacing, size = middle_space_classic(fixed, moving)
    grid_f = _grid_image(origin, spacing, fixed.direction, size)
    grid_m = _grid_image(origin, spacing, moving.direction, size)
    ident = Tfm("affine")
    mov_img, mov_mask = _resample_through(moving, mmask, grid_m, ident, mmask_geom, rp.store)
    base = geometry_like(grid_m, mov_img)
    last = tfm.params()
    for it in range(abs(rp.iterations)):
        fix_img, fix_mask = _resample_through(fixed, fmask, grid_f, tfm, fmask_geom, rp.store)
        search = geometry_like(grid_f, fix_img)
        bp, mp = get_offsets(base, search, mov_mask, fix_mask, rp.bm, threads)
        lts_classic(tfm, bp, mp, rp.lts_keep)
        p = tfm.params()
        d = float(np.sum((last - p) ** 2))
        if trace is not None:
            trace.append(dict(iteration=it, n_points=bp.shape[0], params=p.copy(), delta=d))
        last = p
        if d < 1e-3:
            break
    return tfm


def symmetric_level(fixed: Image, moving: Image, fmask, mmask, fmask_geom, mmask_geom,
                    tfm: Tfm, rp: RegParams, threads=0, trace=None):
    """StartOptimization, itkSymMirorrRegistrationMethod.txx:238-720."""
    cf, cm = fixed.center(), moving.center()
    origin, spacing, size = middle_space_symmetric(fixed, moving)
    grid_f = _grid_image(origin, spacing, fixed.direction, size)
    grid_m = _grid_image(origin, spacing, moving.direction, size)
    initial_center = tfm.c.copy()
    set_center_to_origin(tfm)
    fixed_tr = Tfm("rigid"); fixed_tr.set_params([0, 0, 0, *cf])
    moving_tr = Tfm("rigid"); moving_tr.set_params([0, 0, 0, *cm])
    tfm.compose(fixed_tr.inverse(), pre=False)
    tfm.compose(moving_tr, pre=True)
    t12f, t12b = compute_half_space(tfm)
    last = tfm.params()

    def centered():
        cF = tfm.create_another(); cF.set_params(t12f.params()); cF.compose(fixed_tr, pre=False)
        cB = tfm.create_another(); cB.set_params(t12b.params()); cB.compose(moving_tr, pre=False)
        return cF, cB

    for it in range(abs(rp.iterations)):
        cF, cB = centered()
        mov_img, mov_mask = _resample_through(moving, mmask, grid_m, cB, mmask_geom, rp.store)
        fix_img, fix_mask = _resample_through(fixed, fmask, grid_f, cF, fmask_geom, rp.store)
        base = geometry_like(grid_m, mov_img)
        search = geometry_like(grid_f, fix_img)
        bp1, mp1 = get_offsets(base, search, mov_mask, fix_mask, rp.bm, threads)
        bp2, mp2 = get_offsets(search, base, fix_mask, mov_mask, rp.bm, threads)
        init = np.concatenate([bp1, mp2])
        moved = np.concatenate([mp1, bp2])
        lts_symmetric(tfm, t12f, t12b, init, moved, rp.lts_keep)
        p = tfm.params()
        d = float(np.sum((last - p) ** 2))
        if trace is not None:
            trace.append(dict(iteration=it, n_points=init.shape[0], params=p.copy(), delta=d))
        last = p
        if d < 1e-3:
            break
    cF, cB = centered()
    inv_b = cB.inverse()
    tfm.set_identity()
    tfm.compose(inv_b, pre=True)
    tfm.compose(cF, pre=False)
    update_center(tfm, initial_center)
    return tfm


# ---------------------------------------------------------------------------
# Pyramid (this project's own spec; see module docstring)
# ---------------------------------------------------------------------------
def _num_octaves(dim, base):
    return math.floor(math.log(dim / base) / math.log(2.0))


def _num_levels(dim, base):
    return 1 + int(max(0.0, _num_octaves(dim, base)))


def _best_rate(big, small):
    e = int(max(0.0, _num_octaves(big * 4.0 / 3.0, small)))
    return 2 ** e


def pyramid_schedule(fixed_size, moving_size, fixed_spacing, moving_spacing, min_length=32,
                     max_levels=1024):
    """PyramidScheduleTuner::UpdateSymmetric, itkPyramidScheduleTuner.txx:291-414.
    Returns (moving_schedule, fixed_schedule), coarsest level first."""
    lm = max(moving_size)
    lf = max(fixed_size)
    mpl = 1 + max(_num_levels(lm, min_length), _num_levels(lf, min_length))
    sm = np.full((mpl, 3), -1, dtype=np.int64)
    sf = np.full((mpl, 3), -1, dtype=np.int64)
    for d in range(3):
        r = 1
        sm[mpl - r, d] = 1
        sf[mpl - r, d] = 1
        mb, fb = moving_spacing[d], fixed_spacing[d]
        me = 2 ** (_num_levels(moving_size[d], min_length) - 1)
        fe = 2 ** (_num_levels(fixed_size[d], min_length) - 1)
        r = 2
        if mb < fb:
            rate = min(_best_rate(fb, mb), me)
            s = 2 if rate >= 2 else 1
            while s <= rate:
                sm[mpl - r, d] = s; sf[mpl - r, d] = 1; r += 1; s *= 2
        elif mb > fb:
            rate = min(_best_rate(mb, fb), fe)
            s = 2 if rate >= 2 else 1
            while s <= rate:
                sm[mpl - r, d] = 1; sf[mpl - r, d] = s; r += 1; s *= 2
        else:
            sm[mpl - r, d] = 1; sf[mpl - r, d] = 1; r += 1
        for lev in range(mpl - r, -1, -1):
            if 2 * sm[lev + 1, d] > me or 2 * sf[lev + 1, d] > fe:
                sm[lev, d] = sm[lev + 1, d]; sf[lev, d] = sf[lev + 1, d]
            else:
                sm[lev, d] = 2 * sm[lev + 1, d]; sf[lev, d] = 2 * sf[lev + 1, d]
    first = 0
    nd = sum(int(sm[mpl - 1, d] != sm[mpl - 2, d]) + int(sf[mpl - 1, d] != sf[mpl - 2, d])
             for d in range(3))
    if nd == 0:
        first = 1
    last = mpl
    for lev in range(2, mpl):
        nd = sum(int(sm[mpl - lev - 1, d] != sm[mpl - lev, d]) +
                 int(sf[mpl - lev - 1, d] != sf[mpl - lev, d]) for d in range(3))
        if nd < 3:
            last = lev
            break
    n = min(last - first, max_levels)
    out_m = np.zeros((n, 3), np.int64)
    out_f = np.zeros((n, 3), np.int64)
    for lev in range(n):
        out_m[n - lev - 1] = sm[mpl - first - lev - 1]
        out_f[n - lev - 1] = sf[mpl - first - lev - 1]
    return out_m, out_f


def gaussian_weights(factor):
    """Discrete Gaussian of sigma = factor / 2 voxels, radius ceil(3 sigma),
    normalised by the sequential sum of its taps (FP64, libm exp)."""
    if factor <= 1:
        return np.array([1.0])
    sigma = factor / 2.0
    r = int(math.ceil(3.0 * sigma))
    w = [math.exp(-(float(k) * float(k)) / (2.0 * sigma * sigma)) for k in range(-r, r + 1)]
    s = 0.0
    for v in w:
        s += v
    return np.array([v / s for v in w], dtype=np.float64)


def smooth_axis(vol: np.ndarray, w: np.ndarray, axis: int) -> np.ndarray:
    """One separable pass, clamp-to-edge, FP64 accumulation in tap order, float output."""
    if w.size == 1:
        return vol.astype(np.float32)
    r = w.size // 2
    n = vol.shape[axis]
    acc = np.zeros(vol.shape, np.float64)
    idx = np.arange(n)
    for t in range(w.size):
        src = np.clip(idx + t - r, 0, n - 1)
        acc = acc + w[t] * np.take(vol, src, axis=axis).astype(np.float64)
    return acc.astype(np.float32)


def pyramid_level(img: Image, factors) -> Image:
    """Smooth (x, then y, then z) and decimate by `factors` (fx, fy, fz)."""
    v = img.data
    v = smooth_axis(v, gaussian_weights(int(factors[0])), 2)
    v = smooth_axis(v, gaussian_weights(int(factors[1])), 1)
    v = smooth_axis(v, gaussian_weights(int(factors[2])), 0)
    f = np.array(factors, dtype=np.float64)
    size = tuple(max(1, int(math.floor(s / fi))) for s, fi in zip(img.size, f))
    spacing = img.spacing * f
    origin = img.origin + img.direction @ ((spacing - img.spacing) * 0.5)
    C = np.diag(f)
    e = (f - 1.0) / 2.0
    out, _ = resample(v, None, size, C, e)
    return Image(out, spacing, origin, img.direction.copy())


# ---------------------------------------------------------------------------
# Full registration
# ---------------------------------------------------------------------------
def centered_initial_transform(fixed: Image, moving: Image, kind: str) -> Tfm:
    """CenteredTransformInitializer with GeometryOn, as wired in
    itkMirorrPyramidWrapper.txx:611-623 (fixed <- moving image, moving <- fixed)."""
    t = Tfm(kind)
    t.set_identity()
    cm = moving.center()
    cf = fixed.center()
    t.set_center(cm)
    t.set_translation(cf - cm)
    return t


def register(fixed: Image, moving: Image, rp: RegParams, levels: int, fixed_mask=None,
             moving_mask=None, min_length=32, threads=0, init: Tfm | None = None, trace=None):
    """RunMirorr (itkMirorrPyramidImplement.txx:71-158) over the `levels` finest
    pyramid levels (reference CLI: --pyr-num levels --pyr-end 0).  With
    rp.store set, the input images are taken as stored in that 16-bit type
    and every middle-space image is rounded to it, as the 16-bit device path
    stores them (pyramid levels above the finest stay float32)."""
    if rp.store not in (None, "f32"):
        fixed = geometry_like(fixed, round_storage(fixed.data, rp.store))
        moving = geometry_like(moving, round_storage(moving.data, rp.store))
    sm, sf = pyramid_schedule(fixed.size, moving.size, fixed.spacing, moving.spacing, min_length,
                              levels)
    tfm = init.copy() if init is not None else centered_initial_transform(fixed, moving, rp.kind)
    params = tfm.params()
    for lev in range(sm.shape[0]):
        fl = pyramid_level(fixed, sf[lev])
        ml = pyramid_level(moving, sm[lev])
        tfm.set_params(params)
        tr = [] if trace is not None else None
        if rp.mode == "classic":
            classic_level(fl, ml, fixed_mask, moving_mask, fixed, moving, tfm, rp, threads, tr)
        else:
            symmetric_level(fl, ml, fixed_mask, moving_mask, fixed, moving, tfm, rp, threads, tr)
        params = tfm.params()
        if trace is not None:
            trace.append(dict(level=lev, schedule_fixed=sf[lev].tolist(),
                              schedule_moving=sm[lev].tolist(), iterations=tr))
    tfm.set_params(params)
    return tfm
