"""mirorr_b200 -- B200-native block-matching registration (Mirorr's hot path).

Python binding of the C ABI in include/mirorr_b200.h (libmirorr_b200.so,
built in tree by mirorr_b200/build.py).  The classes mirror the reference's
interfaces:

* BlockMatcher   -- itk::AbstractBlockMatcher (src/mirorr/itkAbstractBlockMatcher.h):
  SetBaseImage / SetSearchImage / SetBaseMask / SetSearchMask / parameter
  setters / SwapImageOrder / GetOffsets.
* register()     -- MirorrPyramidImplement::RunMirorr with the classic or
  symmetric method (the `mirorr` CLI's --reg-mode, -t, -n, --pyr-*, block
  options).
* resample(), lts_classic(), lts_symmetric() -- the resampler and
  OptimizeTransform stages on their own.

There is no CPU fallback: without the CUDA library or a B200 every call raises
MirorrError.
"""
from __future__ import annotations

import atexit
import ctypes
import os
import sys
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmirorr_b200.so")

STATUS = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ENOBLOCKS", 4: "ECUDA", 5: "ETIMEOUT",
          6: "ESTATE", 7: "ERANGE", 8: "EBUSY"}
RIGID, AFFINE = 0, 1


class MirorrError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


class Geometry(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int32 * 3), ("spacing", ctypes.c_double * 3),
                ("origin", ctypes.c_double * 3), ("direction", ctypes.c_double * 9)]

    @staticmethod
    def make(size_xyz, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), direction=None):
        g = Geometry()
        g.size[:] = [int(v) for v in size_xyz]
        g.spacing[:] = [float(v) for v in spacing]
        g.origin[:] = [float(v) for v in origin]
        d = np.eye(3) if direction is None else np.asarray(direction, np.float64)
        g.direction[:] = [float(v) for v in d.reshape(-1)]
        return g

    @staticmethod
    def of(data: np.ndarray, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), direction=None):
        nz, ny, nx = data.shape
        return Geometry.make((nx, ny, nz), spacing, origin, direction)

    def as_dict(self):
        return dict(size=tuple(self.size), spacing=tuple(self.spacing), origin=tuple(self.origin),
                    direction=np.array(self.direction).reshape(3, 3))


class BMParams(ctypes.Structure):
    _fields_ = [("block_width", ctypes.c_uint32), ("block_gap", ctypes.c_uint32),
                ("nhood_gap", ctypes.c_uint32), ("nhood_width", ctypes.c_uint32),
                ("portion_matches_kept", ctypes.c_double), ("block_keep", ctypes.c_double),
                ("verbosity", ctypes.c_int32)]


class Transform(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("matrix", ctypes.c_double * 9),
                ("offset", ctypes.c_double * 3), ("center", ctypes.c_double * 3),
                ("params", ctypes.c_double * 12)]

    @staticmethod
    def make(kind, params, center=(0.0, 0.0, 0.0)):
        t = Transform()
        t.kind = int(kind)
        p = list(params) + [0.0] * (12 - len(params))
        t.params[:] = [float(v) for v in p]
        t.center[:] = [float(v) for v in center]
        return t

    @property
    def M(self):
        return np.array(self.matrix).reshape(3, 3)

    @property
    def off(self):
        return np.array(self.offset)

    def param_vector(self):
        n = 6 if self.kind == RIGID else 12
        return np.array(self.params[:n])


class RegParams(ctypes.Structure):
    _fields_ = [("symmetric", ctypes.c_int32), ("kind", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("iterations", ctypes.c_int32), ("min_length", ctypes.c_int32), ("bm", BMParams),
                ("lts_keep", ctypes.c_double), ("verbosity", ctypes.c_int32),
                ("last_level", ctypes.c_int32), ("storage", ctypes.c_int32)]


# element types of stored volumes (mirorr_dtype)
F32, BF16, F16 = 0, 1, 2
_DTYPES = {"f32": F32, "float32": F32, "bf16": BF16, "bfloat16": BF16, "f16": F16, "float16": F16}


def dtype_code(d) -> int:
    if isinstance(d, int):
        return d
    return _DTYPES[str(d).lower()]


def to_storage(a, dtype):
    """float32 array -> its 16-bit storage bit patterns (uint16, round to
    nearest even), as the library's conversion does; float32 arrays pass
    through for F32."""
    d = dtype_code(dtype)
    a = np.ascontiguousarray(a, np.float32)
    if d == F32:
        return a
    if d == F16:
        return a.astype(np.float16).view(np.uint16)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_storage(bits, dtype):
    """16-bit storage bit patterns -> float32 values."""
    d = dtype_code(dtype)
    if d == F32:
        return np.ascontiguousarray(bits, np.float32)
    b = np.ascontiguousarray(bits, np.uint16)
    if d == F16:
        return b.view(np.float16).astype(np.float32)
    return (b.astype(np.uint32) << 16).view(np.float32)


class RegStats(ctypes.Structure):
    _fields_ = [("levels_run", ctypes.c_int32), ("iterations_run", ctypes.c_int32 * 16),
                ("block_ncc_evaluated", ctypes.c_int64), ("matcher_calls", ctypes.c_int64),
                ("seconds", ctypes.c_double), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64)]


_lib = None
_live_matchers = weakref.WeakSet()
_live_contexts = weakref.WeakSet()


@atexit.register
def _close_all():
    for m in list(_live_matchers):
        m.close()
    for c in list(_live_contexts):
        c.close()


def lib():
    """Loads libmirorr_b200.so; raises MirorrError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MirorrError(4, f"CUDA library not built: {LIB_PATH} (run mirorr_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sigs = {
        "mirorr_ctx_create": [ctypes.c_int32, P(vp)],
        "mirorr_ctx_destroy": [vp],
        "mirorr_bm_create": [vp, P(vp)],
        "mirorr_bm_destroy": [vp],
        "mirorr_bm_default_params": [P(BMParams)],
        "mirorr_bm_set_params": [vp, P(BMParams)],
        "mirorr_bm_set_metric": [vp, ctypes.c_char_p],
        "mirorr_bm_set_base_image": [vp, P(Geometry), vp],
        "mirorr_bm_set_search_image": [vp, P(Geometry), vp],
        "mirorr_bm_set_base_mask": [vp, vp],
        "mirorr_bm_set_search_mask": [vp, vp],
        "mirorr_bm_set_base_image_device": [vp, P(Geometry), vp],
        "mirorr_bm_set_search_image_device": [vp, P(Geometry), vp],
        "mirorr_bm_set_base_mask_device": [vp, vp],
        "mirorr_bm_set_search_mask_device": [vp, vp],
        "mirorr_bm_swap_image_order": [vp],
        "mirorr_bm_set_storage": [vp, ctypes.c_int32],
        "mirorr_bm_set_base_image_device16": [vp, P(Geometry), vp],
        "mirorr_bm_set_search_image_device16": [vp, P(Geometry), vp],
        "mirorr_bm_grid": [vp, vp, vp],
        "mirorr_bm_get_offsets": [vp, ctypes.c_size_t, vp, vp, P(ctypes.c_size_t)],
        "mirorr_bm_block_results": [vp, ctypes.c_size_t, vp, vp, vp, vp, P(ctypes.c_size_t)],
        "mirorr_bm_last_timings": [vp, vp],
        "mirorr_bm_last_diagnostics": [vp, vp],
        "mirorr_resample": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "mirorr_resample_map": [P(Geometry), P(Geometry), vp, vp, vp, vp],
        "mirorr_resample_nearest": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "mirorr_resample_bspline": [vp, vp, vp, vp, vp, vp, vp],
        "mirorr_resample_device": [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int32],
        "mirorr_resample_sinc": [vp, vp, vp, vp, vp, vp, vp],
        "mirorr_lts_classic": [vp, P(Transform), ctypes.c_size_t, vp, vp, ctypes.c_double,
                               P(ctypes.c_int32)],
        "mirorr_lts_symmetric": [vp, P(Transform), P(Transform), P(Transform), ctypes.c_size_t,
                                 vp, vp, ctypes.c_double, P(ctypes.c_int32)],
        "mirorr_lts_noalloc": [vp, P(Transform), vp, vp, ctypes.c_size_t, vp, vp,
                               ctypes.c_double, P(ctypes.c_int32)],
        "mirorr_reg_default_params": [P(RegParams)],
        "mirorr_register": [vp, P(Geometry), vp, vp, P(Geometry), vp, vp, P(RegParams),
                            P(Transform), P(Transform), P(RegStats)],
        "mirorr_register_device": [vp, P(Geometry), vp, vp, P(Geometry), vp, vp, P(RegParams),
                                   P(Transform), P(Transform), P(RegStats)],
        "mirorr_pyramid_schedule": [P(Geometry), P(Geometry), ctypes.c_int32, ctypes.c_int32,
                                    P(ctypes.c_int32), vp, vp],
        "mirorr_pyramid_level": [vp, P(Geometry), vp, vp, P(Geometry), vp, ctypes.c_size_t],
        "mirorr_batch_create": [vp, ctypes.c_int32, ctypes.c_uint64, P(vp)],
        "mirorr_batch_destroy": [vp],
        "mirorr_batch_submit": [vp, P(Geometry), vp, vp, P(Geometry), vp, vp, P(RegParams),
                                P(Transform), P(ctypes.c_int64)],
        "mirorr_batch_step": [vp, P(ctypes.c_int32), P(ctypes.c_int32)],
        "mirorr_batch_run": [vp],
        "mirorr_batch_poll": [vp, vp, ctypes.c_int32, P(ctypes.c_int32)],
        "mirorr_batch_result": [vp, ctypes.c_int64, P(Transform), P(RegStats)],
        "mirorr_batch_cancel": [vp, ctypes.c_int64],
        "mirorr_batch_info": [vp, vp],
        "mirorr_batch_set_graphs": [vp, ctypes.c_int32],
        "mirorr_batch_times": [vp, vp],
        "mirorr_ctx_set_graphs": [vp, ctypes.c_int32],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = st
    L.mirorr_last_error.restype = ctypes.c_char_p
    L.mirorr_last_error.argtypes = []
    L.mirorr_abi_version.restype = ctypes.c_int32
    L.mirorr_ctx_kernel_launches.restype = ctypes.c_int64
    L.mirorr_ctx_kernel_launches.argtypes = [vp]
    L.mirorr_ctx_stream.restype = vp
    L.mirorr_ctx_stream.argtypes = [vp]
    L.mirorr_ctx_set_profiling.restype = st
    L.mirorr_ctx_set_profiling.argtypes = [vp, ctypes.c_int32]
    L.mirorr_ctx_stage_times.restype = st
    L.mirorr_ctx_stage_times.argtypes = [vp, vp, P(ctypes.c_int64)]
    L.mirorr_ctx_search_kernel_times.restype = st
    L.mirorr_ctx_search_kernel_times.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_int64),
                                                 P(ctypes.c_int64)]
    L.mirorr_ctx_resample_times.restype = st
    L.mirorr_ctx_resample_times.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_int64),
                                            P(ctypes.c_int64)]
    L.mirorr_ctx_set_wait_limit.restype = st
    L.mirorr_ctx_set_wait_limit.argtypes = [vp, ctypes.c_int64]
    _lib = L
    return L


def _check(status):
    if status != 0:
        msg = lib().mirorr_last_error().decode(errors="replace")
        raise MirorrError(status, msg)


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


class Context:
    """A CUDA device + stream + scratch memory (mirorr_ctx)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().mirorr_ctx_create(int(device), ctypes.byref(self._h)))
        _live_contexts.add(self)

    @property
    def handle(self):
        return self._h

    def kernel_launches(self) -> int:
        return int(lib().mirorr_ctx_kernel_launches(self._h))

    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer."""
        return int(lib().mirorr_ctx_stream(self._h) or 0)

    def set_profiling(self, on: bool):
        _check(lib().mirorr_ctx_set_profiling(self._h, 1 if on else 0))

    def set_graphs(self, on: bool):
        """Iteration graphs of float32 registrations on (default) or off."""
        _check(lib().mirorr_ctx_set_graphs(self._h, 1 if on else 0))

    def stage_times(self):
        """(ms[box_stats, selection, ncc, postfilter], matcher calls) since the last read."""
        ms = np.zeros(4, np.float64)
        calls = ctypes.c_int64(0)
        _check(lib().mirorr_ctx_stage_times(self._h, _ptr(ms), ctypes.byref(calls)))
        return ms, calls.value

    def search_kernel_times(self):
        """(ms, launches, candidates) of the per-x-lane FP32 search kernel since
        the last read (profiling on)."""
        ms = ctypes.c_double(0.0)
        launches = ctypes.c_int64(0)
        cands = ctypes.c_int64(0)
        _check(lib().mirorr_ctx_search_kernel_times(self._h, ctypes.byref(ms), ctypes.byref(launches),
                                                    ctypes.byref(cands)))
        return ms.value, launches.value, cands.value

    def resample_times(self):
        """(ms, passes, output voxels) of the registrations' resampling passes
        since the last read (profiling on)."""
        ms = ctypes.c_double(0.0)
        passes = ctypes.c_int64(0)
        voxels = ctypes.c_int64(0)
        _check(lib().mirorr_ctx_resample_times(self._h, ctypes.byref(ms), ctypes.byref(passes),
                                               ctypes.byref(voxels)))
        return ms.value, passes.value, voxels.value

    def set_wait_limit(self, polls: int):
        """Polls of an LTS grid-barrier wait before it gives up (0: the default)."""
        _check(lib().mirorr_ctx_set_wait_limit(self._h, int(polls)))

    def close(self):
        if self._h:
            for m in list(_live_matchers):
                if m.ctx is self:
                    m.close()
            lib().mirorr_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if sys.is_finalizing():
                return
            self.close()
        except Exception:
            pass


class BlockMatcher:
    """Drop-in for itk::AbstractBlockMatcher (GPU implementation)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        _check(lib().mirorr_bm_create(ctx.handle, ctypes.byref(self._h)))
        self._p = BMParams()
        _check(lib().mirorr_bm_default_params(ctypes.byref(self._p)))
        _live_matchers.add(self)

    # parameters (itkAbstractBlockMatcher.h:101-127)
    def _apply(self):
        _check(lib().mirorr_bm_set_params(self._h, ctypes.byref(self._p)))

    def SetBlockWidth(self, v):
        self._p.block_width = int(v); self._apply()

    def SetBlockGap(self, v):
        self._p.block_gap = int(v); self._apply()

    def SetNhoodGap(self, v):
        self._p.nhood_gap = int(v); self._apply()

    def SetNhoodWidth(self, v):
        self._p.nhood_width = int(v); self._apply()

    def SetPortionMatchesKept(self, v):
        old = self._p.portion_matches_kept
        self._p.portion_matches_kept = float(v)
        try:
            self._apply()
        except MirorrError:
            self._p.portion_matches_kept = old
            raise

    def SetBlockKeep(self, v):
        self._p.block_keep = float(v); self._apply()

    def SetVerbosity(self, v):
        self._p.verbosity = int(v); self._apply()

    def SetBlockMetricType(self, name: str):
        _check(lib().mirorr_bm_set_metric(self._h, name.encode()))

    def GetBlockWidth(self):
        return self._p.block_width

    def GetNhoodGap(self):
        return self._p.nhood_gap

    def GetPortionMatchesKept(self):
        return self._p.portion_matches_kept

    # images
    def SetBaseImage(self, data, spacing=(1, 1, 1), origin=(0, 0, 0), direction=None):
        d = _f32(data)
        _check(lib().mirorr_bm_set_base_image(self._h, ctypes.byref(Geometry.of(d, spacing, origin, direction)), _ptr(d)))

    def SetSearchImage(self, data, spacing=(1, 1, 1), origin=(0, 0, 0), direction=None):
        d = _f32(data)
        _check(lib().mirorr_bm_set_search_image(self._h, ctypes.byref(Geometry.of(d, spacing, origin, direction)), _ptr(d)))

    def SetBaseMask(self, mask):
        _check(lib().mirorr_bm_set_base_mask(self._h, _ptr(_u8(mask))))

    def SetSearchMask(self, mask):
        _check(lib().mirorr_bm_set_search_mask(self._h, _ptr(_u8(mask))))

    def SetBaseImageDevice(self, geom: Geometry, dev_ptr: int):
        _check(lib().mirorr_bm_set_base_image_device(self._h, ctypes.byref(geom), ctypes.c_void_p(dev_ptr)))

    def SetSearchImageDevice(self, geom: Geometry, dev_ptr: int):
        _check(lib().mirorr_bm_set_search_image_device(self._h, ctypes.byref(geom), ctypes.c_void_p(dev_ptr)))

    def SetBaseMaskDevice(self, dev_ptr):
        _check(lib().mirorr_bm_set_base_mask_device(self._h, ctypes.c_void_p(dev_ptr) if dev_ptr else None))

    def SetSearchMaskDevice(self, dev_ptr):
        _check(lib().mirorr_bm_set_search_mask_device(self._h, ctypes.c_void_p(dev_ptr) if dev_ptr else None))

    def SetStorage(self, dtype):
        """Element type of the stored images: "f32" (default), "bf16" or "f16"
        (no reference counterpart); set it before the images."""
        _check(lib().mirorr_bm_set_storage(self._h, dtype_code(dtype)))

    def SetBaseImageDevice16(self, geom: Geometry, dev_ptr: int):
        _check(lib().mirorr_bm_set_base_image_device16(self._h, ctypes.byref(geom),
                                                       ctypes.c_void_p(dev_ptr)))

    def SetSearchImageDevice16(self, geom: Geometry, dev_ptr: int):
        _check(lib().mirorr_bm_set_search_image_device16(self._h, ctypes.byref(geom),
                                                         ctypes.c_void_p(dev_ptr)))

    def SwapImageOrder(self):
        _check(lib().mirorr_bm_swap_image_order(self._h))

    def Grid(self):
        nb = (ctypes.c_int32 * 3)()
        st = (ctypes.c_int32 * 3)()
        _check(lib().mirorr_bm_grid(self._h, nb, st))
        return tuple(nb), tuple(st)

    def GetOffsets(self):
        """Returns (block_positions, match_positions): (n, 3) float64 arrays in mm."""
        nb, _ = self.Grid()
        cap = nb[0] * nb[1] * nb[2]
        bp = np.zeros((cap, 3), np.float64)
        mp = np.zeros((cap, 3), np.float64)
        n = ctypes.c_size_t(0)
        _check(lib().mirorr_bm_get_offsets(self._h, cap, _ptr(bp), _ptr(mp), ctypes.byref(n)))
        return bp[:n.value], mp[:n.value]

    def BlockResults(self):
        """Per-block (match_index (N,3), best, second, status) of the last GetOffsets."""
        nb, _ = self.Grid()
        cap = nb[0] * nb[1] * nb[2]
        mi = np.zeros((cap, 3), np.int32)
        best = np.zeros(cap, np.float32)
        second = np.zeros(cap, np.float32)
        status = np.zeros(cap, np.uint8)
        n = ctypes.c_size_t(0)
        _check(lib().mirorr_bm_block_results(self._h, cap, _ptr(mi), _ptr(best), _ptr(second),
                                             _ptr(status), ctypes.byref(n)))
        k = n.value
        return mi[:k], best[:k], second[:k], status[:k]

    def LastTimings(self):
        ms = np.zeros(4, np.float32)
        _check(lib().mirorr_bm_last_timings(self._h, _ptr(ms)))
        return ms

    def LastDiagnostics(self):
        """(FP64-refined candidates, fully re-scored blocks, kept blocks, grid blocks,
        blocks scored by the register-blocked kernels (unmasked and masked
        window), blocks with a partly masked base block)."""
        d = np.zeros(6, np.int64)
        _check(lib().mirorr_bm_last_diagnostics(self._h, _ptr(d)))
        return tuple(int(v) for v in d)

    def close(self):
        if self._h:
            lib().mirorr_bm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if sys.is_finalizing():
                return
            self.close()
        except Exception:
            pass


def resample_map(out_geom: Geometry, in_geom: Geometry, M, offset):
    C = np.zeros(9, np.float64)
    e = np.zeros(3, np.float64)
    Mm = np.ascontiguousarray(np.asarray(M, np.float64).reshape(-1))
    o = np.ascontiguousarray(np.asarray(offset, np.float64))
    _check(lib().mirorr_resample_map(ctypes.byref(out_geom), ctypes.byref(in_geom), _ptr(Mm),
                                     _ptr(o), _ptr(C), _ptr(e)))
    return C.reshape(3, 3), e


def resample(ctx: Context, image, mask, out_size_xyz, C, e, nearest=False):
    """Linear (or nearest-neighbour) resampling of image (float32) and/or mask
    (uint8) on an index map."""
    ref = image if image is not None else mask
    in_size = (ctypes.c_int32 * 3)(ref.shape[2], ref.shape[1], ref.shape[0])
    out_size = (ctypes.c_int32 * 3)(*[int(v) for v in out_size_xyz])
    shape = (int(out_size_xyz[2]), int(out_size_xyz[1]), int(out_size_xyz[0]))
    img = _f32(image) if image is not None else None
    msk = _u8(mask)
    out = np.zeros(shape, np.float32) if img is not None else None
    outm = np.zeros(shape, np.uint8) if msk is not None else None
    Cc = np.ascontiguousarray(np.asarray(C, np.float64).reshape(-1))
    ec = np.ascontiguousarray(np.asarray(e, np.float64))
    fn = lib().mirorr_resample_nearest if nearest else lib().mirorr_resample
    _check(fn(ctx.handle, in_size, _ptr(img), _ptr(msk), out_size, _ptr(Cc), _ptr(ec), _ptr(out),
              _ptr(outm)))
    return out, outm


def resample_device(ctx: Context, in_image_ptr, in_mask_ptr, in_size_xyz, out_size_xyz, C, e,
                    out_image_ptr, out_mask_ptr, nearest=False):
    """Linear (or nearest) resampling of device buffers (integer addresses on
    the context's device; either image or mask may be None), issued on the
    context's stream without waiting for it."""
    in_size = (ctypes.c_int32 * 3)(*[int(v) for v in in_size_xyz])
    out_size = (ctypes.c_int32 * 3)(*[int(v) for v in out_size_xyz])
    Cc = np.ascontiguousarray(np.asarray(C, np.float64).reshape(-1))
    ec = np.ascontiguousarray(np.asarray(e, np.float64))
    vp = ctypes.c_void_p
    _check(lib().mirorr_resample_device(
        ctx.handle, in_size, vp(in_image_ptr) if in_image_ptr else None,
        vp(in_mask_ptr) if in_mask_ptr else None, out_size, _ptr(Cc), _ptr(ec),
        vp(out_image_ptr) if out_image_ptr else None, vp(out_mask_ptr) if out_mask_ptr else None,
        1 if nearest else 0))


def resample_final(ctx: Context, image, out_size_xyz, C, e, interpolator="bspline"):
    """Final resampling of image (float32, z, y, x) on an index map with the
    cubic B-spline ("bspline") or the radius-5 Welch-windowed sinc ("sinc")
    interpolator of GetResampledImage."""
    img = _f32(image)
    in_size = (ctypes.c_int32 * 3)(img.shape[2], img.shape[1], img.shape[0])
    out_size = (ctypes.c_int32 * 3)(*[int(v) for v in out_size_xyz])
    out = np.zeros((int(out_size_xyz[2]), int(out_size_xyz[1]), int(out_size_xyz[0])), np.float32)
    Cc = np.ascontiguousarray(np.asarray(C, np.float64).reshape(-1))
    ec = np.ascontiguousarray(np.asarray(e, np.float64))
    if interpolator == "bspline":
        fn = lib().mirorr_resample_bspline
    elif interpolator == "sinc":
        fn = lib().mirorr_resample_sinc
    else:
        raise ValueError("interpolator must be 'bspline' or 'sinc'")
    _check(fn(ctx.handle, in_size, _ptr(img), out_size, _ptr(Cc), _ptr(ec), _ptr(out)))
    return out


def lts_classic(ctx: Context, t: Transform, init, moved, lts_keep=0.5):
    init = np.ascontiguousarray(init, np.float64)
    moved = np.ascontiguousarray(moved, np.float64)
    it = ctypes.c_int32(0)
    _check(lib().mirorr_lts_classic(ctx.handle, ctypes.byref(t), init.shape[0], _ptr(init),
                                    _ptr(moved), float(lts_keep), ctypes.byref(it)))
    return it.value


def lts_symmetric(ctx: Context, t: Transform, t12f: Transform, t12b: Transform, init, moved,
                  lts_keep=0.5):
    init = np.ascontiguousarray(init, np.float64)
    moved = np.ascontiguousarray(moved, np.float64)
    it = ctypes.c_int32(0)
    _check(lib().mirorr_lts_symmetric(ctx.handle, ctypes.byref(t), ctypes.byref(t12f),
                                      ctypes.byref(t12b), init.shape[0], _ptr(init), _ptr(moved),
                                      float(lts_keep), ctypes.byref(it)))
    return it.value


LTS_NOALLOC_MAX_POINTS = 524288


def lts_noalloc(ctx: Context, t: Transform, n: int, init_dev: int, moved_dev: int,
                lts_keep=0.5, t12f: Transform | None = None, t12b: Transform | None = None):
    """LTS fit on point pairs already in device memory, allocating no device memory.

    No reference counterpart.  For callers that must not allocate after
    set-up (cudaFree synchronises the device; cudaMalloc fails when another
    allocator holds the memory).  init_dev / moved_dev are device addresses
    of n x 3 float64 arrays on the context's device (e.g. a CUDA tensor's
    data_ptr()).  Classic fit when t12f and t12b are None, symmetric when
    both are given; the results equal lts_classic / lts_symmetric.  The
    scratch is a static device array sized for LTS_NOALLOC_MAX_POINTS pairs
    (larger n raises MirorrError with MIRORR_ERANGE).  The first call on a
    device does the set-up (loading the device code reserves the array), so
    make it before a caching allocator takes the free memory.  Every call
    synchronises the context's stream, so none can run under stream capture.
    Calls on one device share the scratch, so calls that overlap in time race.
    Returns the number of LTS inner iterations."""
    it = ctypes.c_int32(0)
    pf = None if t12f is None else ctypes.byref(t12f)
    pb = None if t12b is None else ctypes.byref(t12b)
    _check(lib().mirorr_lts_noalloc(ctx.handle, ctypes.byref(t), pf, pb, int(n),
                                    ctypes.c_void_p(init_dev), ctypes.c_void_p(moved_dev),
                                    float(lts_keep), ctypes.byref(it)))
    return it.value


def reg_params(symmetric=True, kind="rigid", levels=0, iterations=5, block_width=4, block_gap=1,
               nhood_gap=3, nhood_width=7, block_keep=1.0, lts_keep=0.5, min_length=32,
               verbosity=0, last_level=0, storage="f32") -> RegParams:
    p = RegParams()
    _check(lib().mirorr_reg_default_params(ctypes.byref(p)))
    p.symmetric = 1 if symmetric else 0
    p.kind = RIGID if kind == "rigid" else AFFINE
    p.levels = int(levels)
    p.iterations = int(iterations)
    p.min_length = int(min_length)
    p.bm.block_width = int(block_width)
    p.bm.block_gap = int(block_gap)
    p.bm.nhood_gap = int(nhood_gap)
    p.bm.nhood_width = int(nhood_width)
    p.bm.block_keep = float(block_keep)
    p.lts_keep = float(lts_keep)
    p.verbosity = int(verbosity)
    p.last_level = int(last_level)
    p.storage = dtype_code(storage)
    return p


def register(ctx: Context, fixed, moving, params: RegParams, fixed_geom: Geometry | None = None,
             moving_geom: Geometry | None = None, fixed_mask=None, moving_mask=None,
             init: Transform | None = None):
    """Full registration from host arrays.  Returns (Transform, RegStats).
    With 16-bit storage (params.storage) float32 arrays are converted with
    to_storage() first; uint16 arrays are taken as storage bit patterns."""
    if params.storage == F32:
        f = _f32(fixed)
        m = _f32(moving)
    else:
        f = fixed if np.asarray(fixed).dtype == np.uint16 else to_storage(fixed, params.storage)
        m = moving if np.asarray(moving).dtype == np.uint16 else to_storage(moving, params.storage)
        f = np.ascontiguousarray(f)
        m = np.ascontiguousarray(m)
    fg = fixed_geom or Geometry.of(f)
    mg = moving_geom or Geometry.of(m)
    res = Transform()
    st = RegStats()
    _check(lib().mirorr_register(ctx.handle, ctypes.byref(fg), _ptr(f), _ptr(_u8(fixed_mask)),
                                 ctypes.byref(mg), _ptr(m), _ptr(_u8(moving_mask)),
                                 ctypes.byref(params), ctypes.byref(init) if init else None,
                                 ctypes.byref(res), ctypes.byref(st)))
    return res, st


def register_device(ctx: Context, fixed_ptr: int, fixed_geom: Geometry, moving_ptr: int,
                    moving_geom: Geometry, params: RegParams, fixed_mask_ptr=None,
                    moving_mask_ptr=None, init: Transform | None = None):
    res = Transform()
    st = RegStats()
    _check(lib().mirorr_register_device(
        ctx.handle, ctypes.byref(fixed_geom), ctypes.c_void_p(fixed_ptr),
        ctypes.c_void_p(fixed_mask_ptr) if fixed_mask_ptr else None, ctypes.byref(moving_geom),
        ctypes.c_void_p(moving_ptr), ctypes.c_void_p(moving_mask_ptr) if moving_mask_ptr else None,
        ctypes.byref(params), ctypes.byref(init) if init else None, ctypes.byref(res),
        ctypes.byref(st)))
    return res, st


def pyramid_schedule(fixed_geom: Geometry, moving_geom: Geometry, min_length=32, max_levels=0):
    n = ctypes.c_int32(0)
    mf = np.zeros((16, 3), np.int32)
    ff = np.zeros((16, 3), np.int32)
    _check(lib().mirorr_pyramid_schedule(ctypes.byref(fixed_geom), ctypes.byref(moving_geom),
                                         int(min_length), int(max_levels), ctypes.byref(n),
                                         _ptr(mf), _ptr(ff)))
    return mf[:n.value].copy(), ff[:n.value].copy()


def pyramid_level(ctx: Context, image, factors, geom: Geometry | None = None):
    img = _f32(image)
    g = geom or Geometry.of(img)
    og = Geometry()
    cap = int(np.prod([max(1, s // f) for s, f in zip(tuple(g.size), factors)]))
    out = np.zeros(cap, np.float32)
    fac = (ctypes.c_int32 * 3)(*[int(v) for v in factors])
    _check(lib().mirorr_pyramid_level(ctx.handle, ctypes.byref(g), _ptr(img), fac, ctypes.byref(og),
                                      _ptr(out), cap))
    nx, ny, nz = tuple(og.size)
    return out[: nx * ny * nz].reshape(nz, ny, nx), og


class Batch:
    """Many registrations on the device at once (mirorr_batch; no reference
    counterpart).  submit() admits a request while a slot and the memory
    budget allow (MirorrError EBUSY otherwise), step() advances every running
    request by one iteration, result() returns a finished request's transform
    and frees its slot.  Requests may be submitted between steps."""

    def __init__(self, ctx: Context, max_slots=64, hbm_budget=150e9):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        _check(lib().mirorr_batch_create(ctx.handle, int(max_slots), int(hbm_budget),
                                         ctypes.byref(self._h)))

    def submit(self, fixed, moving, params: RegParams, fixed_geom: Geometry | None = None,
               moving_geom: Geometry | None = None, fixed_mask=None, moving_mask=None,
               init: Transform | None = None) -> int:
        f = fixed if np.asarray(fixed).dtype == np.uint16 else to_storage(fixed, params.storage)
        m = moving if np.asarray(moving).dtype == np.uint16 else to_storage(moving, params.storage)
        f = np.ascontiguousarray(f)
        m = np.ascontiguousarray(m)
        fg = fixed_geom or Geometry.of(f)
        mg = moving_geom or Geometry.of(m)
        rid = ctypes.c_int64(0)
        _check(lib().mirorr_batch_submit(self._h, ctypes.byref(fg), _ptr(f), _ptr(_u8(fixed_mask)),
                                         ctypes.byref(mg), _ptr(m), _ptr(_u8(moving_mask)),
                                         ctypes.byref(params), ctypes.byref(init) if init else None,
                                         ctypes.byref(rid)))
        return rid.value

    def step(self):
        """One iteration of every running request: (running, finished)."""
        r = ctypes.c_int32(0)
        f = ctypes.c_int32(0)
        _check(lib().mirorr_batch_step(self._h, ctypes.byref(r), ctypes.byref(f)))
        return r.value, f.value

    def run(self):
        _check(lib().mirorr_batch_run(self._h))

    def poll(self):
        ids = np.zeros(256, np.int64)
        n = ctypes.c_int32(0)
        _check(lib().mirorr_batch_poll(self._h, _ptr(ids), 256, ctypes.byref(n)))
        return [int(v) for v in ids[:min(n.value, 256)]]

    def result(self, request_id: int):
        res = Transform()
        st = RegStats()
        _check(lib().mirorr_batch_result(self._h, int(request_id), ctypes.byref(res),
                                         ctypes.byref(st)))
        return res, st

    def cancel(self, request_id: int):
        _check(lib().mirorr_batch_cancel(self._h, int(request_id)))

    def info(self):
        v = np.zeros(8, np.int64)
        _check(lib().mirorr_batch_info(self._h, _ptr(v)))
        keys = ["running", "finished", "bytes_reserved", "budget", "steps", "replays", "captures",
                "updates"]
        return dict(zip(keys, [int(x) for x in v]))

    def times(self):
        """Host-clock seconds spent by the steps so far: level setup, descriptor
        and graph building, launch to end of device work, request advance."""
        v = np.zeros(4, np.float64)
        _check(lib().mirorr_batch_times(self._h, _ptr(v)))
        return dict(zip(["setup", "issue", "device", "advance"], [float(x) for x in v]))

    def set_graphs(self, on: bool):
        _check(lib().mirorr_batch_set_graphs(self._h, 1 if on else 0))

    def close(self):
        if self._h:
            lib().mirorr_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if not sys.is_finalizing():
                self.close()
        except Exception:
            pass

