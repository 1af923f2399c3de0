"""The allocation-free LTS entry point (mirorr_lts_noalloc) against the
allocating ones (mirorr_lts_classic / mirorr_lts_symmetric) on the same point
pairs, through the C ABI.

mirorr_lts_noalloc has no reference counterpart: it runs the same cooperative
LTS kernel with its scratch in a static device array, for callers that must
not allocate device memory.  Each case runs two calls in a row of each entry
point from the same starting transforms (the second call of the static-scratch
path reuses the array the first one left behind) and requires the fits to
agree within 1e-12 and take the same number of inner iterations.  This file is
collected last so that it also runs after every other GPU test; it passes
alone in a fresh process too.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import random_rotation
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _pairs(kind, seed, n, outliers=0.25):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-60, 60, size=(n, 3))
    m = random_rotation(rng, 4.0)
    if kind == "affine":
        m = m @ np.diag(rng.uniform(0.95, 1.05, 3))
    y = x @ m.T + rng.uniform(-4, 4, 3) + rng.normal(0, 0.3, size=(n, 3))
    k = int(outliers * n)
    y[:k] += rng.normal(0, 10, size=(k, 3))
    return x, y


def _start(kind):
    params = ([0.01, -0.02, 0.015, 1.0, 0.5, -0.5] if kind == "rigid" else
              [1.01, 0.01, 0, 0, 0.99, 0.02, 0, -0.01, 1.0, 1.0, 0.5, -0.5])
    return mb.Transform.make(mb.RIGID if kind == "rigid" else mb.AFFINE, params,
                             (3.0, -2.0, 5.0))


def _copy(t):
    return mb.Transform.from_buffer_copy(t)


def _to_mb(t):
    return mb.Transform.make(mb.RIGID if t.kind == "rigid" else mb.AFFINE, t.params(), t.c)


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).to("cuda:0")


def _same(a, b):
    np.testing.assert_allclose(a.M, b.M, rtol=0, atol=TOL)
    np.testing.assert_allclose(a.off, b.off, rtol=0, atol=TOL)
    np.testing.assert_allclose(np.array(a.center), np.array(b.center), rtol=0, atol=TOL)


@pytest.mark.parametrize("kind,n", [("affine", 3000), ("rigid", 20000), ("affine", 400000)])
def test_noalloc_classic_matches(ctx, kind, n):
    import torch
    x, y = _pairs(kind, 21, n)
    xd, yd = _device(x), _device(y)
    torch.cuda.synchronize()
    for _ in range(2):
        ta, tb = _start(kind), _start(kind)
        it_a = mb.lts_classic(ctx, ta, x, y, 0.5)
        it_b = mb.lts_noalloc(ctx, tb, n, xd.data_ptr(), yd.data_ptr(), 0.5)
        assert it_b == it_a
        _same(tb, ta)
    # the defining property: once set up, a call takes no device memory
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        mb.lts_noalloc(ctx, _start(kind), n, xd.data_ptr(), yd.data_ptr(), 0.5)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.parametrize("kind", ["rigid", "affine"])
def test_noalloc_symmetric_matches(ctx, kind):
    import torch
    n = 50000
    x, y = _pairs(kind, 22, n)
    xd, yd = _device(x), _device(y)
    torch.cuda.synchronize()
    t = O.Tfm(kind)
    t.set_params([0.01, -0.02, 0.015, 1.0, 0.5, -0.5] if kind == "rigid" else
                 [1.01, 0.01, 0, 0, 0.99, 0.02, 0, -0.01, 1.0, 1.0, 0.5, -0.5])
    f, b = O.compute_half_space(t)
    t0, f0, b0 = _to_mb(t), _to_mb(f), _to_mb(b)
    for _ in range(2):
        ta, fa, ba = _copy(t0), _copy(f0), _copy(b0)
        tb, fb, bb = _copy(t0), _copy(f0), _copy(b0)
        it_a = mb.lts_symmetric(ctx, ta, fa, ba, x, y, 0.5)
        it_b = mb.lts_noalloc(ctx, tb, n, xd.data_ptr(), yd.data_ptr(), 0.5, t12f=fb, t12b=bb)
        assert it_b == it_a
        for a, b in [(ta, tb), (fa, fb), (ba, bb)]:
            _same(b, a)


def test_noalloc_rejects(ctx):
    import torch
    x, y = _pairs("affine", 23, 64)
    xd, yd = _device(x), _device(y)
    torch.cuda.synchronize()
    with pytest.raises(mb.MirorrError) as e:
        mb.lts_noalloc(ctx, _start("affine"), mb.LTS_NOALLOC_MAX_POINTS + 1, xd.data_ptr(),
                       yd.data_ptr(), 0.5)
    assert e.value.name == "ERANGE"
    with pytest.raises(mb.MirorrError) as e:  # host memory is refused before any launch
        mb.lts_noalloc(ctx, _start("affine"), 64, x.ctypes.data, y.ctypes.data, 0.5)
    assert e.value.name == "EINVAL"
    # arrays shorter than n x 3 doubles: an allocation of its own (not a slice
    # of a caching allocator's segment) holding 64 pairs, asked for 65
    from cuda.bindings import runtime as cudart
    err, raw = cudart.cudaMalloc(64 * 3 * 8)
    assert err == cudart.cudaError_t.cudaSuccess
    try:
        err, = cudart.cudaMemcpy(raw, x.ctypes.data, 64 * 3 * 8,
                                 cudart.cudaMemcpyKind.cudaMemcpyHostToDevice)
        assert err == cudart.cudaError_t.cudaSuccess
        assert mb.lts_noalloc(ctx, _start("affine"), 64, raw, yd.data_ptr(), 0.5) >= 0
        with pytest.raises(mb.MirorrError) as e:
            mb.lts_noalloc(ctx, _start("affine"), 65, raw, yd.data_ptr(), 0.5)
        assert e.value.name == "EINVAL"
    finally:
        cudart.cudaFree(raw)
    with pytest.raises(mb.MirorrError) as e:  # only one half-space transform
        mb.lts_noalloc(ctx, _start("affine"), 64, xd.data_ptr(), yd.data_ptr(), 0.5,
                       t12f=_start("affine"))
    assert e.value.name == "EINVAL"
