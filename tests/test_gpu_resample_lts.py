"""Resampler, pyramid and LTS fits through the C ABI against the oracle.

* resampler: bit-exact for the same index map (FP64 arithmetic restated
  with explicit rounding on both sides); map construction within 1e-12;
* pyramid level: bit-exact;
* LTS fits: matrices and offsets within 1e-9 of the oracle on the same point
  pairs, same number of inner iterations.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom, random_rotation
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_resample_bit_exact(ctx, seed):
    rng = np.random.default_rng(seed)
    img = rng.random((23, 29, 31)).astype(np.float32)
    msk = (rng.random(img.shape) > 0.3).astype(np.uint8) * 255
    M = random_rotation(rng, 10.0) @ np.diag(rng.uniform(0.9, 1.1, 3))
    off = rng.uniform(-3, 3, 3)
    gin = O.Image(img, np.array([1.0, 1.1, 0.9]), np.array([0.5, -1.0, 2.0]))
    gout = O.Image(np.zeros((20, 27, 33), np.float32), np.array([1.05, 1.0, 1.0]),
                   np.array([1.0, 0.0, 1.5]))
    C, e = O.resample_map(gout, gin, M, off)
    out_o, outm_o = O.resample(img, msk, gout.size, C, e)
    out_g, outm_g = mb.resample(ctx, img, msk, gout.size, C, e)
    np.testing.assert_array_equal(out_g, out_o)
    np.testing.assert_array_equal(outm_g, outm_o)
    Cg, eg = mb.resample_map(mb.Geometry.make(gout.size, gout.spacing, gout.origin),
                             mb.Geometry.make(gin.size, gin.spacing, gin.origin), M, off)
    np.testing.assert_allclose(Cg, C, atol=1e-12)
    np.testing.assert_allclose(eg, e, atol=1e-12)


def test_resample_image_only_and_mask_only(ctx):
    # separate launches for an image alone and a mask alone, an output size
    # that is not a multiple of the 4-voxel run (ragged last run)
    rng = np.random.default_rng(5)
    img = rng.random((13, 17, 19)).astype(np.float32)
    msk = (rng.random(img.shape) > 0.5).astype(np.uint8) * 255
    M = random_rotation(rng, 7.0)
    gin = O.Image(img, np.array([1.0, 1.0, 1.0]), np.zeros(3))
    gout = O.Image(np.zeros((11, 15, 21), np.float32), np.array([1.1, 1.0, 0.9]),
                   np.array([0.5, 0.5, 0.0]))
    C, e = O.resample_map(gout, gin, M, rng.uniform(-2, 2, 3))
    out_o, outm_o = O.resample(img, msk, gout.size, C, e)
    out_g, _ = mb.resample(ctx, img, None, gout.size, C, e)
    _, outm_g = mb.resample(ctx, None, msk, gout.size, C, e)
    np.testing.assert_array_equal(out_g, out_o)
    np.testing.assert_array_equal(outm_g, outm_o)


@pytest.mark.parametrize("seed", [3, 4])
def test_resample_nearest_bit_exact(ctx, seed):
    rng = np.random.default_rng(seed)
    img = rng.random((21, 26, 30)).astype(np.float32)
    msk = (rng.random(img.shape) > 0.4).astype(np.uint8) * 255
    M = random_rotation(rng, 12.0) @ np.diag(rng.uniform(0.85, 1.15, 3))
    off = rng.uniform(-4, 4, 3)
    gin = O.Image(img, np.array([1.0, 0.8, 1.1]), np.array([0.0, 1.0, -2.0]))
    gout = O.Image(np.zeros((19, 25, 31), np.float32), np.array([1.1, 0.9, 1.0]),
                   np.array([0.5, 0.0, -1.0]))
    C, e = O.resample_map(gout, gin, M, off)
    out_o, outm_o = O.resample_nearest(img, msk, gout.size, C, e)
    out_g, outm_g = mb.resample(ctx, img, msk, gout.size, C, e, nearest=True)
    np.testing.assert_array_equal(out_g, out_o)
    np.testing.assert_array_equal(outm_g, outm_o)


@pytest.mark.parametrize("shape", [(17, 19, 23), (9, 2, 14), (6, 11, 1)])
def test_resample_bspline_bit_exact(ctx, shape):
    # final resampling, cubic B-spline: FP64 prefilter and evaluation restated
    # with explicit rounding on both sides; axes of length 2 and 1 included
    rng = np.random.default_rng(sum(shape))
    img = (rng.random(shape) * 100.0).astype(np.float32)
    M = random_rotation(rng, 9.0) @ np.diag(rng.uniform(0.9, 1.1, 3))
    off = rng.uniform(-2, 2, 3)
    gin = O.Image(img, np.array([1.0, 0.9, 1.1]), np.array([0.5, -1.0, 2.0]))
    gout = O.Image(np.zeros((15, 18, 20), np.float32), np.array([1.05, 1.0, 0.95]),
                   np.array([1.0, 0.0, 1.5]))
    C, e = O.resample_map(gout, gin, M, off)
    want = O.resample_bspline(img, gout.size, C, e)
    got = mb.resample_final(ctx, img, gout.size, C, e, "bspline")
    np.testing.assert_array_equal(got, want)


def test_resample_sinc_matches_oracle(ctx):
    # windowed sinc: the taps call sin(), so CUDA's and the host's results may
    # differ in the last FP64 bits; after the float cast they agree to 1e-5
    rng = np.random.default_rng(7)
    img = (rng.random((14, 16, 18)) * 100.0).astype(np.float32)
    M = random_rotation(rng, 7.0)
    off = rng.uniform(-2, 2, 3)
    gin = O.Image(img, np.array([1.0, 1.0, 1.0]), np.array([0.0, 0.0, 0.0]))
    gout = O.Image(np.zeros((12, 15, 17), np.float32), np.array([1.1, 0.95, 1.0]),
                   np.array([0.3, 0.2, -0.4]))
    C, e = O.resample_map(gout, gin, M, off)
    want = O.resample_sinc(img, gout.size, C, e)
    got = mb.resample_final(ctx, img, gout.size, C, e, "sinc")
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-4)
    # on the grid the weights are a delta: an exact copy
    same = mb.resample_final(ctx, img, (18, 16, 14), np.eye(3), np.zeros(3), "sinc")
    np.testing.assert_array_equal(same, img)


@pytest.mark.parametrize("factors", [(2, 2, 2), (4, 4, 2), (2, 2, 1), (8, 8, 4)])
def test_pyramid_level_bit_exact(ctx, factors):
    ph = make_phantom((64, 48, 40), n_gauss=10, seed=3)
    img = O.Image(ph.fixed, np.array([1.0, 0.9, 1.2]), np.array([2.0, -1.0, 0.5]))
    lo = O.pyramid_level(img, factors)
    lg, g = mb.pyramid_level(ctx, ph.fixed, factors,
                             mb.Geometry.make(img.size, img.spacing, img.origin))
    np.testing.assert_array_equal(lg, lo.data)
    np.testing.assert_allclose(np.array(g.spacing), lo.spacing, rtol=0, atol=0)
    np.testing.assert_allclose(np.array(g.origin), lo.origin, atol=1e-12)


def _pairs(kind, seed, n=3000, outliers=0.25):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-60, 60, size=(n, 3))
    m = random_rotation(rng, 4.0)
    if kind == "affine":
        m = m @ np.diag(rng.uniform(0.95, 1.05, 3))
    y = x @ m.T + rng.uniform(-4, 4, 3) + rng.normal(0, 0.3, size=(n, 3))
    k = int(outliers * n)
    y[:k] += rng.normal(0, 10, size=(k, 3))
    return x, y


def _to_mb(t: O.Tfm):
    return mb.Transform.make(mb.RIGID if t.kind == "rigid" else mb.AFFINE, t.params(), t.c)


@pytest.mark.parametrize("kind", ["affine", "rigid"])
@pytest.mark.parametrize("keep", [0.5, 0.7])
def test_lts_classic_matches_oracle(ctx, kind, keep):
    x, y = _pairs(kind, 11)
    t = O.Tfm(kind)
    t.set_center([3.0, -2.0, 5.0])
    t.set_params([0.01, -0.02, 0.015, 1.0, 0.5, -0.5] if kind == "rigid" else
                 [1.01, 0.01, 0, 0, 0.99, 0.02, 0, -0.01, 1.0, 1.0, 0.5, -0.5])
    tg = _to_mb(t)
    it_o = O.lts_classic(t, x, y, keep)
    it_g = mb.lts_classic(ctx, tg, x, y, keep)
    assert it_g == it_o
    np.testing.assert_allclose(tg.M, t.M, atol=1e-9)
    np.testing.assert_allclose(tg.off, t.off, atol=1e-8)


@pytest.mark.parametrize("kind", ["affine", "rigid"])
def test_lts_symmetric_matches_oracle(ctx, kind):
    x, y = _pairs(kind, 12)
    t = O.Tfm(kind)
    t.set_params([0.01, -0.02, 0.015, 1.0, 0.5, -0.5] if kind == "rigid" else
                 [1.01, 0.01, 0, 0, 0.99, 0.02, 0, -0.01, 1.0, 1.0, 0.5, -0.5])
    f, b = O.compute_half_space(t)
    tg, fg, bg = _to_mb(t), _to_mb(f), _to_mb(b)
    it_o = O.lts_symmetric(t, f, b, x, y, 0.5)
    it_g = mb.lts_symmetric(ctx, tg, fg, bg, x, y, 0.5)
    assert it_g == it_o
    for a, o in [(tg, t), (fg, f), (bg, b)]:
        np.testing.assert_allclose(a.M, o.M, atol=1e-9)
        np.testing.assert_allclose(a.off, o.off, atol=1e-8)


def test_lts_large_point_set(ctx):
    # exercises the multi-pass radix select and the multi-CTA reductions
    x, y = _pairs("affine", 13, n=400000)
    t = O.Tfm("affine")
    tg = _to_mb(t)
    it_o = O.lts_classic(t, x, y, 0.5)
    it_g = mb.lts_classic(ctx, tg, x, y, 0.5)
    assert it_g == it_o
    np.testing.assert_allclose(tg.M, t.M, atol=1e-9)
    np.testing.assert_allclose(tg.off, t.off, atol=1e-8)


def test_lts_barrier_wait_gives_up_and_context_recovers(ctx):
    """The LTS kernel's grid-barrier waits are bounded.  With a limit of one
    poll the CTAs that reach a barrier before the others give up, every CTA
    returns, and the call reports ETIMEOUT without touching the transform; the
    default limit then fits the same pairs as the oracle (the context and the
    GPU are still usable).  Nothing faults: the waits just end early."""
    x, y = _pairs("affine", 13, n=400000)  # many CTAs, so arrivals are spread out
    t0 = O.Tfm("affine")
    tg = _to_mb(t0)
    before = (tg.M.copy(), tg.off.copy())
    ctx.set_wait_limit(1)
    try:
        with pytest.raises(mb.MirorrError) as e:
            mb.lts_classic(ctx, tg, x, y, 0.5)
        assert e.value.name == "ETIMEOUT"
        np.testing.assert_array_equal(tg.M, before[0])
        np.testing.assert_array_equal(tg.off, before[1])
    finally:
        ctx.set_wait_limit(0)
    it_o = O.lts_classic(t0, x, y, 0.5)
    it_g = mb.lts_classic(ctx, tg, x, y, 0.5)
    assert it_g == it_o
    np.testing.assert_allclose(tg.M, t0.M, atol=1e-9)
