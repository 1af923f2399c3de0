"""The oracle's final-resampling interpolators (cubic B-spline, Welch-windowed
sinc) against properties the published algorithms guarantee: interpolation
of the samples on the grid, reproduction of a quadratic by the cubic spline
away from the boundaries, and a band-limited signal by the sinc."""
import numpy as np

from oracle import oracle as O


def test_bspline_interpolates_the_samples():
    rng = np.random.default_rng(0)
    img = rng.random((9, 11, 13)).astype(np.float32)
    out = O.resample_bspline(img, (13, 11, 9), np.eye(3), [0.0, 0.0, 0.0])
    np.testing.assert_allclose(out, img, rtol=0, atol=2e-6)


def test_bspline_coefficients_of_a_constant_are_the_constant():
    # lines longer than the causal horizon (18 taps) truncate the initial sum
    # at the prefilter's tolerance, 1e-10
    img = np.full((5, 7, 30), 3.25, np.float32)
    np.testing.assert_allclose(O.bspline_coefficients(img), 3.25, rtol=1e-9)


def test_bspline_reproduces_a_quadratic_inside():
    x = np.arange(40, dtype=np.float64)
    img = np.broadcast_to((0.01 * (x - 17) ** 2 + 3)[None, None, :], (6, 6, 40)).astype(np.float32)
    out = O.resample_bspline(img, (40, 6, 6), np.eye(3), [0.37, 0.0, 0.0])
    xs = x[10:30] + 0.37
    np.testing.assert_allclose(out[3, 3, 10:30], 0.01 * (xs - 17) ** 2 + 3, rtol=0, atol=2e-6)


def test_bspline_outside_is_zero():
    img = np.ones((4, 5, 6), np.float32)
    out = O.resample_bspline(img, (3, 1, 1), np.eye(3), [-0.6, 0.0, 0.0])
    assert out[0, 0, 0] == 0.0 and out[0, 0, 1] == 1.0


def test_sinc_copies_on_the_grid_and_follows_a_smooth_signal():
    rng = np.random.default_rng(1)
    img = rng.random((8, 9, 10)).astype(np.float32)
    np.testing.assert_array_equal(O.resample_sinc(img, (10, 9, 8), np.eye(3), [0, 0, 0]), img)
    x = np.arange(40, dtype=np.float64)
    s = np.broadcast_to(np.sin(2 * np.pi * x / 16.0)[None, None, :], (12, 12, 40)).astype(np.float32)
    out = O.resample_sinc(s, (40, 12, 12), np.eye(3), [0.5, 0.0, 0.0])
    np.testing.assert_allclose(out[6, 6, 8:30], np.sin(2 * np.pi * (x[8:30] + 0.5) / 16.0),
                               atol=5e-3)


def test_bspline_short_lines_interpolate_the_samples():
    # lines of length 1 and 2 (the full mirror-symmetric initial sum; the
    # mirror boundary with period 2N - 2) still pass through the samples
    rng = np.random.default_rng(2)
    for shape in [(1, 2, 5), (2, 1, 3), (1, 1, 2)]:
        img = rng.random(shape).astype(np.float32)
        size = (shape[2], shape[1], shape[0])
        out = O.resample_bspline(img, size, np.eye(3), [0.0, 0.0, 0.0])
        np.testing.assert_allclose(out, img, rtol=0, atol=2e-6)
