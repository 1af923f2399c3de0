"""Full registration (mirorr_register through the C ABI) against the FP64
oracle run on the same inputs.

The bar: final 3x3 matrices within 1e-4 of the oracle's (entry-wise) and
offsets within 1e-3 mm.  Target registration error against the known
synthetic transform is reported; it must match the oracle's and improve on
the initial misalignment.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom, tre
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    dict(id="classic_rigid", mode="classic", kind="rigid", shape=(64, 64, 40), levels=2,
         iters=4, G=3, nw=7, keep=1.0, seed=21),
    dict(id="symmetric_affine", mode="symmetric", kind="affine", shape=(64, 64, 40), levels=2,
         iters=4, G=3, nw=7, keep=1.0, seed=22),
    dict(id="symmetric_rigid_keep05", mode="symmetric", kind="rigid", shape=(72, 64, 40),
         levels=2, iters=3, G=3, nw=7, keep=0.5, seed=23),
    # three iterations do not converge on this small pair: the oracle ends
    # worse than the start too; the case still checks parity
    dict(id="classic_affine", mode="classic", kind="affine", shape=(64, 64, 48), levels=2,
         iters=3, G=3, nw=7, keep=1.0, seed=24, improves=False),
]


@pytest.mark.parametrize("c", CASES, ids=[c["id"] for c in CASES])
def test_registration_matches_oracle(ctx, c):
    ph = make_phantom(c["shape"], n_gauss=20, kind=c["kind"], seed=c["seed"], max_angle_deg=4.0,
                      max_shift_vox=4.0)
    rp = O.RegParams(c["mode"], c["kind"], c["iters"], O.BMParams(4, 1, c["G"], c["nw"], c["keep"]),
                     0.5)
    fixed = O.Image(ph.fixed, ph.spacing, ph.origin)
    moving = O.Image(ph.moving, ph.spacing, ph.origin)
    to = O.register(fixed, moving, rp, c["levels"])
    p = mb.reg_params(symmetric=c["mode"] == "symmetric", kind=c["kind"], levels=c["levels"],
                      iterations=c["iters"], nhood_gap=c["G"], nhood_width=c["nw"],
                      block_keep=c["keep"])
    tg, st = mb.register(ctx, ph.fixed, ph.moving, p)
    assert st.levels_run == c["levels"] and st.block_ncc_evaluated > 0
    np.testing.assert_allclose(tg.M, to.M, atol=1e-4, rtol=0)
    np.testing.assert_allclose(tg.off, to.off, atol=1e-3, rtol=0)
    err = tre(tg.M, tg.off, ph.true_matrix, ph.true_offset, c["shape"], ph.spacing)
    err_o = tre(to.M, to.off, ph.true_matrix, ph.true_offset, c["shape"], ph.spacing)
    err_0 = tre(np.eye(3), np.zeros(3), ph.true_matrix, ph.true_offset, c["shape"], ph.spacing)
    print(f"{c['id']}: TRE gpu {err:.4f} mm, oracle {err_o:.4f} mm, initial {err_0:.4f} mm, "
          f"max |dM| {np.max(np.abs(tg.M - to.M)):.2e}")
    assert abs(err - err_o) < 1e-3
    if c.get("improves", True):
        assert err < err_0


def test_registration_matches_oracle_at_classic_rigid_128x128x64(ctx):
    """The classic rigid configuration at its full size: 128x128x64 pair of 40
    Gaussians (intensity-mapped moving image, rotation up to 5 degrees,
    translation up to 8 voxels), 2 pyramid levels, block 4, block spacing 4,
    radius 3 (343 candidates), top 50 % of blocks by variance, LTS keep 0.5,
    10 iterations per level.  Same bars as the small cases."""
    shape = (128, 128, 64)
    ph = make_phantom(shape, n_gauss=40, kind="rigid", seed=0, max_angle_deg=5.0,
                      max_shift_vox=8.0)
    rp = O.RegParams("classic", "rigid", 10, O.BMParams(4, 1, 4, 7, 0.5), 0.5)
    fixed = O.Image(ph.fixed, ph.spacing, ph.origin)
    moving = O.Image(ph.moving, ph.spacing, ph.origin)
    to = O.register(fixed, moving, rp, 2)
    p = mb.reg_params(symmetric=False, kind="rigid", levels=2, iterations=10, nhood_gap=4,
                      nhood_width=7, block_keep=0.5, lts_keep=0.5)
    tg, st = mb.register(ctx, ph.fixed, ph.moving, p)
    assert st.levels_run == 2
    np.testing.assert_allclose(tg.M, to.M, atol=1e-4, rtol=0)
    np.testing.assert_allclose(tg.off, to.off, atol=1e-3, rtol=0)
    err = tre(tg.M, tg.off, ph.true_matrix, ph.true_offset, shape, ph.spacing)
    err_o = tre(to.M, to.off, ph.true_matrix, ph.true_offset, shape, ph.spacing)
    err_0 = tre(np.eye(3), np.zeros(3), ph.true_matrix, ph.true_offset, shape, ph.spacing)
    print(f"128x128x64 classic rigid: TRE gpu {err:.4f} mm, oracle {err_o:.4f} mm, initial "
          f"{err_0:.4f} mm, max |dM| {np.max(np.abs(tg.M - to.M)):.2e}")
    assert abs(err - err_o) < 1e-3
    assert err < err_0


@pytest.mark.parametrize("mode,kind,keep", [("symmetric", "affine", 1.0), ("classic", "rigid", 1.0),
                                            ("symmetric", "affine", 0.5)])
def test_iteration_graphs_equal_direct_launches(ctx, mode, kind, keep):
    """Iterations replayed from a per-level CUDA graph (the default for float32
    storage) run the same kernels on the same data as direct launches: the
    registration is bit-identical either way (block keep 0.5: the variance
    selection's cooperative launch inside the graph)."""
    ph = make_phantom((72, 64, 48), n_gauss=20, kind=kind, seed=71, max_angle_deg=4.0,
                      max_shift_vox=4.0)
    p = mb.reg_params(symmetric=mode == "symmetric", kind=kind, levels=2, iterations=5,
                      nhood_gap=3, nhood_width=7, block_keep=keep)
    try:
        ctx.set_graphs(False)
        direct, st0 = mb.register(ctx, ph.fixed, ph.moving, p)
        ctx.set_graphs(True)
        replayed, st1 = mb.register(ctx, ph.fixed, ph.moving, p)
    finally:
        ctx.set_graphs(True)
    assert sum(st1.iterations_run) > 2  # some iterations were replayed
    np.testing.assert_array_equal(replayed.M, direct.M)
    np.testing.assert_array_equal(replayed.off, direct.off)
    assert st1.matcher_calls == st0.matcher_calls
    assert st1.block_ncc_evaluated == st0.block_ncc_evaluated
