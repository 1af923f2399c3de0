"""16-bit storage (BF16 / FP16) path through the C ABI against the FP64 oracle
run on the same stored values.

The images are stored in 16 bits (round to nearest even from float32); the
oracle sees exactly those values (oracle.round_storage), so every difference
left is the arithmetic: the block search sums in FP32 -- the cross term on the
tensor cores from two 16-bit parts of the centred base block, the rest on the
CUDA cores -- where the reference sums in FP64.  The bars, per the block
matcher's own acceptance rule:
* the searched blocks (variance selection) are identical;
* best and second-best scores within 1e-4 of the oracle's (FP32 rounding);
* the argmax equals the oracle's on every block whose oracle best-vs-second
  gap exceeds 1e-4, and on at least 99.5 % of all searched blocks;
* registrations: final matrices within 1e-4 of the oracle's registration on
  the same stored inputs, offsets within 1e-3 mm.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom, tre
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SCORE_TOL = 1e-4
GAP = 1e-4

CASES = [
    dict(id="w7_G3", shape=(52, 44, 30), nw=7, G=3, keep=1.0, mask=None, seed=31),
    dict(id="w7_G3_search_masked", shape=(52, 44, 30), nw=7, G=3, keep=1.0, mask="search", seed=32),
    dict(id="w7_G3_both_masked", shape=(48, 40, 28), nw=7, G=3, keep=1.0, mask="both", seed=33),
    dict(id="w7_G2_keep05", shape=(41, 37, 26), nw=7, G=2, keep=0.5, mask=None, seed=34),
    dict(id="w5_G1", shape=(30, 28, 22), nw=5, G=1, keep=1.0, mask="search", seed=35),
    dict(id="w7_G4_x_ragged", shape=(67, 30, 24), nw=7, G=4, keep=1.0, mask=None, seed=36),
    # window 9: every block through the direct FP32 search
    dict(id="w9_G3_direct", shape=(40, 36, 28), nw=9, G=3, keep=1.0, mask="search", seed=37),
    # block width 5 (direct search), the large stress configuration's
    # geometry at small size: window 11, spacing 3, 30 % of the blocks kept
    dict(id="bw5_w11_G3_keep03", shape=(44, 40, 30), nw=11, G=3, keep=0.3, mask=None, seed=38, bw=5),
    dict(id="bw5_w7_G2_masked", shape=(36, 34, 26), nw=7, G=2, keep=1.0, mask="both", seed=39, bw=5),
]


def make_inputs(c, store):
    ph = make_phantom(c["shape"], n_gauss=12, kind="affine" if c["seed"] % 2 else "rigid",
                      seed=200 + c["seed"])
    base = O.round_storage(ph.moving, store)
    search = O.round_storage(ph.fixed, store)
    bm = sm = None
    if c["mask"] in ("search", "both"):
        sm = np.full(search.shape, 255, np.uint8)
        sm[:, :, :6] = 0
        sm[:3] = 0
        sm[:, 12:14, 9:11] = 0
    if c["mask"] == "both":
        bm = np.full(base.shape, 255, np.uint8)
        bm[:, -7:, :] = 0
        bm[4:6, :, 11:14] = 0
    return ph, base, search, bm, sm


@pytest.mark.parametrize("store", ["bf16", "f16"])
@pytest.mark.parametrize("c", CASES, ids=[c["id"] for c in CASES])
def test_matcher16_matches_oracle(ctx, c, store):
    ph, base, search, bm, sm = make_inputs(c, store)
    m = mb.BlockMatcher(ctx)
    m.SetStorage(store)
    bw = c.get("bw", 4)
    m.SetBlockWidth(bw)
    m.SetNhoodGap(c["G"])
    m.SetNhoodWidth(c["nw"])
    m.SetBlockKeep(c["keep"])
    m.SetBaseImage(base)
    m.SetSearchImage(search)
    if bm is not None:
        m.SetBaseMask(bm)
    if sm is not None:
        m.SetSearchMask(sm)
    try:
        bp, mp = m.GetOffsets()
    except mb.MirorrError as e:
        assert e.name == "ENOBLOCKS"
        bp = np.zeros((0, 3))
    mi, best, second, status = m.BlockResults()
    diag = m.LastDiagnostics()
    m.close()
    p = O.BMParams(bw, 1, c["G"], c["nw"], c["keep"])
    ref = O.match_blocks(base, search, bm, sm, p)
    np.testing.assert_array_equal((status & 1).astype(np.uint8), ref.status)
    s = ref.status == 1
    err = np.abs(best[s].astype(np.float64) - ref.best[s])
    err2 = np.abs(second[s].astype(np.float64) - ref.second[s])
    assert err.max() <= SCORE_TOL, f"best score error {err.max():.3g}"
    assert err2.max() <= SCORE_TOL, f"second score error {err2.max():.3g}"
    same = np.all(mi == ref.match, axis=1)[s]
    gap = (ref.best.astype(np.float64) - ref.second)[s]
    clear = gap > GAP
    assert np.all(same[clear]), f"{np.sum(~same[clear])} blocks with a clear gap moved"
    assert same.mean() >= 0.995, f"argmax agreement {same.mean():.4f}"
    if c["nw"] <= 7 and bw == 4:
        assert diag[4] > 0, "no block took the tensor-core search"
    print(f"{c['id']} {store}: {s.sum()} blocks, tensor {diag[4]}, direct {diag[5]}, "
          f"max |d best| {err.max():.2e}, argmax agreement {same.mean():.5f}")


@pytest.mark.parametrize("store", ["bf16", "f16"])
@pytest.mark.parametrize("mode,kind,bw,nw,keep,shape,levels", [
    ("symmetric", "affine", 4, 7, 1.0, (72, 64, 48), 2),
    ("classic", "rigid", 4, 7, 1.0, (72, 64, 48), 2),
    # block width 5, window 11, 30 % kept (the large stress configuration's
    # search), one level of a volume where the registration converges
    ("symmetric", "affine", 5, 11, 0.3, (96, 88, 64), 1)])
def test_register16_matches_oracle(ctx, store, mode, kind, bw, nw, keep, shape, levels):
    ph = make_phantom(shape, n_gauss=20, kind=kind, seed=41 if kind == "affine" else 42,
                      max_angle_deg=4.0, max_shift_vox=4.0)
    rp = O.RegParams(mode, kind, 4, O.BMParams(bw, 1, 3, nw, keep), 0.5, store)
    fixed = O.Image(ph.fixed, ph.spacing, ph.origin)
    moving = O.Image(ph.moving, ph.spacing, ph.origin)
    to = O.register(fixed, moving, rp, levels)
    p = mb.reg_params(symmetric=mode == "symmetric", kind=kind, levels=levels, iterations=4,
                      block_width=bw, nhood_gap=3, nhood_width=nw, block_keep=keep,
                      storage=store)
    tg, st = mb.register(ctx, ph.fixed, ph.moving, p)
    assert st.levels_run == levels and st.block_ncc_evaluated > 0
    # the host copies carried 2 bytes per voxel
    assert st.h2d_bytes >= 2 * 2 * ph.fixed.size
    dM = np.max(np.abs(tg.M - to.M))
    err = tre(tg.M, tg.off, ph.true_matrix, ph.true_offset, shape, ph.spacing)
    err_o = tre(to.M, to.off, ph.true_matrix, ph.true_offset, shape, ph.spacing)
    print(f"{mode} {kind} {store}: max |dM| {dM:.2e}, TRE gpu {err:.4f} oracle {err_o:.4f}")
    np.testing.assert_allclose(tg.M, to.M, atol=1e-4, rtol=0)
    np.testing.assert_allclose(tg.off, to.off, atol=1e-3, rtol=0)


def test_register16_large_config_slab_matches_oracle(ctx):
    """The large stress configuration's settings (FP16 storage, block 5,
    radius 5, 30 % of blocks kept, symmetric affine, LTS keep 0.5) on a
    112x104x64 slab cropped from the centre of its 512x512x256 phantom pair
    (GPU-generated from seed 4000 with the quadratic +-20 % bias field, the
    first pair the large-configuration benchmark times).  Both slabs keep the
    crop's physical origin, so they stay related by the phantom's transform.
    The registration (one level, 4 iterations) must equal the FP64 oracle's on
    the same stored values: matrices within 1e-4, offsets within 1e-3 mm."""
    from mirorr_b200.phantom import make_phantom_gpu
    full = (512, 512, 256)
    ph = make_phantom_gpu(full, n_gauss=200, kind="affine", seed=4000, bias=0.2,
                          max_angle_deg=8.0, max_shift_vox=12.0)
    sx, sy, sz = 112, 104, 64
    x0, y0, z0 = (full[0] - sx) // 2, (full[1] - sy) // 2, (full[2] - sz) // 2
    fixed = np.ascontiguousarray(ph.fixed[z0:z0 + sz, y0:y0 + sy, x0:x0 + sx])
    moving = np.ascontiguousarray(ph.moving[z0:z0 + sz, y0:y0 + sy, x0:x0 + sx])
    origin = np.array([x0, y0, z0], np.float64)
    spacing = np.ones(3)
    rp = O.RegParams("symmetric", "affine", 4, O.BMParams(5, 1, 3, 11, 0.3), 0.5, "f16")
    to = O.register(O.Image(fixed, spacing, origin), O.Image(moving, spacing, origin), rp, 1)
    p = mb.reg_params(symmetric=True, kind="affine", levels=1, iterations=4, block_width=5,
                      nhood_gap=3, nhood_width=11, block_keep=0.3, lts_keep=0.5, storage="f16")
    fs, ms = mb.to_storage(fixed, "f16"), mb.to_storage(moving, "f16")
    tg, st = mb.register(ctx, fs, ms, p, fixed_geom=mb.Geometry.of(fs, spacing, origin),
                         moving_geom=mb.Geometry.of(ms, spacing, origin))
    assert st.levels_run == 1 and st.block_ncc_evaluated > 0
    dM = np.max(np.abs(tg.M - to.M))
    print(f"large-configuration slab: max |dM| {dM:.2e}, max |d offset| "
          f"{np.max(np.abs(tg.off - to.off)):.2e}")
    np.testing.assert_allclose(tg.M, to.M, atol=1e-4, rtol=0)
    np.testing.assert_allclose(tg.off, to.off, atol=1e-3, rtol=0)
