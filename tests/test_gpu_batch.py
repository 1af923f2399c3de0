"""Batched and served registrations (mirorr_batch_*) through the C ABI.

A request's result must be the same alone and in a mix of requests of other
sizes, methods and transform kinds: the batch runs the same kernels on each
request's own buffers, so the only differences allowed are the order of the
LTS fit's FP64 sums (a group of CTAs per request instead of the whole GPU),
bounded here at 1e-9 on the matrices.  Each is also checked against the
single-request path (mirorr_register with the same 16-bit storage).
Admission (slots, memory budget), cancellation, malformed requests and failed
requests are exercised on the host side; nothing faults a GPU.
"""
import numpy as np
import pytest

import mirorr_b200 as mb
from mirorr_b200.phantom import make_phantom

pytestmark = pytest.mark.gpu

REQS = [
    dict(shape=(72, 64, 48), mode="symmetric", kind="affine", seed=51, levels=2),
    dict(shape=(64, 80, 40), mode="classic", kind="rigid", seed=52, levels=2),
    dict(shape=(96, 72, 56), mode="symmetric", kind="rigid", seed=53, levels=2),
    dict(shape=(80, 64, 48), mode="classic", kind="affine", seed=54, levels=1),
]


def _req(r, store="bf16"):
    ph = make_phantom(r["shape"], n_gauss=16, kind=r["kind"], seed=r["seed"], max_angle_deg=4.0,
                      max_shift_vox=4.0)
    p = mb.reg_params(symmetric=r["mode"] == "symmetric", kind=r["kind"], levels=r["levels"],
                      iterations=4, nhood_gap=3, nhood_width=7, storage=store)
    return ph, p


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_equals_single_requests(ctx, graphs):
    singles = []
    for r in REQS:
        ph, p = _req(r)
        singles.append(mb.register(ctx, ph.fixed, ph.moving, p)[0])
    b = mb.Batch(ctx, max_slots=8, hbm_budget=8e9)
    b.set_graphs(graphs)
    ids = []
    for r in REQS:
        ph, p = _req(r)
        ids.append(b.submit(ph.fixed, ph.moving, p))
    b.run()
    info = b.info()
    assert info["running"] == 0 and info["finished"] == len(REQS)
    for rid, t1 in zip(ids, singles):
        t, st = b.result(rid)
        np.testing.assert_allclose(t.M, t1.M, atol=1e-9, rtol=0)
        np.testing.assert_allclose(t.off, t1.off, atol=1e-7, rtol=0)
        assert st.matcher_calls > 0 and st.block_ncc_evaluated > 0
    if graphs:
        assert info["replays"] > 0
    b.close()


def test_batch_block_width5_keep_fraction(ctx):
    """Block width 5, window 11, 30 % of the blocks kept (the large stress
    configuration's search at small size): the batch runs the variance
    selection of every call on its resampled base image; each request's
    result equals the single-request path's."""
    reqs = [dict(shape=(72, 64, 48), mode="symmetric", kind="affine", seed=61, levels=2),
            dict(shape=(64, 80, 40), mode="classic", kind="rigid", seed=62, levels=2)]
    singles, subs = [], []
    for r in reqs:
        ph = make_phantom(r["shape"], n_gauss=16, kind=r["kind"], seed=r["seed"], max_angle_deg=4.0,
                          max_shift_vox=4.0)
        p = mb.reg_params(symmetric=r["mode"] == "symmetric", kind=r["kind"], levels=r["levels"],
                          iterations=4, block_width=5, nhood_gap=3, nhood_width=11, block_keep=0.3,
                          storage="f16")
        singles.append(mb.register(ctx, ph.fixed, ph.moving, p)[0])
        subs.append((ph, p))
    b = mb.Batch(ctx, max_slots=4, hbm_budget=8e9)
    ids = [b.submit(ph.fixed, ph.moving, p) for ph, p in subs]
    b.run()
    for rid, t1 in zip(ids, singles):
        t, st = b.result(rid)
        np.testing.assert_allclose(t.M, t1.M, atol=1e-9, rtol=0)
        np.testing.assert_allclose(t.off, t1.off, atol=1e-7, rtol=0)
        assert st.block_ncc_evaluated > 0
    b.close()


def test_batch_alone_equals_in_the_mix(ctx):
    """Continuous batching: request 0 runs alone; then again while others are
    admitted between its steps.  Its result must not change."""
    ph0, p0 = _req(REQS[0])
    b = mb.Batch(ctx, max_slots=4, hbm_budget=8e9)
    r = b.submit(ph0.fixed, ph0.moving, p0)
    b.run()
    alone, _ = b.result(r)
    r = b.submit(ph0.fixed, ph0.moving, p0)
    b.step()
    others = []
    for q in REQS[1:]:
        ph, p = _req(q)
        others.append(b.submit(ph.fixed, ph.moving, p))
        b.step()
    b.run()
    mixed, _ = b.result(r)
    for o in others:
        b.result(o)
    np.testing.assert_allclose(mixed.M, alone.M, atol=1e-12, rtol=0)
    np.testing.assert_allclose(mixed.off, alone.off, atol=1e-10, rtol=0)
    b.close()


def test_batch_admission_and_failures(ctx):
    ph, p = _req(REQS[0])
    # the memory one request of this size reserves
    b = mb.Batch(ctx, max_slots=4, hbm_budget=8e9)
    b.submit(ph.fixed, ph.moving, p)
    one = b.info()["bytes_reserved"]
    assert one > 0
    b.close()
    # a budget that holds one request of this size but not two
    b = mb.Batch(ctx, max_slots=4, hbm_budget=int(1.5 * one))
    r1 = b.submit(ph.fixed, ph.moving, p)
    with pytest.raises(mb.MirorrError) as e:
        b.submit(ph.fixed, ph.moving, p)
    assert e.value.name == "EBUSY"
    b.cancel(r1)  # frees the slot and the memory
    r2 = b.submit(ph.fixed, ph.moving, p)
    b.run()
    b.result(r2)
    # larger than the whole budget: refused for good
    big, pb = _req(dict(shape=(160, 160, 96), mode="symmetric", kind="affine", seed=9, levels=2))
    with pytest.raises(mb.MirorrError) as e:
        b.submit(big.fixed, big.moving, pb)
    assert e.value.name == "ERANGE"
    b.close()
    b = mb.Batch(ctx, max_slots=1, hbm_budget=8e9)
    b.submit(ph.fixed, ph.moving, p)
    with pytest.raises(mb.MirorrError) as e:  # no free slot
        b.submit(ph.fixed, ph.moving, p)
    assert e.value.name == "EBUSY"
    b.close()
    b = mb.Batch(ctx, max_slots=2, hbm_budget=8e9)
    # malformed: a volume smaller than one block / FP32 storage
    tiny = np.zeros((2, 2, 2), np.float32)
    with pytest.raises(mb.MirorrError) as e:
        b.submit(tiny, tiny, p)
    assert e.value.name == "EINVAL"
    p32 = mb.reg_params(symmetric=True, kind="affine", levels=2, storage="f32")
    with pytest.raises(mb.MirorrError) as e:
        b.submit(ph.fixed, ph.moving, p32)
    assert e.value.name == "EINVAL"
    # a request with no overlap fails alone (ENOBLOCKS), the other finishes
    flat = np.full(ph.fixed.shape, 0.5, np.float32)
    bad = b.submit(flat, flat, p)
    good = b.submit(ph.fixed, ph.moving, p)
    b.run()
    with pytest.raises(mb.MirorrError) as e:
        b.result(bad)
    assert e.value.name == "ENOBLOCKS"
    b.result(good)
    b.close()
