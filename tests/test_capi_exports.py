"""The C ABI library loads and exports every entry point include/mirorr_b200.h
declares; without a GPU it fails loudly instead of falling back to the CPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "mirorr_b200.h")).read()
    return sorted(set(re.findall(r"MIRORR_API\s+[\w\s\*]+?\b(mirorr_\w+)\s*\(", hdr)))


@pytest.fixture(scope="module")
def so():
    from mirorr_b200 import build as mb_build
    return ctypes.CDLL(mb_build.build())


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ["mirorr_bm_get_offsets", "mirorr_bm_set_base_image", "mirorr_bm_swap_image_order",
              "mirorr_register", "mirorr_resample", "mirorr_lts_classic", "mirorr_lts_symmetric"]:
        assert s in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(so):
    missing = [s for s in declared_symbols() if not hasattr(so, s)]
    assert not missing, missing


def test_abi_version(so):
    so.mirorr_abi_version.restype = ctypes.c_int32
    assert so.mirorr_abi_version() == 2


def test_no_gpu_fails_loudly(so):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    so.mirorr_ctx_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    st = so.mirorr_ctx_create(0, ctypes.byref(h))
    assert st == 4  # MIRORR_ECUDA
    so.mirorr_last_error.restype = ctypes.c_char_p
    assert b"device" in so.mirorr_last_error().lower()


def test_python_binding_raises_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import mirorr_b200 as mb
    with pytest.raises(mb.MirorrError) as e:
        mb.Context(0)
    assert e.value.name == "ECUDA"


def test_params_validation_without_gpu(so):
    import mirorr_b200 as mb
    p = mb.BMParams()
    assert mb.lib().mirorr_bm_default_params(ctypes.byref(p)) == 0
    assert (p.block_width, p.block_gap, p.nhood_gap, p.nhood_width) == (4, 1, 2, 5)
    assert p.portion_matches_kept == 0.5
    r = mb.RegParams()
    assert mb.lib().mirorr_reg_default_params(ctypes.byref(r)) == 0
    assert (r.bm.nhood_gap, r.bm.nhood_width, r.iterations, r.symmetric) == (3, 7, 5, 1)


def test_pyramid_schedule_host_logic_matches_oracle():
    import numpy as np
    import mirorr_b200 as mb
    from oracle import oracle as O
    for size in [(128, 128, 64), (256, 256, 128), (512, 512, 256), (96, 96, 48), (320, 200, 160)]:
        g = mb.Geometry.make(size)
        ms, fs = mb.pyramid_schedule(g, g)
        oms, ofs = O.pyramid_schedule(size, size, np.ones(3), np.ones(3))
        np.testing.assert_array_equal(ms, oms)
        np.testing.assert_array_equal(fs, ofs)
    gf = mb.Geometry.make((200, 180, 60), spacing=(1.0, 1.0, 3.0))
    gm = mb.Geometry.make((256, 256, 120), spacing=(0.8, 0.8, 1.5))
    ms, fs = mb.pyramid_schedule(gf, gm, 32, 0)
    oms, ofs = O.pyramid_schedule((200, 180, 60), (256, 256, 120), np.array([1, 1, 3.0]),
                                  np.array([0.8, 0.8, 1.5]))
    np.testing.assert_array_equal(ms, oms)
    np.testing.assert_array_equal(fs, ofs)
