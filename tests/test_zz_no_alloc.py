"""GPU test of molints_eri_packed_noalloc, the entry point for callers that cannot allocate
device memory where they need integrals (code running under CUDA stream capture, where
cudaMalloc is not allowed, or frameworks whose allocator owns the whole GPU).

It is called through the C ABI twice in a row, on two different molecules, and each result
is compared with molints_eri_packed's (every primitive pair kept, as the noalloc path does)
within the FP64 tolerance of the other parity tests.  This file sorts last so that a run
stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def test_noalloc_matches_eri_packed_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    lib = engine.load_library()
    eng = engine.Engine(0)
    err = ctypes.create_string_buffer(256)
    try:
        for sh in (mi.config2(), mi.config0()):
            arrs = engine._BasisArrays(sh)
            opts = engine.make_options()
            out = torch.full((sh.npacked,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            stream = torch.cuda.current_stream().cuda_stream
            rc = lib.molints_eri_packed_noalloc(ctypes.byref(arrs.c), ctypes.byref(opts),
                                                ctypes.c_void_p(out.data_ptr()),
                                                ctypes.c_void_p(stream), err, len(err))
            assert rc == 0, err.value
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            ref = eng.eri_packed(sh, prim_cutoff=0.0)
            assert not np.isnan(got).any()
            assert np.max(np.abs(got - ref)) < TOL_FP64
    finally:
        eng.close()


def test_noalloc_rejects_oversize_basis():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    lib = engine.load_library()
    sh = mi.config1()
    big = mi.Shells.from_list(
        [(sh.xyz[s] + 40.0 * k, int(sh.L[s]),
          list(zip(sh.expn[sh.prim_off[s]:sh.prim_off[s] + sh.nprim[s]],
                   sh.coef[sh.prim_off[s]:sh.prim_off[s] + sh.nprim[s]])))
         for k in range(4) for s in range(sh.nshell)])
    arrs = engine._BasisArrays(big)
    err = ctypes.create_string_buffer(256)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = lib.molints_eri_packed_noalloc(ctypes.byref(arrs.c), None, ctypes.c_void_p(out.data_ptr()),
                                        None, err, len(err))
    assert rc == -2
    assert b"at most" in err.value
