"""GPU test of molints_eri_packed_noalloc, the entry point for callers that cannot allocate
device memory where they need integrals: host programs whose own allocator has reserved the
GPU's memory, and time-critical loops that cannot take the synchronisation a cudaMalloc may
cause.

It is called through the C ABI twice in a row, on two different molecules, and each result is
compared with molints_eri_packed's (every primitive pair kept, as the noalloc path does) within
the FP64 tolerance of the other parity tests, and with the CPU oracle.  The device's free
memory is the same before and after the two calls: the calls allocate nothing.  This file sorts
last so that a run stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _noalloc(lib, sh, out, err):
    import torch
    from molints_b200 import engine
    arrs = engine._BasisArrays(sh)
    opts = engine.make_options()
    stream = torch.cuda.current_stream().cuda_stream
    return lib.molints_eri_packed_noalloc(ctypes.byref(arrs.c), ctypes.byref(opts),
                                          ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream),
                                          err, len(err))


def test_noalloc_matches_eri_packed_twice(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    lib = engine.load_library()
    err = ctypes.create_string_buffer(256)
    mols = (mi.config2(), mi.config0())
    # references first: the engine's own plans allocate from its memory pool
    eng = engine.Engine(0)
    try:
        refs = [eng.eri_packed(sh, prim_cutoff=0.0) for sh in mols]
    finally:
        eng.close()
    with oracle.stable_orientation():
        orc = [oracle.eri_packed_hgp_ld(sh, nthreads=0) for sh in mols]
    outs = [torch.full((sh.npacked,), float("nan"), dtype=torch.float64, device="cuda") for sh in mols]
    warm = torch.empty(max(sh.npacked for sh in mols), dtype=torch.float64, device="cuda")
    # the first call on the device does the one-time set-up; the warm-up over both molecules
    # also has the driver load the code of every class kernel they use (modules load lazily,
    # and loading code takes device memory that is not the entry point's)
    for sh in mols:
        assert _noalloc(lib, sh, warm, err) == 0, err.value
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for sh, out in zip(mols, outs):
        rc = _noalloc(lib, sh, out, err)
        assert rc == 0, err.value
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free1 - free0) < 2 * 2**20, (free0, free1)
    for sh, out, ref, ld in zip(mols, outs, refs, orc):
        got = out.cpu().numpy()
        assert not np.isnan(got).any()
        assert np.max(np.abs(got - ref)) < TOL_FP64
        assert np.max(np.abs(got - ld)) < TOL_FP64


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
