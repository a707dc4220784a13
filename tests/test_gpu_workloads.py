"""GPU parity on the benchmark workloads' own molecules: molecules of the 256-molecule batch
(seeds 3000+m, from its first eight, those under 150 functions) and requests of the serving
stream (l <= 3, with f shells), through the library's default per-class table (the tuned
HGP/Rys choice) and through the serving API, against the long-double restatement of the
reference HGP (src/HGP.jl:22-242, all_twoe_ints layout) in the engine's pair orientation, with
the exact Boys function on both sides.

Bars (max abs, Eh): FP64 within 1e-12 plus the basis's FP64 floor (twice the FP64
restatement's own error against the long-double value); MIXED within 1e-9.  Each test prints
the floor and the errors it measured."""
import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-9

BATCH_MOLECULES = (6, 4, 2, 1, 0)        # 39, 67, 82, 130 and 134 functions
SERVING_REQUESTS = (31, 9, 20, 6)        # 40 (f), 50, 105 (f) and 115 (f) functions


@pytest.fixture(scope="module")
def eng():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    e = engine.Engine(0)
    yield e
    e.close()


_CACHE = {}


def _oracle_pair(oracle, sh):
    """(long-double value, FP64 floor) in the engine's orientation with exact Boys."""
    if sh.name not in _CACHE:
        with oracle.exact_boys(), oracle.stable_orientation():
            ld = oracle.eri_packed_hgp_ld(sh, nthreads=0)
            f64 = oracle.eri_packed_hgp(sh, nthreads=0)
        _CACHE[sh.name] = (ld, 2.0 * float(np.max(np.abs(f64 - ld))))
    return _CACHE[sh.name]


def _check(eng, sh, ld, floor, label, fp32_cut):
    from molints_b200 import engine
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    err64 = float(np.max(np.abs(got - ld)))
    mixed = eng.eri_packed(sh, boys=engine.BOYS_EXACT, precision=engine.MIXED, fp32_cutoff=fp32_cut)
    errmx = float(np.max(np.abs(mixed - ld)))
    # every FP32 variant enabled (not only those the default table keeps)
    eng.set_class_methods({k: v & ~engine.CLASS_NO_FP32 for k, v in eng.class_methods().items()})
    try:
        all32, st = eng.eri_packed(sh, boys=engine.BOYS_EXACT, precision=engine.MIXED,
                                   fp32_cutoff=fp32_cut, with_stats=True)
    finally:
        eng.set_class_methods(None)
    err32 = float(np.max(np.abs(all32 - ld)))
    print(f"{label}: nbf {sh.nbf}, {sh.npacked} integrals; floor {floor:.2e}; |FP64 - oracle| "
          f"{err64:.2e}; |MIXED - oracle| {errmx:.2e} (default table), {err32:.2e} (every FP32 "
          f"variant, {st['n_fp32_quartets']} FP32 quartets in {st['n_fp32_launches']} launches)")
    assert err64 < TOL_FP64 + floor, (label, err64, floor)
    assert errmx < TOL_MIXED and err32 < TOL_MIXED, (label, errmx, err32)
    return got


@pytest.mark.parametrize("m", BATCH_MOLECULES)
def test_batch_molecule_against_oracle(eng, oracle, m):
    sh = mi.config3_molecule(m)
    ld, floor = _oracle_pair(oracle, sh)
    _check(eng, sh, ld, floor, f"batch molecule {m}", 1e-5)


@pytest.mark.parametrize("r", SERVING_REQUESTS)
def test_serving_request_against_oracle(eng, oracle, r):
    from molints_b200 import engine
    sh = mi.config4_request(r)
    ld, floor = _oracle_pair(oracle, sh)
    _check(eng, sh, ld, floor, f"serving request {r}", 1e-5)


def test_served_requests_against_oracle(oracle):
    """The same requests through the serving API (submitted together to two slots, default
    table): every result within the FP64 bar of the oracle."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    srv = engine.Engine(0)
    try:
        srv.serve_start(nslots=2, hbm_budget_bytes=8 * 2**30)
        mols = [mi.config4_request(r) for r in SERVING_REQUESTS]
        reqs = [srv.submit(sh, boys=engine.BOYS_EXACT) for sh in mols]
        for r, sh, req in zip(SERVING_REQUESTS, mols, reqs):
            assert req.poll(-1)
            got = req.result()
            req.release()
            ld, floor = _oracle_pair(oracle, sh)
            err = float(np.max(np.abs(got - ld)))
            print(f"served request {r}: floor {floor:.2e}, |FP64 - oracle| {err:.2e}")
            assert err < TOL_FP64 + floor, (r, err, floor)
    finally:
        srv.close()
