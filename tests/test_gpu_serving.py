"""GPU tests of the serving API (molints_submit / poll / result / release): results in a mix of
concurrent requests equal the same molecule computed alone, admission follows the HBM
budget, and release / stop behave."""
import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    e = engine.Engine(0)
    yield e
    e.close()


def _f_molecule(seed, nheavy=2, nh=2):
    return mi.basis.synthetic_molecule(seed, nheavy, nh, mi.basis.POLARISED_C, mi.basis.POLARISED_H,
                                       0.1, 1e4, f"fmol{seed}", heavy_extra=[(3, 1)])


def _mix():
    return [mi.config2(), mi.config0(), _f_molecule(21), mi.config4_request(6), _f_molecule(22, 1, 3),
            mi.config1(), mi.build_basis(mi.h2()), mi.config4_request(7)]


def test_results_equal_alone_and_in_the_mix(eng):
    """All requests submitted at once to 4 slots (their plans run concurrently and their
    kernels overlap): each result is bit-identical to the molecule computed alone."""
    from molints_b200 import engine
    mols = _mix()
    alone = [eng.eri_packed(sh) for sh in mols]
    srv = engine.Engine(0)
    try:
        srv.serve_start(nslots=4)
        reqs = [srv.submit(sh) for sh in mols] + [srv.submit(sh) for sh in mols[:3]]
        for r in reqs:
            assert r.poll(timeout_ms=120000)
        for k, r in enumerate(reqs):
            got = r.result()
            assert np.array_equal(got, alone[k % len(mols)]), k
        infos = [r.info() for r in reqs]
        assert len({i["slot"] for i in infos}) > 1
        # some requests were admitted while others were still running
        assert any(b["t_admit"] < a["t_done"] for a in infos for b in infos if a is not b)
        st = srv.serve_stats()
        assert st["done"] == len(reqs) and st["failed"] == 0 and st["queued"] == 0
        for r in reqs:
            r.release()
        assert srv.serve_stats()["ledger_bytes"] == 0
    finally:
        srv.close()


def test_mixed_precision_requests(eng):
    from molints_b200 import engine
    sh = mi.config2()
    ref = eng.eri_packed(sh)
    srv = engine.Engine(0)
    try:
        srv.serve_start(nslots=2)
        r = srv.submit(sh, precision=engine.MIXED, fp32_cutoff=1e-3)
        assert r.poll(-1)
        assert np.max(np.abs(r.result() - ref)) < 1e-9
        r.release()
    finally:
        srv.close()


def test_budget_admission_and_refusal(eng):
    """With room for one request at a time, each request is admitted only after the previous
    one was released; a request larger than the budget fails with MOLINTS_ERR_BUDGET."""
    from molints_b200 import engine
    sh = mi.config2()
    need = sh.npacked * 8
    srv = engine.Engine(0)
    try:
        srv.serve_start(nslots=4, hbm_budget_bytes=need + (12 << 20))
        big = srv.submit(mi.config1())
        with pytest.raises(engine.MolintsError) as e:
            big.poll(0)
        assert e.value.status == -3
        big.release()
        reqs = [srv.submit(sh) for _ in range(3)]
        ref = eng.eri_packed(sh)
        times = []
        for r in reqs:
            assert r.poll(timeout_ms=60000)
            assert np.array_equal(r.result(), ref)
            times.append(r.info())
            r.release()
        for a, b in zip(times, times[1:]):
            assert b["t_admit"] >= a["t_done"] - 1e-6
    finally:
        srv.close()


def test_release_queued_and_stop(eng):
    from molints_b200 import engine
    srv = engine.Engine(0)
    srv.serve_start(nslots=1)
    reqs = [srv.submit(mi.config2()) for _ in range(4)]
    reqs[3].release()  # withdrawn while queued (or freed when it finishes)
    assert reqs[0].poll(60000)
    srv.serve_stop()  # queued ones fail, finished results stay valid
    assert reqs[0].result().shape == (mi.config2().npacked,)
    for r in reqs[:3]:
        try:
            r.poll(0)
        except engine.MolintsError:
            pass
        r.release()
    srv.close()
