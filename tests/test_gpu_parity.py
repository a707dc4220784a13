"""GPU parity: libmolints_cuda.so (through its C ABI) against the CPU oracle.

Tolerances (max abs, Eh): FP64 path 1e-12 against the restated reference HGP with the same
Boys branch; mixed precision 1e-9 against the FP64 oracle."""
import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-9


@pytest.fixture(scope="module")
def eng():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    e = engine.Engine(0)
    yield e
    e.close()


def _rand_basis(seed, lmax, natom=3, kmax=3, lo=0.15, hi=20.0):
    rng = np.random.default_rng(seed)
    lst = []
    for _ in range(natom):
        xyz = rng.uniform(-2.0, 2.0, 3)
        for l in range(lmax + 1):
            for _ in range(int(rng.integers(1, 3))):
                lst.append((xyz, l, mi.basis._random_shell(rng, l, int(rng.integers(1, kmax + 1)), lo, hi)))
    return mi.Shells.from_list(lst, f"rand{seed}")


def test_boys_table_against_oracle(eng, oracle):
    from molints_b200 import engine
    T = np.concatenate([np.linspace(0, 45, 1441), [1e-20, 1e-12, 29.999999, 30.0, 39.9999, 40.0, 60, 200]])
    for mmax in (1, 3, 9, 13):
        got = eng.boys(mmax, T, engine.BOYS_EXACT)
        for t, row in zip(T[::7], got[::7]):
            for m in range(mmax):
                ex = oracle.boys_mpmath(m, t) if t < 40 else oracle.boys(m, t)
                # beyond T = 40 the asymptotic form omits terms below e^-T / (2T) ~ 5e-20
                atol = 0.0 if t < 40 else np.exp(-t) / t
                assert abs(row[m] - ex) <= 4e-15 * ex + atol, (mmax, m, t)
        ref = eng.boys(mmax, T, engine.BOYS_REFERENCE)
        for t, row in zip(T, ref):
            np.testing.assert_allclose(row, oracle.farray(mmax, t), rtol=5e-15, atol=0)


def test_h2_sto3g_golden(eng, golden, oracle):
    ints = eng.eri_packed(mi.build_basis(mi.h2()))
    idx = {"llll": (0, 0, 0, 0), "rrrr": (1, 1, 1, 1), "llrr": (0, 0, 1, 1),
           "lllr": (0, 0, 0, 1), "lrlr": (0, 1, 0, 1)}
    for key, case in golden["h2_sto3g_coulomb"].items():
        assert ints[oracle.iindex(*idx[key])] == pytest.approx(case["value"], rel=1.5e-8)


def test_ethane_sto3g_matches_reference_hgp(eng, oracle):
    sh = mi.config0()
    got = eng.eri_packed(sh)
    ref = oracle.eri_packed_hgp(sh, nthreads=8)
    huz = oracle.eri_packed_huzinaga(sh, nthreads=8)
    assert got.shape == (9316,)
    assert np.max(np.abs(got - ref)) < TOL_FP64
    assert np.max(np.abs(got - huz)) < TOL_FP64


# FP64 parity.  The reference algorithm (HGP, restated by the oracle) is evaluated in long
# double as the near-exact value; the FP64 GPU path must be within 1e-12 Eh of it.  The same
# algorithm in FP64 -- the reference's own arithmetic -- is itself up to ~2.4e-12 (config 1)
# and ~1.1e-11 (config 2, in the reference's quartet orientation) from that value: tight
# primitives (exponents to 1e4) with random-sign contractions cancel, and the reference
# orients (p d| pairs with the diffuse shell first, which the HRR amplifies.  Against the
# FP64 oracle the GPU is therefore checked within that oracle's own measured error.


def _fp64_oracle_bound(oracle, sh, ld):
    ref = oracle.eri_packed_hgp(sh, nthreads=8)
    return ref, float(np.max(np.abs(ref - ld)))


def test_ethane_polarised_all_classes(eng, oracle):
    """Config 2 (l<=2, every class pair up to (dd|dd)), both Boys modes."""
    from molints_b200 import engine
    sh = mi.config2()
    got = eng.eri_packed(sh)
    ld = oracle.eri_packed_hgp_ld(sh, nthreads=8)
    assert np.max(np.abs(got - ld)) < TOL_FP64
    ref, own = _fp64_oracle_bound(oracle, sh, ld)
    assert np.max(np.abs(got - ref)) < own + TOL_FP64
    got_x = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    with oracle.exact_boys():
        ld_x = oracle.eri_packed_hgp_ld(sh, nthreads=8)
    assert np.max(np.abs(got_x - ld_x)) < TOL_FP64


def test_split_valence_24_full(eng, oracle):
    """Config 1 at full size: all 14,908,530 integrals against the long-double oracle, and
    the Schwarz inequality over the whole vector."""
    sh = mi.config1()
    got = eng.eri_packed(sh)
    assert got.shape == (14908530,)
    ld = oracle.eri_packed_hgp_ld(sh, nthreads=0)
    assert np.max(np.abs(got - ld)) < TOL_FP64
    n = sh.nbf
    npair = n * (n + 1) // 2
    diag = got[np.arange(npair) * (np.arange(npair) + 1) // 2 + np.arange(npair)]
    assert np.all(diag >= -1e-14)
    ij = np.repeat(np.arange(npair), np.arange(1, npair + 1))
    kl = np.arange(len(got)) - ij * (ij + 1) // 2
    bound = np.sqrt(np.abs(diag[ij] * diag[kl]))
    # each value carries up to the parity tolerance, so equality cases may exceed by that much
    excess = np.abs(got) - bound * (1 + 1e-10)
    assert excess.max() < TOL_FP64, (excess.max(), int(np.argmax(excess)))


def test_auto_output_falls_back_to_direct_under_budget():
    """AUTO takes the two-phase output for a large molecule (2^25+ integrals), whose scratch is
    about as large as the output.  Under an HBM budget that the scratch does not fit, AUTO plans
    still succeed with the direct stores (the same vector bit for bit); an explicit TWO_PHASE
    plan fails with MOLINTS_ERR_BUDGET."""
    import torch
    from molints_b200 import engine
    sh = mi.config3_molecule(0)  # 134 functions, 40.9 M integrals (327 MB)
    assert sh.npacked >= 1 << 25
    small = engine.Engine(0, hbm_budget_bytes=150 * 2**20)
    big = engine.Engine(0)
    outs = []
    try:
        for e, mode in ((small, engine.OUTPUT_AUTO), (big, engine.OUTPUT_DIRECT)):
            e.set_stream(torch.cuda.current_stream().cuda_stream)
            plan = e.plan(sh, output=mode)
            out = torch.full((sh.npacked,), float("nan"), dtype=torch.float64, device="cuda")
            plan.execute(out.data_ptr())
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy())
            plan.close()
            e.set_stream(None)
        with pytest.raises(engine.MolintsError) as ex:
            small.plan(sh, output=engine.OUTPUT_TWO_PHASE)
        assert ex.value.status == -3
    finally:
        small.close()
        big.close()
    assert not np.isnan(outs[0]).any() and np.array_equal(outs[0], outs[1])


def test_two_phase_output_equals_direct(eng):
    """The two-phase output (quartet blocks into a class-major scratch, then the packed vector
    gathered in order) gives the direct path's vector bit for bit: HGP and Rys classes (an f
    molecule), FP64, MIXED and MIXED with quartet screening (whose two-phase plans order the
    pairs by Schwarz factor and leave the screened quartets to the gather), a batch plan over
    several molecules, every entry written (NaN sentinel), and J/K digested from a two-phase
    plan."""
    import torch
    from molints_b200 import engine
    TP, DIR = engine.OUTPUT_TWO_PHASE, engine.OUTPUT_DIRECT
    for sh in (mi.config2(), _f_molecule(7), _rand_basis(105, 2)):
        for prec, cut, scut in ((engine.FP64, 0.0, 0.0), (engine.MIXED, 1e-3, 0.0), (engine.MIXED, 1e-3, 1e-8)):
            a = eng.eri_packed(sh, precision=prec, fp32_cutoff=cut, screen_cutoff=scut, output=DIR)
            b = eng.eri_packed(sh, precision=prec, fp32_cutoff=cut, screen_cutoff=scut, output=TP)
            assert np.array_equal(a, b)
            if scut > 0.0:
                assert (a == 0.0).sum() > 0
    mols = [mi.config2(), mi.config0(), _rand_basis(106, 2), _f_molecule(8), mi.config3_molecule(6)]
    for scut in (0.0, 1e-9):
        outs = []
        for mode in (DIR, TP):
            plan = eng.plan_batch(mols, output=mode, precision=engine.MIXED if scut else engine.FP64,
                                  fp32_cutoff=1e-3 if scut else 0.0, screen_cutoff=scut)
            out = torch.full((plan.npacked,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            eng.set_stream(torch.cuda.current_stream().cuda_stream)
            try:
                plan.execute(out.data_ptr())
                torch.cuda.synchronize()
            finally:
                eng.set_stream(None)
            outs.append(out.cpu().numpy())
            plan.close()
        assert not np.isnan(outs[1]).any() and np.array_equal(outs[0], outs[1])
    sh = _f_molecule(9)
    n = sh.nbf
    rng = np.random.default_rng(3)
    A = rng.normal(size=(n, n))
    D = torch.from_numpy((A + A.T) / n).cuda()
    res = []
    for mode in (DIR, TP):
        plan = eng.plan(sh, output=mode)
        J, K = torch.empty_like(D), torch.empty_like(D)
        plan.jk(D.data_ptr(), J.data_ptr(), K.data_ptr())
        torch.cuda.synchronize()
        res.append((J.cpu().numpy(), K.cpu().numpy()))
        plan.close()
    scale = max(1.0, np.abs(res[0][0]).max(), np.abs(res[0][1]).max())
    assert np.max(np.abs(res[0][0] - res[1][0])) < 1e-12 * scale
    assert np.max(np.abs(res[0][1] - res[1][1])) < 1e-12 * scale
    # AUTO takes the two-phase output above MOLINTS_TWO_PHASE_MIN (2^25) integrals, for a
    # batch plan and for one molecule, and keeps a smaller molecule direct
    big = [mi.config4_request(1), mi.config4_request(7)]
    total = sum(sh.npacked for sh in big)
    assert big[0].npacked >= 1 << 25 > big[1].npacked
    out = torch.empty(total, dtype=torch.float64, device="cuda")
    for mols, expect in ((big, True), (big[0], True), (big[1], False)):
        plan = eng.plan_batch(mols) if isinstance(mols, list) else eng.plan(mols)
        plan.set_profiling(True)
        plan.execute(out.data_ptr())
        torch.cuda.synchronize()
        assert ("gather_packed" in [n for n, _ in plan.launch_times()]) == expect
        plan.close()
    plan = eng.plan_batch(big)
    plan.execute(out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    plan.close()
    assert np.array_equal(got[:big[0].npacked], eng.eri_packed(big[0], output=DIR))
    assert np.array_equal(got[big[0].npacked:total], eng.eri_packed(big[1], output=DIR))


@pytest.mark.parametrize("seed,lmax", [(101, 0), (102, 1), (103, 2), (104, 2)])
def test_random_bases_against_huzinaga(eng, oracle, seed, lmax):
    from molints_b200 import engine
    sh = _rand_basis(seed, lmax)
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    huz = oracle.eri_packed_huzinaga(sh, nthreads=8)
    assert np.max(np.abs(got - huz)) < TOL_FP64 * max(1.0, np.max(np.abs(huz)))


def test_every_slot_written(eng):
    """A NaN-filled device output has no NaN left after one execute."""
    import torch
    sh = mi.config2()
    out = torch.full((sh.npacked,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    eng.eri_packed_device(sh, out.data_ptr())
    assert not torch.isnan(out).any().item()


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_mixed_precision_error_bound(eng, cfg):
    """The tuned FP32 cutoff keeps max |MIXED - FP64| below 1e-9 Eh and uses FP32."""
    from molints_b200 import autotune, engine
    sh = getattr(mi, cfg)()
    cut, table = autotune.tune_fp32_cutoff(eng, sh)
    assert cut > 0, table
    ref = eng.eri_packed(sh)
    # HGP everywhere with every FP32 variant enabled, so that FP32 kernels certainly run
    eng.set_class_methods({})
    try:
        got, st = eng.eri_packed(sh, precision=engine.MIXED, fp32_cutoff=cut, with_stats=True)
        plan = eng.plan(sh, precision=engine.MIXED, fp32_cutoff=cut)
        import torch
        out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
        plan.execute(out.data_ptr())
        pst = plan.stats()
        plan.close()
    finally:
        eng.set_class_methods(None)
    assert st["n_fp32_quartets"] > 0 and st["n_fp32_launches"] > 0, st
    assert pst["n_fp32_launches"] == st["n_fp32_launches"]
    assert np.max(np.abs(got - ref)) < TOL_MIXED
    # with the shipped default table, the stats count FP32 quartets only where FP32 kernels run
    _, st_def = eng.eri_packed(sh, precision=engine.MIXED, fp32_cutoff=cut, with_stats=True)
    assert (st_def["n_fp32_quartets"] > 0) == (st_def["n_fp32_launches"] > 0), st_def


def test_primitive_screening_bound(eng, oracle):
    """Dropping primitive pairs with b_i * max Qabs < 1e-18 changes no integral by more than
    1e-15, and removes a large share of config 1's primitive pairs."""
    sh = mi.config1()
    full, st0 = eng.eri_packed(sh, prim_cutoff=0.0, with_stats=True)
    scr, st1 = eng.eri_packed(sh, with_stats=True)
    assert st0["n_prim_pairs_kept"] == st0["n_prim_pairs"]
    assert st1["n_prim_pairs_kept"] < 0.7 * st1["n_prim_pairs"]
    assert np.max(np.abs(full - scr)) < 1e-15


def test_screening_writes_zeros(eng):
    sh = mi.config2()
    full = eng.eri_packed(sh)
    scr, st = eng.eri_packed(sh, screen_cutoff=1e-8, with_stats=True)
    assert st["n_screened"] > 0
    assert np.max(np.abs(scr - full)) < 1e-8


def test_deterministic(eng):
    sh = mi.config2()
    a = eng.eri_packed(sh)
    b = eng.eri_packed(sh)
    assert np.array_equal(a, b)


def test_contracted_schwarz_bounds(eng, oracle):
    sh = mi.config0()
    plan = eng.plan(sh)
    import torch
    out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
    plan.execute(out.data_ptr())
    q = plan.schwarz()
    ints = out.cpu().numpy()
    off = sh.fn_offsets()
    for i in range(sh.nshell):
        for j in range(i + 1):
            m = 0.0
            for a in range(off[i], off[i + 1]):
                for b in range(off[j], off[j + 1]):
                    m = max(m, abs(ints[oracle.iindex(a, b, a, b)]))
            assert q[i * (i + 1) // 2 + j] == pytest.approx(np.sqrt(m), rel=1e-13)
    plan.close()


def test_plan_execute_twice_on_torch_stream(eng, oracle):
    import torch
    sh = mi.config0()
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        plan = eng.plan(sh)
        out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
        plan.execute(out.data_ptr())
        first = out.cpu().numpy().copy()
        out.zero_()
        plan.execute(out.data_ptr())
        second = out.cpu().numpy()
        assert np.array_equal(first, second)
        q = plan.schwarz()
        assert q.shape == (sh.nshell * (sh.nshell + 1) // 2,) and np.all(q > 0)
        plan.close()
    finally:
        eng.set_stream(None)
    assert np.max(np.abs(first - oracle.eri_packed_hgp(sh))) < TOL_FP64


def test_batch_plan_equals_single_plans(eng):
    """Three molecules in one batch plan (one work queue per class pair across molecules)
    give each molecule's single-plan vector exactly, at its offset."""
    import torch
    mols = [mi.config2(), mi.config0(), _rand_basis(105, 2), _f_molecule(7)]
    plan = eng.plan_batch(mols)
    out = torch.full((plan.npacked,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        plan.execute(out.data_ptr())
    finally:
        eng.set_stream(None)
    got = out.cpu().numpy()
    assert not np.isnan(got).any()
    for m, sh in enumerate(mols):
        single = eng.eri_packed(sh)
        part = got[plan.offsets[m]:plan.offsets[m + 1]]
        assert np.array_equal(part, single), m
    st = plan.stats()
    assert st["n_eri"] == plan.npacked
    plan.close()


def test_edge_cases(eng):
    from molints_b200 import engine
    one = mi.Shells.from_list([((0.0, 0.0, 0.0), 0, [(1.0, 1.0)])])
    v = eng.eri_packed(one)
    assert v.shape == (1,) and v[0] == pytest.approx(2 / np.sqrt(np.pi) * np.sqrt(2.0 / 2), rel=1e-14)
    empty = mi.Shells.from_list([])
    assert eng.eri_packed(empty).shape == (0,)
    # a g shell runs the generic kernel (tests/test_gpu_gshells.py); l = 5 is refused
    g_shell = mi.Shells.from_list([((0.0, 0.0, 0.0), 4, [(1.0, 1.0)])])
    assert eng.eri_packed(g_shell).shape == (mi.Shells.from_list([((0.0, 0.0, 0.0), 4, [(1.0, 1.0)])]).npacked,)
    h_shell = mi.Shells.from_list([((0.0, 0.0, 0.0), 5, [(1.0, 1.0)])])
    with pytest.raises(engine.MolintsError) as e:
        eng.eri_packed(h_shell)
    assert e.value.status == -2
    # one f shell: (ff|ff) on one centre, against the oracle
    f_shell = mi.Shells.from_list([((0.1, -0.2, 0.3), 3, [(1.3, 1.0)])])
    from oracle import oracle as O
    with O.exact_boys():
        ref = O.eri_packed_hgp_ld(f_shell, nthreads=4)
    assert np.max(np.abs(eng.eri_packed(f_shell) - ref)) < TOL_FP64
    bad = mi.Shells.from_list([((0.0, 0.0, 0.0), 0, [(-1.0, 1.0)])])
    with pytest.raises(engine.MolintsError) as e:
        eng.eri_packed(bad)
    assert e.value.status == -1


def test_budget_refusal():
    from molints_b200 import engine
    e = engine.Engine(0, hbm_budget_bytes=1 << 20)
    try:
        with pytest.raises(engine.MolintsError) as err:
            e.eri_packed(mi.config1())
        assert err.value.status == -3
    finally:
        e.close()


# ------------------------------------------------------------------ f shells and Rys
def _f_molecule(seed, nheavy=2, nh=2):
    """A small molecule of the serving workload's shape: polarised heavy atoms that carry an
    f(K=1) shell, and hydrogens."""
    return mi.basis.synthetic_molecule(seed, nheavy, nh, mi.basis.POLARISED_C, mi.basis.POLARISED_H,
                                       0.1, 1e4, f"fmol{seed}", heavy_extra=[(3, 1)])


def _exact_ld(oracle, sh):
    """Near-exact reference: the HGP restatement in long double, exact Boys function, in the
    stable orientation (tighter shell first where the HRR would otherwise cancel)."""
    with oracle.exact_boys(), oracle.stable_orientation():
        return oracle.eri_packed_hgp_ld(sh, nthreads=0)


def _fp64_floor(oracle, sh, ld):
    """What plain FP64 arithmetic of the same algorithm reaches on this basis: twice the FP64
    restatement's own max error against the long-double value.  Random contractions of
    nearly equal exponents cancel (coefficients ~1e3 of alternating sign); no FP64
    evaluation gets much closer than the restatement, and one that sums the primitive
    quartets in another order (the device splits heavy quartets over lanes) lands at a
    different point of the same rounding spread, measured up to 1.1x the restatement's."""
    with oracle.exact_boys(), oracle.stable_orientation():
        return 2.0 * float(np.max(np.abs(oracle.eri_packed_hgp(sh, nthreads=0) - ld)))


@pytest.mark.parametrize("seed", [201, 202, 203])
def test_f_shells_random_bases(eng, oracle, seed):
    """Random l <= 3 bases (every class pair up to (ff|ff); the f classes run the Rys
    kernels): within 1e-12 Eh of the long-double HGP oracle, and of Huzinaga."""
    from molints_b200 import engine
    sh = _rand_basis(seed, 3, natom=2, kmax=2)
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    ld = _exact_ld(oracle, sh)
    assert np.max(np.abs(got - ld)) < TOL_FP64 + _fp64_floor(oracle, sh, ld)
    huz = oracle.eri_packed_huzinaga(sh, nthreads=0)
    assert np.max(np.abs(got - huz)) < TOL_FP64


def test_f_molecule_serving_shape(eng, oracle):
    """A molecule of the serving workload's recipe (l <= 3, exponents to 1e4, K up to 7)."""
    from molints_b200 import engine
    sh = _f_molecule(11)
    assert 3 in set(sh.L.tolist())
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    ld = _exact_ld(oracle, sh)
    assert np.max(np.abs(got - ld)) < TOL_FP64 + _fp64_floor(oracle, sh, ld)


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_rys_method_every_class(eng, oracle, cfg):
    """METHOD_RYS (all_twoe_ints_rys's algorithm) for every class pair of configs 1 and 2."""
    from molints_b200 import engine
    sh = getattr(mi, cfg)()
    got = eng.eri_packed(sh, method=engine.METHOD_RYS, boys=engine.BOYS_EXACT)
    ld = _exact_ld(oracle, sh)
    assert np.max(np.abs(got - ld)) < TOL_FP64 + _fp64_floor(oracle, sh, ld)


def test_class_method_table(eng):
    """AUTO follows the context's per-class table; HGP and Rys agree class by class."""
    from molints_b200 import engine
    sh = mi.config2()
    hgp = eng.eri_packed(sh, boys=engine.BOYS_EXACT, method=engine.METHOD_HGP)
    table = {(x, y): engine.METHOD_RYS for x in range(engine.NUM_PAIR_CLASSES) for y in range(x + 1)
             if (x + y) % 2 == 0}
    eng.set_class_methods(table)
    try:
        mix = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
        plan = eng.plan(sh, boys=engine.BOYS_EXACT)
        import torch
        out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
        plan.set_profiling(True)
        plan.execute(out.data_ptr())
        names = [n for n, _ in plan.launch_times()]
        plan.close()
    finally:
        eng.set_class_methods(None)
    assert any(n.startswith("rys_") for n in names) and any(n.startswith("eri_") for n in names)
    # None restores the shipped default: on a B200 the tuned table (Rys for (dd|dd))
    import torch
    if torch.cuda.get_device_name(0).startswith("NVIDIA B200"):
        assert eng.class_methods()[(6, 6)] & 3 == engine.METHOD_RYS
        fresh = engine.Engine(0)
        assert fresh.class_methods() == eng.class_methods()
        fresh.close()
    assert np.max(np.abs(mix - hgp)) < TOL_FP64
    with pytest.raises(engine.MolintsError):
        eng.set_class_methods({(0, 0): 7})


def test_schedule_knobs_keep_results(eng, oracle):
    """The work-queue schedule changes how quartets are grouped and split over lanes and how
    many gather blocks share an SM, not what is computed: extreme schedules give the default's
    integrals within the FP64 bar, on a d molecule (HGP lane splits) and an f molecule (Rys
    chunks), with direct stores and the two-phase gather, and every slot is written."""
    from molints_b200 import engine
    default = eng.schedule()
    assert set(default) == {"lane_cost", "hgp_widen", "rys_chunks", "rys_max_width", "gather_blocks"}
    mols = [mi.config2(), _f_molecule(21, nheavy=2, nh=1)]
    refs = [eng.eri_packed(sh, boys=engine.BOYS_EXACT) for sh in mols]
    try:
        for sched in ({"lane_cost": 20.0, "hgp_widen": 4, "rys_chunks": 1, "rys_max_width": 16, "gather_blocks": 1},
                      {"lane_cost": 1e6, "hgp_widen": 1, "rys_chunks": 1 << 30, "rys_max_width": 1,
                       "gather_blocks": 16}):
            eng.set_schedule(sched)
            assert eng.schedule() == {k: (float(v) if k == "lane_cost" else v) for k, v in sched.items()}
            for sh, ref in zip(mols, refs):
                for out in (engine.OUTPUT_DIRECT, engine.OUTPUT_TWO_PHASE):
                    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT, output=out)
                    assert not np.isnan(got).any()
                    assert np.max(np.abs(got - ref)) < TOL_FP64
        with pytest.raises(engine.MolintsError):
            eng.set_schedule({"hgp_widen": 0})
        with pytest.raises(engine.MolintsError):
            eng.set_schedule({"lane_cost": -1.0})
        with pytest.raises(engine.MolintsError):
            eng.set_schedule({"gather_blocks": 17})
    finally:
        eng.set_schedule(None)
    assert eng.schedule() == default
    fresh = engine.Engine(0)
    assert fresh.schedule() == default
    fresh.close()


def test_f_shell_schwarz_bounds(eng, oracle):
    """Contracted Schwarz bounds of pairs with f shells (the Rys bound kernels)."""
    import torch
    sh = _f_molecule(13, nheavy=1, nh=1)
    plan = eng.plan(sh)
    out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
    plan.execute(out.data_ptr())
    q = plan.schwarz()
    ints = out.cpu().numpy()
    plan.close()
    off = sh.fn_offsets()
    n = sh.nbf
    npair = n * (n + 1) // 2
    diag = ints[np.arange(npair) * (np.arange(npair) + 1) // 2 + np.arange(npair)]
    for i in range(sh.nshell):
        for j in range(i + 1):
            m = 0.0
            for a in range(off[i], off[i + 1]):
                for b in range(off[j], off[j + 1]):
                    ab = a * (a + 1) // 2 + b if a >= b else b * (b + 1) // 2 + a
                    m = max(m, abs(diag[ab]))
            assert q[i * (i + 1) // 2 + j] == pytest.approx(np.sqrt(m), rel=1e-12)


def test_rys_mixed_error_bound(eng):
    """MIXED with the Rys kernels (FP32 2-D tables and batch sums, FP64 accumulation): the
    tuned cutoff keeps max |MIXED - FP64| below 1e-9 Eh on config 2 and an f molecule."""
    from molints_b200 import autotune, engine
    for sh in (mi.config2(), _f_molecule(12)):
        cut, table = autotune.tune_fp32_cutoff(eng, sh, method=engine.METHOD_RYS)
        assert cut > 0, table
        ref = eng.eri_packed(sh, method=engine.METHOD_RYS)
        eng.set_class_methods({})  # every FP32 variant enabled
        try:
            got, st = eng.eri_packed(sh, precision=engine.MIXED, fp32_cutoff=cut,
                                     method=engine.METHOD_RYS, with_stats=True)
        finally:
            eng.set_class_methods(None)
        assert st["n_fp32_quartets"] > 0 and st["n_fp32_launches"] > 0, st
        assert np.max(np.abs(got - ref)) < TOL_MIXED


def test_class_method_tuner(eng, oracle):
    """tune_class_methods times both kernels of every HGP-capable class pair present and
    returns a valid table; plans under it and HGP plans both stay within 1e-12 Eh (plus the
    basis's FP64 floor) of the long-double oracle."""
    from molints_b200 import autotune, engine
    mols = [mi.config2(), _f_molecule(14)]
    table, timings = autotune.tune_class_methods(eng, mols, repeats=2, fp32_cutoff=1e-3)
    assert timings and {v & 3 for v in table.values()} <= {engine.METHOD_HGP, engine.METHOD_RYS}
    assert all(t is None or t > 0 for ts in timings.values() for t in ts)
    eng.set_class_methods(table)
    try:
        for sh in mols:
            got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
            ref = eng.eri_packed(sh, boys=engine.BOYS_EXACT, method=engine.METHOD_HGP)
            ld = _exact_ld(oracle, sh)
            bar = TOL_FP64 + _fp64_floor(oracle, sh, ld)
            assert np.max(np.abs(got - ld)) < bar and np.max(np.abs(ref - ld)) < bar
    finally:
        eng.set_class_methods(None)


def test_plan_cuda_graph(eng):
    """An execute captured as a CUDA graph (side streams included) gives the eager result
    bit for bit, on repeat launches and after a recapture for a new output vector."""
    import torch
    from molints_b200 import engine
    sh = _f_molecule(15)
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        plan = eng.plan(sh, precision=engine.MIXED, fp32_cutoff=1e-4)
        ref = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
        plan.execute(ref.data_ptr())
        plan.set_graph(True)
        outs = [torch.full_like(ref, float("nan")) for _ in range(2)]
        for out in (outs[0], outs[0], outs[1]):
            out.fill_(float("nan"))
            plan.execute(out.data_ptr())
            torch.cuda.synchronize()
            assert torch.equal(out, ref)
        assert plan.stats()["device_ms"] > 0
        plan.close()
    finally:
        eng.set_stream(None)


@pytest.mark.parametrize("which", ["config2", "fmol"])
def test_jk_digestion_matches_make2JmK(eng, oracle, which):
    """J and K digested on the device (no packed vector) equal make2JmK's contraction of the
    packed vector (src/ERI.jl:114-128, restated in the oracle) for a random symmetric density."""
    import torch
    from molints_b200 import engine
    sh = mi.config2() if which == "config2" else _f_molecule(16)
    n = sh.nbf
    rng = np.random.default_rng(5)
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    J, K = eng.jk(sh, D)
    ints = eng.eri_packed(sh)
    G, Jr, Kr = oracle.make2JmK(D, ints)
    scale = max(1.0, np.max(np.abs(Jr)), np.max(np.abs(Kr)))
    assert np.max(np.abs(J - Jr)) < 1e-11 * scale
    assert np.max(np.abs(K - Kr)) < 1e-11 * scale
    assert np.allclose(J, J.T, atol=1e-12 * scale) and np.allclose(K, K.T, atol=1e-12 * scale)
    assert np.max(np.abs(engine.make2JmK(D, sh) - G)) < 3e-11 * scale
    # device form on a plan, and the shards' shares summing to the whole
    from molints_b200 import shard
    Dd = torch.from_numpy(D).cuda()
    Jd = torch.empty_like(Dd)
    Kd = torch.empty_like(Dd)
    Js, Ks = np.zeros((n, n)), np.zeros((n, n))
    for r in range(3):
        plan = eng.plan_shard(sh, r, 3)
        plan.jk(Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr())
        torch.cuda.synchronize()
        Js += Jd.cpu().numpy()
        Ks += Kd.cpu().numpy()
        plan.close()
    assert np.max(np.abs(Js - Jr)) < 1e-11 * scale and np.max(np.abs(Ks - Kr)) < 1e-11 * scale


def test_plan_outliving_its_engine():
    """A plan whose engine was closed first fails cleanly (invalid argument) and can still be
    destroyed: the context's destruction released the plan's device state."""
    import torch
    from molints_b200 import engine
    e = engine.Engine(0)
    sh = mi.config0()
    plan = e.plan(sh)
    out = torch.empty(sh.npacked, dtype=torch.float64, device="cuda")
    plan.execute(out.data_ptr())
    torch.cuda.synchronize()
    e.close()
    with pytest.raises(engine.MolintsError) as err:
        plan.execute(out.data_ptr())
    assert err.value.status == -1
    plan.close()


@pytest.mark.parametrize("method", ["hgp", "rys"])
def test_reference_coulomb_pins_on_device(eng, golden, oracle, method):
    """The known answers of test/runtests.jl (coulomb and coulomb_rys cases: (ss|ss), (ss|pxpx)
    and the s-s distance sweep on unit-exponent primitives) computed by the device path with
    either method, at the reference's own tolerance (rtol 1.5e-8)."""
    from molints_b200 import engine
    m = engine.METHOD_HGP if method == "hgp" else engine.METHOD_RYS
    o = (0.0, 0.0, 0.0)
    g = golden["coulomb"]
    one_s = mi.Shells.from_list([(o, 0, [(1.0, 1.0)])])
    assert eng.eri_packed(one_s, method=m, boys=engine.BOYS_EXACT)[0] == pytest.approx(
        g["c,c,c,c"]["value"], rel=1.5e-8)
    sp = mi.Shells.from_list([(o, 0, [(1.0, 1.0)]), (o, 1, [(1.0, 1.0)])])
    v = eng.eri_packed(sp, method=m, boys=engine.BOYS_EXACT)
    assert v[oracle.iindex(0, 0, 1, 1)] == pytest.approx(g["s,s,px,px"]["value"], rel=1.5e-8)
    assert abs(v[oracle.iindex(0, 0, 0, 1)]) < 1e-17
    for case in golden["ss_distance_sweep"]:
        two = mi.Shells.from_list([(o, 0, [(1.0, 1.0)]), ((0.0, 0.0, case["r"]), 0, [(1.0, 1.0)])])
        w = eng.eri_packed(two, method=m, boys=engine.BOYS_EXACT)
        assert w[oracle.iindex(0, 0, 1, 1)] == pytest.approx(case["value"], rel=1.5e-8)


def test_one_electron_matrices(eng, oracle):
    """S, T and V on the device (molints_one_e, the drop-in for all_1e_ints) against the
    oracle's restatement of src/OneInts.jl: H2/STO-3G pins of test/runtests.jl:42-47, staggered
    ethane in STO-3G, and a random basis with shells up to f around four point charges."""
    from molints_b200 import engine
    h2 = mi.h2()
    S, T, V = engine.all_1e_ints(mi.build_basis(h2), h2)
    assert S[0, 1] == pytest.approx(0.6647387449282997, rel=1.5e-8)
    assert T[0, 0] == pytest.approx(0.76003188, rel=1.5e-8)
    assert T[0, 1] == pytest.approx(0.24141861181119084, rel=1.5e-8)
    eth = mi.ethane_staggered()
    cases = [(mi.config0(), [a.xyz for a in eth], [a.atno for a in eth])]
    rng = np.random.default_rng(9)
    cases.append((_rand_basis(301, 3, natom=2, kmax=2), rng.uniform(-2, 2, (4, 3)), [1.0, 6.0, 8.0, 1.0]))
    for sh, xyz, z in cases:
        S, T, V = eng.one_e(sh, xyz, z)
        Sr, Tr, Vr = oracle.all_1e_ints(sh, xyz, z)
        for got, ref in ((S, Sr), (T, Tr), (V, Vr)):
            assert np.max(np.abs(got - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))
        assert np.allclose(np.diag(S), 1.0, atol=1e-13)
