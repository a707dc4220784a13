"""g shells (l = 4): the reference's tables go to l = 4 (shell_indices, src/Basis.jl:269-279)
and its Huzinaga driver all_twoe_ints (src/ERI.jl:15-112) accepts them; here every shell quartet
with a g shell runs the generic Rys kernel (up to nine roots).  Checked against the oracle's
Huzinaga restatement and its long-double HGP restatement (both general in l), with the exact
Boys function; FP64 bar 1e-12 plus the basis's FP64 floor."""
import numpy as np
import pytest

import molints_b200 as mi

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


@pytest.fixture(scope="module")
def eng():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine
    e = engine.Engine(0)
    yield e
    e.close()


def _g_basis(seed, natom=2, kmax=2):
    rng = np.random.default_rng(seed)
    lst = []
    for _ in range(natom):
        xyz = rng.uniform(-1.5, 1.5, 3)
        for l in (0, 1, 2, 3, 4):
            lst.append((xyz, l, mi.basis._random_shell(rng, l, int(rng.integers(1, kmax + 1)), 0.3, 8.0)))
    return mi.Shells.from_list(lst, f"g{seed}")


def _ld(oracle, sh):
    with oracle.exact_boys(), oracle.stable_orientation():
        ld = oracle.eri_packed_hgp_ld(sh, nthreads=0)
        f64 = oracle.eri_packed_hgp(sh, nthreads=0)
    return ld, 2.0 * float(np.max(np.abs(f64 - ld)))


def test_single_g_shell(eng, oracle):
    from molints_b200 import engine
    sh = mi.Shells.from_list([((0.1, -0.2, 0.3), 4, [(1.3, 1.0)])])
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    ld, floor = _ld(oracle, sh)
    err = float(np.max(np.abs(got - ld)))
    print(f"(gg|gg) one centre: {got.size} integrals, |GPU - oracle| {err:.2e}")
    assert err < TOL_FP64 + floor


@pytest.mark.parametrize("seed", [401, 402])
def test_g_basis_against_oracle(eng, oracle, seed):
    """Two centres with s, p, d, f and g shells: every class pair up to (gg|gg), the g ones on
    the generic kernel and the rest on the class kernels, in one packed vector."""
    from molints_b200 import engine
    sh = _g_basis(seed)
    got = eng.eri_packed(sh, boys=engine.BOYS_EXACT)
    ld, floor = _ld(oracle, sh)
    err = float(np.max(np.abs(got - ld)))
    print(f"g basis {seed}: nbf {sh.nbf}, floor {floor:.2e}, |GPU - ld| {err:.2e}")
    assert err < TOL_FP64 + floor
    # every method and both precisions write the same g entries (FP64 kernel for g quartets)
    for kw in ({"method": engine.METHOD_RYS}, {"method": engine.METHOD_HGP},
               {"precision": engine.MIXED, "fp32_cutoff": 1e-6}):
        other = eng.eri_packed(sh, boys=engine.BOYS_EXACT, **kw)
        assert np.max(np.abs(other - ld)) < 1e-9, kw


def test_g_batch_plan_and_limits(eng):
    """A batch plan over a g basis and two others equals the single plans; sharding, J/K
    digestion and Schwarz bounds refuse g shells (MOLINTS_ERR_UNSUPPORTED); l = 5 is refused."""
    import torch
    from molints_b200 import engine
    mols = [_g_basis(403, natom=1), mi.config0(), _g_basis(404, natom=1, kmax=1)]
    single = [eng.eri_packed(sh, boys=engine.BOYS_EXACT) for sh in mols]
    plan = eng.plan_batch(mols, boys=engine.BOYS_EXACT)
    out = torch.full((plan.npacked,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        plan.execute(out.data_ptr())
        torch.cuda.synchronize()
    finally:
        eng.set_stream(None)
    got = out.cpu().numpy()
    for m, ref in enumerate(single):
        seg = got[plan.offsets[m]:plan.offsets[m + 1]]
        assert not np.isnan(seg).any()
        assert np.array_equal(seg, ref), m
    plan.close()
    sh = mols[0]
    with pytest.raises(engine.MolintsError) as e:
        eng.plan_shard(sh, 0, 2)
    assert e.value.status == -2
    with pytest.raises(engine.MolintsError) as e:
        eng.jk(sh, np.eye(sh.nbf))
    assert e.value.status == -2
    h = mi.Shells.from_list([((0.0, 0.0, 0.0), 5, [(1.0, 1.0)])])
    with pytest.raises(engine.MolintsError) as e:
        eng.eri_packed(h)
    assert e.value.status == -2


def test_g_adapter(oracle):
    """The reference wrapper's all_twoe_ints on a one-centre s-g basis, against the oracle's
    Huzinaga restatement (the reference's own all_twoe_ints algorithm)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import molecular_integrals as M
    sh = _g_basis(405, natom=1, kmax=2)
    with oracle.exact_boys():
        huz = oracle.eri_packed_huzinaga(sh, nthreads=0)
    got = M.MolecularIntegrals().all_twoe_ints(M.Basis.from_shells(sh))
    err = float(np.max(np.abs(got - huz)))
    print(f"adapter, one-centre s-g basis: |GPU - Huzinaga| {err:.2e}")
    assert err < 1e-11
