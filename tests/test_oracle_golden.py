"""Pin the CPU oracle to the reference's own known-answer values (test/runtests.jl).

The reference compares with Julia's default isapprox (rtol = sqrt(eps) ~ 1.5e-8); these
tests use that tolerance for values the reference prints to ~10 digits and a tight one
where the reference value is exact to double precision."""
import math

import numpy as np
import pytest

import molints_b200 as mi

RTOL_REF = 1.5e-8  # Julia's default isapprox, as test/runtests.jl uses


def test_iindex_pins(golden, oracle):
    for case in golden["iindex"]:
        i, j, k, l = (x - 1 for x in case["ijkl_1based"])
        assert oracle.iindex(i, j, k, l) + 1 == case["value_1based"], case


def test_fgamma_pins(golden, oracle):
    for case in golden["fgamma"]:
        assert oracle.boys(case["m"], case["T"]) == pytest.approx(case["value"], rel=RTOL_REF)
    # F0(1) = sqrt(pi)/2 erf(1) is known to full precision
    assert oracle.boys(0, 1.0) == pytest.approx(math.sqrt(math.pi) / 2 * math.erf(1.0), rel=1e-15)


@pytest.mark.parametrize("m", [0, 1, 2, 4, 8, 12, 16, 20])
def test_boys_series_against_mpmath(oracle, m):
    for T in [0.0, 1e-12, 1e-6, 0.01, 0.3, 1.0, 2.5, 7.0, 15.0, 29.9, 35.0, 45.0, 80.0]:
        exact = oracle.boys_mpmath(m, T)
        assert abs(oracle.boys(m, T) - exact) <= 2e-15 * exact, (m, T)


def test_farray_follows_reference_branches(oracle):
    # T < 30: top order exact, downward recursion; T >= 30: asymptotic (src/Boys.jl:19-27)
    f = oracle.farray(9, 12.0)
    for m in range(9):
        assert f[m] == pytest.approx(oracle.boys_mpmath(m, 12.0), rel=1e-14)
    f = oracle.farray(5, 31.0)
    for m in range(5):
        asym = math.sqrt(math.pi / 2) * math.prod(range(2 * m - 1, 0, -2)) / (62.0 ** (m + 0.5))
        assert f[m] == pytest.approx(asym, rel=1e-14)


def test_vrr_pins(golden, oracle):
    for case in golden["vrr"]:
        a, c = case["a_ijk"], case["c_ijk"]
        v = oracle.vrr(sum(a), sum(c), 1.0, 1.0, 1.0, 1.0, case["A"], [0, 0, 0], [0, 0, 0],
                       [0, 0, 0])
        got = v[0, oracle.ao_index(*a), oracle.ao_index(*c)]
        assert got == pytest.approx(case["value"], rel=RTOL_REF), case


def test_hrr_pins(golden, oracle):
    for case in golden["hrr"]:
        a, b, c, d = case["a_ijk"], case["b_ijk"], case["c_ijk"], case["d_ijk"]
        h = oracle.hrr(sum(a), sum(b), sum(c), sum(d), 1.0, 1.0, 1.0, 1.0, case["A"],
                       [0, 0, 0], [0, 0, 0], [0, 0, 0])
        got = h[oracle.ao_index(*a), oracle.ao_index(*b), oracle.ao_index(*c), oracle.ao_index(*d)]
        assert got == pytest.approx(case["value"], rel=RTOL_REF), case


def _norm_prim(oracle, expn, ijk):
    return oracle.pgbf_norm(expn, *ijk)


def test_coulomb_pins(golden, oracle):
    o = (0.0, 0.0, 0.0)
    s = (1.0, o, (0, 0, 0))
    px = (1.0, o, (1, 0, 0))
    ns, npx = _norm_prim(oracle, 1.0, (0, 0, 0)), _norm_prim(oracle, 1.0, (1, 0, 0))
    g = golden["coulomb"]
    raw = oracle.coulomb_prim(s, s, s, s)
    assert raw == pytest.approx(g["1,0,0,0,0,0,0,1,0,0,0,0,0,0,1,0,0,0,0,0,0,1,0,0,0,0,0,0"]["value"],
                                rel=RTOL_REF)
    assert ns ** 4 * raw == pytest.approx(g["c,c,c,c"]["value"], rel=RTOL_REF)
    assert ns ** 2 * npx ** 2 * oracle.coulomb_prim(s, s, px, px) == pytest.approx(
        g["s,s,px,px"]["value"], rel=RTOL_REF)
    assert oracle.coulomb_prim(s, s, s, px) == g["s,s,s,px"]["value"]
    for case in golden["ss_distance_sweep"]:
        s3 = (1.0, (0.0, 0.0, case["r"]), (0, 0, 0))
        got = ns ** 4 * oracle.coulomb_prim(s, s, s3, s3)
        assert got == pytest.approx(case["value"], rel=RTOL_REF), case


@pytest.mark.parametrize("driver", ["hgp", "huzinaga"])
def test_h2_sto3g_pins(golden, oracle, driver):
    sh = mi.build_basis(mi.h2())
    assert sh.nbf == 2
    ints = oracle.eri_packed_hgp(sh) if driver == "hgp" else oracle.eri_packed_huzinaga(sh)
    idx = {"llll": (0, 0, 0, 0), "rrrr": (1, 1, 1, 1), "llrr": (0, 0, 1, 1),
           "lllr": (0, 0, 0, 1), "lrlr": (0, 1, 0, 1)}
    for key, case in golden["h2_sto3g_coulomb"].items():
        assert ints[oracle.iindex(*idx[key])] == pytest.approx(case["value"], rel=RTOL_REF), key


def test_prefactor_defect_d5(oracle):
    """vrr! (src/HGP.jl:150) matches the HGP prefactor only when zeta*eta == zeta+eta."""
    A, B, C, D = [0.1, 0.2, 0.3], [0.0, -0.4, 0.2], [0.5, 0.1, -0.3], [-0.2, 0.3, 0.0]
    v0 = oracle.vrr(0, 0, 1.0, 1.0, 1.0, 1.0, A, B, C, D, 0)
    v1 = oracle.vrr(0, 0, 1.0, 1.0, 1.0, 1.0, A, B, C, D, 1)
    assert v0[0, 0, 0] == pytest.approx(v1[0, 0, 0], rel=1e-15)
    exps = (0.7, 1.9, 0.35, 2.6)
    v0 = oracle.vrr(0, 0, *exps, A, B, C, D, 0)[0, 0, 0]
    v1 = oracle.vrr(0, 0, *exps, A, B, C, D, 1)[0, 0, 0]
    huz = oracle.coulomb_prim(*[(e, x, (0, 0, 0)) for e, x in zip(exps, (A, B, C, D))])
    assert v0 == pytest.approx(huz, rel=1e-13)
    assert abs(v1 - huz) > 1e-3 * abs(huz)


def test_hgp_equals_huzinaga_ethane_sto3g(oracle):
    sh = mi.config0()
    a = oracle.eri_packed_hgp(sh, nthreads=4)
    b = oracle.eri_packed_huzinaga(sh, nthreads=4)
    assert a.shape == (9316,)
    assert np.max(np.abs(a - b)) < 1e-12


def _small_random_basis(seed, lmax, natom=2):
    rng = np.random.default_rng(seed)
    lst = []
    for a in range(natom):
        xyz = rng.uniform(-1.5, 1.5, size=3)
        for l in range(lmax + 1):
            k = int(rng.integers(1, 3))
            lst.append((xyz, l, mi.basis._random_shell(rng, l, k, 0.2, 8.0)))
    return mi.Shells.from_list(lst, f"rand{seed}")


@pytest.mark.parametrize("lmax,seed", [(1, 11), (2, 12), (3, 13)])
def test_hgp_equals_huzinaga_random_classes(oracle, lmax, seed):
    """With the exact Boys function the restated HGP recurrences agree with Huzinaga."""
    sh = _small_random_basis(seed, lmax)
    with oracle.exact_boys():
        a = oracle.eri_packed_hgp(sh, nthreads=8)
    b = oracle.eri_packed_huzinaga(sh, nthreads=8)
    scale = max(1.0, np.max(np.abs(b)))
    assert np.max(np.abs(a - b)) < 1e-13 * scale


def test_reference_boys_branch_error_is_bounded(oracle):
    """farray's asymptotic branch at T >= 30 (src/Boys.jl:20-26) drops the e^-T terms; on a
    d-shell basis with T ~ 30 quartets the reference HGP is a few 1e-12 from the exact value,
    which is why the engine offers the reference branch (default) and an exact mode."""
    sh = _small_random_basis(12, 2)
    ref = oracle.eri_packed_hgp(sh, nthreads=8)
    with oracle.exact_boys():
        exact = oracle.eri_packed_hgp(sh, nthreads=8)
    d = np.max(np.abs(ref - exact))
    assert 1e-13 < d < 1e-10



def test_hrr_orientation_conditioning(oracle):
    """Config 2's p shell on an H (exponent 0.209) and d shell on a C (exponent 2044): with the
    diffuse p first -- the reference's index order for this pair -- chrr loses ~1e-11 to HRR
    cancellation; with the d first -- the engine's order, larger L first -- it is within
    1e-15 of the 40-digit Huzinaga value."""
    sh = mi.config2()
    p, d = 20, 5
    assert (int(sh.L[p]), int(sh.L[d])) == (1, 2)
    two = mi.Shells.from_list([(sh.xyz[p], 1, [(sh.expn[sh.prim_off[p]], 1.0)]),
                               (sh.xyz[d], 2, [(sh.expn[sh.prim_off[d]], 1.0)])])
    py, dyy = (0, 1, 0), (0, 2, 0)
    exact = oracle.contracted_mpmath(two, [(0, py), (1, dyy), (0, py), (1, dyy)])
    ref_order = oracle.shell_quartet(two, 0, 1, 0, 1)[1, 3, 1, 3]
    eng_order = oracle.shell_quartet(two, 1, 0, 1, 0)[3, 1, 3, 1]
    assert abs(eng_order - exact) < 1e-15
    assert abs(ref_order - exact) > 1e-12


# ------------------------------------------------------------------ Rys (src/Rys.jl)
def test_rys_golden_pins(golden, oracle):
    """The coulomb_rys known answers of test/runtests.jl:130-149 (same values as coulomb)."""
    o = (0.0, 0.0, 0.0)
    s = (1.0, o, (0, 0, 0))
    px = (1.0, o, (1, 0, 0))
    ns, npx = oracle.pgbf_norm(1.0, 0, 0, 0), oracle.pgbf_norm(1.0, 1, 0, 0)
    g = golden["coulomb"]
    assert ns ** 4 * oracle.coulomb_rys_prim(s, s, s, s) == pytest.approx(g["c,c,c,c"]["value"], rel=RTOL_REF)
    assert ns ** 2 * npx ** 2 * oracle.coulomb_rys_prim(s, s, px, px) == pytest.approx(
        g["s,s,px,px"]["value"], rel=RTOL_REF)
    assert abs(oracle.coulomb_rys_prim(s, s, s, px)) < 1e-17
    for case in golden["ss_distance_sweep"]:
        s3 = (1.0, (0.0, 0.0, case["r"]), (0, 0, 0))
        assert ns ** 4 * oracle.coulomb_rys_prim(s, s, s3, s3) == pytest.approx(case["value"], rel=RTOL_REF)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7])
def test_rys_roots_against_mpmath(oracle, n):
    for X in [0.0, 1e-9, 0.4, 3.3, 17.0, 49.5, 99.9, 100.0, 640.0, 1e5]:
        r, w = oracle.rys_roots(n, X)
        R, W = oracle.rys_roots_mpmath(n, X)
        assert np.max(np.abs(r - R) / R) < 4e-15, (n, X)
        assert np.max(np.abs(w - W) / W) < 4e-15, (n, X)
        # sum W_i x_i^k = F_k(X)
        for k in range(2 * n):
            assert np.sum(w * r ** k) == pytest.approx(oracle.boys_mpmath(k, X), rel=1e-13)


def test_rys_h2_whole_basis(oracle):
    """test/runtests.jl:60 compares all_twoe_ints_rys with all_twoe_ints at rtol 1e-7."""
    sh = mi.build_basis(mi.h2())
    assert np.max(np.abs(oracle.eri_packed_rys(sh) - oracle.eri_packed_huzinaga(sh))) < 1e-15


@pytest.mark.parametrize("lmax,seed", [(1, 11), (2, 12), (3, 13)])
def test_rys_equals_hgp_random_classes(oracle, lmax, seed):
    """Rys with the CGBF norms applied (D4 fixed) equals the long-double HGP up to f shells."""
    sh = _small_random_basis(seed, lmax)
    r = oracle.eri_packed_rys(sh, nthreads=8)
    with oracle.exact_boys():
        h = oracle.eri_packed_hgp_ld(sh, nthreads=8)
    assert np.max(np.abs(r - h)) < 1e-13 * max(1.0, np.max(np.abs(h)))


def test_make2JmK_restatement_matches_loops(oracle):
    """The oracle's make2JmK (src/ERI.jl:114-128) against explicit loops on ethane/STO-3G."""
    sh = mi.config0()
    ints = oracle.eri_packed_hgp(sh, nthreads=4)
    n = sh.nbf
    rng = np.random.default_rng(1)
    A = rng.normal(size=(n, n))
    D = A + A.T
    G, J, K = oracle.make2JmK(D, ints)
    for i in (0, 3, 9, 15):
        for j in (0, 7, 15):
            g = sum(D[k, l] * (2 * ints[oracle.iindex(i, j, k, l)] - ints[oracle.iindex(i, k, j, l)])
                    for k in range(n) for l in range(n))
            assert G[i, j] == pytest.approx(g, rel=1e-12, abs=1e-12)


def test_hrr_orientation_tight_first(oracle):
    """D6: a diffuse s shell (0.108) before a tight f (1009), 6.8 bohr apart.  The reference
    orientation chrr(I,J,...) with I >= J by shell index transfers angular momentum onto the
    tight f and cancels: its FP64 value is off by ~4e-9 Eh, and even long double by ~5e-12.
    With the tight shell first (the engine's orientation) FP64 agrees with Huzinaga."""
    A = np.array([1.3, -2.0, 0.4])
    B = A + np.array([4.1, 3.9, -3.6])
    sub = mi.Shells.from_list([(A, 3, [(1008.9973033479797, 1.0)]), (B, 0, [(0.10849250091461012, 1.0)])])
    huz = oracle.eri_packed_huzinaga(sub, nthreads=2)
    with oracle.exact_boys():
        ref_f64 = oracle.eri_packed_hgp(sub, nthreads=2)
        ref_ld = oracle.eri_packed_hgp_ld(sub, nthreads=2)
        with oracle.stable_orientation():
            st_f64 = oracle.eri_packed_hgp(sub, nthreads=2)
            st_ld = oracle.eri_packed_hgp_ld(sub, nthreads=2)
    assert np.max(np.abs(ref_f64 - huz)) > 1e-10
    assert np.max(np.abs(st_f64 - huz)) < 1e-13 * max(1.0, np.max(np.abs(huz)))
    assert np.max(np.abs(st_ld - huz)) < np.max(np.abs(ref_ld - huz))


def test_one_electron_restatement_pins(oracle):
    """The one-electron known answers of test/runtests.jl:42-88 on the oracle's restatement of
    src/OneInts.jl (unit-exponent primitives at the origin, and H2/STO-3G)."""
    o = (0.0, 0.0, 0.0)
    ns = oracle.pgbf_norm(1.0, 0, 0, 0)
    npx = oracle.pgbf_norm(1.0, 1, 0, 0)
    assert ns ** 2 * oracle.kinetic_prim(1.0, o, (0, 0, 0), 1.0, o, (0, 0, 0)) == pytest.approx(1.5, rel=1e-12)
    assert oracle.kinetic_prim(1.0, o, (0, 0, 0), 1.0, o, (0, 0, 0)) == pytest.approx(2.9530518648229536, rel=1e-12)
    assert ns ** 2 * oracle.nuclear_prim(1.0, o, (0, 0, 0), 1.0, o, (0, 0, 0), o) == pytest.approx(-1.59576912, rel=1.5e-8)
    assert npx ** 2 * oracle.nuclear_prim(1.0, o, (1, 0, 0), 1.0, o, (1, 0, 0), o) == pytest.approx(-1.06384608, rel=1.5e-8)
    assert oracle.nuclear_prim(1.0, o, (0, 0, 0), 1.0, o, (0, 0, 0), o) == pytest.approx(-np.pi, rel=1e-12)
    assert oracle.overlap_prim(1.0, o, (0, 0, 0), 1.0, o, (0, 0, 0)) == pytest.approx(1.9687012432, rel=1.5e-8)
    h2 = mi.h2()
    S, T, V = oracle.all_1e_ints(mi.build_basis(h2), [a.xyz for a in h2], [a.atno for a in h2])
    assert S[0, 0] == pytest.approx(1.0, rel=1e-12) and S[1, 1] == pytest.approx(1.0, rel=1e-12)
    assert S[0, 1] == pytest.approx(0.6647387449282997, rel=1.5e-8)
    assert T[0, 0] == pytest.approx(0.76003188, rel=1.5e-8)
    assert T[0, 1] == pytest.approx(0.24141861181119084, rel=1.5e-8)
