"""The Python surface of the reference wrapper (python/molecular_integrals.py), backed by the
C ABI: known answers of test/runtests.jl (values from the committed golden fixture) and the
CPU oracle.  The GPU tests call the library; the others check the host-side logic only."""
import itertools

import numpy as np
import pytest

import molints_b200 as mi
from molints_b200 import molecular_integrals as M

gpu = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_packed_to_4d_matches_iindex():
    n = 5
    v = np.arange(n * (n + 1) * (n * n + n + 2) // 8, dtype=np.float64)
    A = M.packed_to_4d(v, n)
    for i, j, k, l in itertools.product(range(n), repeat=4):
        assert A[i, j, k, l] == M.packed_index(i, j, k, l)
    # the 8-fold symmetry of the expansion
    assert np.array_equal(A, A.transpose(1, 0, 2, 3))
    assert np.array_equal(A, A.transpose(2, 3, 0, 1))


def test_iindex_golden(golden):
    for g in golden["iindex"]:
        i, j, k, l = (x - 1 for x in g["ijkl_1based"])
        assert M.packed_index(i, j, k, l) == g["value_1based"] - 1


def test_primitive_norm_matches_reference_pgbf():
    # s(0,0,0) = 0.71270547 for pgbf(1.0) (test/runtests.jl:28)
    assert abs(M.primitive_norm(1.0, (0, 0, 0)) - 0.71270547) < 1e-8
    c = M.CGBF((0, 0, 0), (0, 0, 0), [1.0], [1.0])
    assert abs(c.norm - 1.0) < 1e-15  # one normalised primitive is already normalised


def test_unknown_method_raises():
    with pytest.raises(ValueError):
        M.MolecularIntegrals().all_twoe_ints(mi.config0(), method="huzinaga")


@gpu
def test_coulomb_repulsion_known_answers(golden, oracle):
    _cuda()
    o = (0.0, 0.0, 0.0)
    # coulomb(1, 0,0,0, 0,0,0, ...) = 4.37335458: raw primitive integral (test/runtests.jl:110)
    v = M.coulomb_repulsion(o, 1.0, (0, 0, 0), 1.0, o, 1.0, (0, 0, 0), 1.0,
                            o, 1.0, (0, 0, 0), 1.0, o, 1.0, (0, 0, 0), 1.0)
    assert abs(v - golden["coulomb"]["1,0,0,0,0,0,0,1,0,0,0,0,0,0,1,0,0,0,0,0,0,1,0,0,0,0,0,0"]["value"]) < 1e-8
    # against the oracle's Huzinaga primitive at FP64 accuracy, p and d powers included
    rng = np.random.default_rng(3)
    for _ in range(6):
        prims = [(tuple(rng.uniform(-1, 1, 3)), tuple(int(x) for x in rng.integers(0, 2, 3)),
                  float(rng.uniform(0.3, 3.0))) for _ in range(4)]
        args = []
        for org, pw, al in prims:
            args += [org, 1.0, pw, al]
        got = M.coulomb_repulsion(*args)
        ref = oracle.coulomb_prim(*[(al, org, pw) for org, pw, al in prims])
        assert abs(got - ref) < 1e-12 * max(1.0, abs(ref)), (prims, got, ref)


@gpu
def test_coulomb_pgbf_and_distance_sweep(golden, oracle):
    """The reference's pyquante2 values hold to its own rtol (about 1.5e-8: pyquante2's Boys
    approximation), and the oracle's Huzinaga values to 1e-12."""
    _cuda()
    m = M.MolecularIntegrals()
    s = M.PGBF(1.0)
    px = M.PGBF(1.0, (0, 0, 0), (1, 0, 0))
    assert abs(m.coulomb_pgbf(s, s, px, px) - golden["coulomb"]["s,s,px,px"]["value"]) < 1e-12
    assert abs(m.coulomb_pgbf(s, s, s, px)) < 1e-15
    c = M.CGBF((0, 0, 0), (0, 0, 0), [1.0], [1.0])
    assert abs(m.coulomb(c, c, c, c) - golden["coulomb"]["c,c,c,c"]["value"]) < 1e-8
    for g in golden["ss_distance_sweep"]:
        s3 = M.PGBF(1.0, (0.0, 0.0, g["r"]))
        v = m.coulomb_pgbf(s, s, s3, s3)
        assert abs(v - g["value"]) <= 1.5e-8 * abs(g["value"]), g
        o = (0.0, 0.0, 0.0)
        with oracle.exact_boys():
            ref = oracle.coulomb_prim((1.0, o, o), (1.0, o, o), (1.0, (0, 0, g["r"]), o),
                                      (1.0, (0, 0, g["r"]), o)) * s.norm ** 4
        assert abs(v - ref) < 1e-12, (g, v, ref)


@gpu
def test_h2_basis_known_answers(golden, oracle):
    """H2/STO-3G: the reference's values (test/runtests.jl:41-52) to its rtol (about 1.5e-8:
    they come from pyquante2), and the oracle's Huzinaga all_twoe_ints to 1e-12."""
    _cuda()
    m = M.MolecularIntegrals()
    b = M.Basis([M.Atom(a.atno, tuple(a.xyz)) for a in mi.h2()], "sto3g")
    assert len(b) == 2
    l, r = b
    h = golden["h2_sto3g_coulomb"]
    with oracle.exact_boys():
        huz = oracle.eri_packed_huzinaga(b.shells, nthreads=1)
    for key, (f1, f2, f3, f4), ijkl in (("llll", (l, l, l, l), (0, 0, 0, 0)),
                                         ("llrr", (l, l, r, r), (0, 0, 1, 1)),
                                         ("lllr", (l, l, l, r), (0, 0, 0, 1)),
                                         ("lrlr", (l, r, l, r), (0, 1, 0, 1))):
        v = m.coulomb(f1, f2, f3, f4)
        assert abs(v - h[key]["value"]) <= 1.5e-8 * h[key]["value"], key
        assert abs(v - huz[M.packed_index(*ijkl)]) < 1e-12, key
    # test/runtests.jl:41-46
    assert abs(m.overlap(l, l) - 1.0) < 1e-12
    assert abs(m.overlap(l, r) - 0.6647387449282997) < 1e-12
    assert abs(m.kinetic(l, l) - 0.76003188) < 1e-8
    assert abs(m.kinetic(l, r) - 0.24141861181119084) < 1e-12
    # all_twoe_ints over the basis by every method, and the 4-D form
    for meth in ("default", "hgp", "rys"):
        v = m.all_twoe_ints(b, meth)
        assert np.max(np.abs(v - huz)) < 1e-12
        A = m.all_twoe_ints_4d(b, meth)
        assert A.shape == (2, 2, 2, 2)
        assert abs(A[0, 0, 1, 1] - huz[M.packed_index(0, 0, 1, 1)]) < 1e-12
        assert abs(A[1, 0, 1, 0] - huz[M.packed_index(0, 1, 0, 1)]) < 1e-12


@gpu
def test_all_twoe_ints_methods_against_huzinaga(oracle):
    _cuda()
    m = M.MolecularIntegrals()
    rng = np.random.default_rng(21)
    sh = mi.Shells.from_list([(rng.uniform(-1.5, 1.5, 3), l, mi.basis._random_shell(rng, l, k, 0.3, 6.0))
                              for l, k in ((0, 3), (1, 2), (2, 1), (3, 1), (0, 1), (1, 1))])
    with oracle.exact_boys():
        ref = oracle.eri_packed_huzinaga(sh, nthreads=4)
    for meth in ("default", "hgp", "rys"):
        got = m.all_twoe_ints(M.Basis.from_shells(sh), meth)
        assert got.shape == ref.shape
        err = float(np.max(np.abs(got - ref)))
        assert err < 1e-11, (meth, err)
