"""The Python surface of MolecularIntegrals.jl's wrapper (python/molecular_integrals.py),
backed by libmolints_cuda.so instead of juliacall and a Julia runtime.

Same names, arguments and results as the reference module:

    coulomb_repulsion(origin_a, norm_a, powers_a, alpha_a, ... d)   python/molecular_integrals.py:68
    PGBF, CGBF, Atom, Basis                                        :132, :188, :262, :301
    MolecularIntegrals().coulomb / coulomb_pgbf                    :385, :367
    MolecularIntegrals().all_twoe_ints(basis, method)              :409-440
    MolecularIntegrals().all_twoe_ints_4d(basis, method)           :442-482
    MolecularIntegrals().overlap / kinetic                         :484-490

Every integral runs on the GPU through the C ABI (include/molints.h): a single integral is the
element of the packed vector of a four-shell basis, so it takes the same kernels as a whole
basis.  ``method`` "default" and "hgp" take the HGP kernels (AUTO's per-class choice for
"default"), "rys" the Rys quadrature kernels; all three return the same normalised values, as
the reference's drivers do.  Unknown methods raise ValueError, like the reference.  There is no
CPU fallback: without the library or a CUDA device these calls raise.
"""
from __future__ import annotations

import math
from typing import List, Optional, Tuple

import numpy as np

from . import basis as _basis
from . import engine as _engine

__all__ = ["coulomb_repulsion", "PGBF", "CGBF", "Atom", "Basis", "MolecularIntegrals",
           "packed_to_4d"]

_METHODS = {"default": _engine.METHOD_AUTO, "hgp": _engine.METHOD_HGP, "rys": _engine.METHOD_RYS}


def _method(method: str) -> int:
    if method not in _METHODS:
        raise ValueError(f"Unknown method: {method}")
    return _METHODS[method]


def _fact2(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def primitive_norm(alpha: float, powers: Tuple[int, int, int]) -> float:
    """The PGBF norm of src/Basis.jl:29-41 (the inverse root of the self-overlap,
    src/OneInts.jl:41-52): (2a/pi)^(3/4) (4a)^(L/2) / sqrt((2I-1)!!(2J-1)!!(2K-1)!!)."""
    I, J, K = powers
    L = I + J + K
    return ((2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (0.5 * L) /
            math.sqrt(_fact2(2 * I - 1) * _fact2(2 * J - 1) * _fact2(2 * K - 1)))


def _component(powers: Tuple[int, int, int]) -> int:
    """Index of a cartesian component within its shell, in shell_indices order."""
    I, J, K = (int(x) for x in powers)
    comps = _basis.shell_components(I + J + K)
    return comps.index((I, J, K))


def _quartet(funcs, method: int, boys: int) -> float:
    """The normalised (ab|cd) of four contracted functions given as (origin, powers,
    exponents, coefficients): one four-shell basis through the engine, one element picked."""
    lst = []
    for origin, powers, ex, co in funcs:
        lst.append((np.asarray(origin, dtype=np.float64), int(sum(powers)), list(zip(ex, co))))
    sh = _basis.Shells.from_list(lst)
    off = sh.fn_offsets()
    idx = [int(off[s]) + _component(f[1]) for s, f in enumerate(funcs)]
    ints = _engine.default_engine().eri_packed(sh, method=method, boys=boys, prim_cutoff=0.0)
    return float(ints[packed_index(*idx)])


def packed_index(i: int, j: int, k: int, l: int) -> int:
    """0-based iindex (src/Utils.jl:14-19)."""
    ij = max(i, j) * (max(i, j) + 1) // 2 + min(i, j)
    kl = max(k, l) * (max(k, l) + 1) // 2 + min(k, l)
    return max(ij, kl) * (max(ij, kl) + 1) // 2 + min(ij, kl)


def packed_to_4d(ints: np.ndarray, n: int) -> np.ndarray:
    """The (n, n, n, n) array of a packed vector: element [i,j,k,l] = ints[iindex(i,j,k,l)]
    (the expansion of python/molecular_integrals.py:460-480, vectorised)."""
    i = np.arange(n)
    pair = np.maximum.outer(i, i) * (np.maximum.outer(i, i) + 1) // 2 + np.minimum.outer(i, i)
    a = pair[:, :, None, None]
    b = pair[None, None, :, :]
    hi, lo = np.maximum(a, b), np.minimum(a, b)
    return np.asarray(ints)[hi * (hi + 1) // 2 + lo]


def coulomb_repulsion(origin_a, norm_a, powers_a, alpha_a,
                      origin_b, norm_b, powers_b, alpha_b,
                      origin_c, norm_c, powers_c, alpha_c,
                      origin_d, norm_d, powers_d, alpha_d) -> float:
    """The ERI of four primitive Gaussians with pyquante2's signature: norm_a ... norm_d times
    the unnormalised primitive integral (python/molecular_integrals.py:68-129, which calls the
    Huzinaga coulomb of src/ERI.jl:15-46).  The engine returns the integral of normalised
    primitives; dividing by their norms gives the unnormalised value."""
    prims = [(origin_a, powers_a, alpha_a), (origin_b, powers_b, alpha_b),
             (origin_c, powers_c, alpha_c), (origin_d, powers_d, alpha_d)]
    v = _quartet([(o, tuple(p), [float(al)], [1.0]) for o, p, al in prims],
                 _engine.METHOD_AUTO, _engine.BOYS_EXACT)
    for _, p, al in prims:
        v /= primitive_norm(float(al), tuple(p))
    return norm_a * norm_b * norm_c * norm_d * v


class PGBF:
    """A primitive Gaussian (python/molecular_integrals.py:132-186): exponent, origin (bohr),
    powers (I, J, K) and its norm, computed as pgbf() does unless given."""

    def __init__(self, expn: float, origin: Tuple[float, float, float] = (0.0, 0.0, 0.0),
                 powers: Tuple[int, int, int] = (0, 0, 0), norm: Optional[float] = None):
        self.expn = float(expn)
        self.origin = tuple(float(x) for x in origin)
        self.powers = tuple(int(x) for x in powers)
        self.norm = primitive_norm(self.expn, self.powers) if norm is None else float(norm)

    def __repr__(self):
        return f"PGBF(expn={self.expn}, origin={self.origin}, powers={self.powers}, norm={self.norm})"


class CGBF:
    """A contracted Gaussian (python/molecular_integrals.py:188-260): origin, powers and the
    primitives' exponents and raw contraction coefficients.  ``norm`` is the contracted norm
    that normalize! gives (src/Basis.jl:73-83), so the function has unit self-overlap."""

    def __init__(self, origin: Tuple[float, float, float] = (0.0, 0.0, 0.0),
                 powers: Tuple[int, int, int] = (0, 0, 0),
                 exponents: Optional[List[float]] = None,
                 coefficients: Optional[List[float]] = None):
        self.origin = tuple(float(x) for x in origin)
        self.powers = tuple(int(x) for x in powers)
        self.exponents = [float(x) for x in (exponents or [])]
        self.coefficients = [float(x) for x in (coefficients or [])]
        if len(self.exponents) != len(self.coefficients):
            raise ValueError("exponents and coefficients differ in length")

    @property
    def norm(self) -> float:
        L = sum(self.powers)
        s = 0.0
        for a, ca in zip(self.exponents, self.coefficients):
            for b, cb in zip(self.exponents, self.coefficients):
                s += ca * cb * (2 * math.sqrt(a * b) / (a + b)) ** (L + 1.5)
        return 1.0 / math.sqrt(s) if s > 0 else float("nan")

    def _spec(self):
        return (self.origin, self.powers, self.exponents, self.coefficients)

    def __repr__(self):
        return f"CGBF(origin={self.origin}, powers={self.powers}, nprims={len(self.exponents)})"


class Atom:
    """An atom: atomic number and position in bohr (python/molecular_integrals.py:262-299)."""

    def __init__(self, atno: int, xyz: Tuple[float, float, float]):
        self.atno = int(atno)
        self.xyz = tuple(float(x) for x in xyz)

    def __repr__(self):
        return f"Atom(atno={self.atno}, xyz={self.xyz})"


class Basis:
    """A basis set over atoms (python/molecular_integrals.py:301-346): build_basis(atoms, name)
    of src/Basis.jl:122-139, functions shell by shell in shell_indices order.  The built-in
    basis set is STO-3G ("sto3g").  ``shells`` is the engine's flat descriptor."""

    def __init__(self, atoms: List[Atom], name: str = "sto3g"):
        ats = [_basis.Atom(a.atno, np.asarray(a.xyz, dtype=np.float64)) for a in atoms]
        self.shells = _basis.build_basis(ats, name)
        self._funcs = []
        sh = self.shells
        for s in range(sh.nshell):
            p0, k = int(sh.prim_off[s]), int(sh.nprim[s])
            for comp in _basis.shell_components(int(sh.L[s])):
                self._funcs.append(CGBF(tuple(sh.xyz[s]), comp, list(sh.expn[p0:p0 + k]),
                                        list(sh.coef[p0:p0 + k])))

    @classmethod
    def from_shells(cls, shells) -> "Basis":
        """A Basis over an existing flat shell descriptor (basis.Shells)."""
        inst = cls.__new__(cls)
        inst.shells = shells
        inst._funcs = []
        for s in range(shells.nshell):
            p0, k = int(shells.prim_off[s]), int(shells.nprim[s])
            for comp in _basis.shell_components(int(shells.L[s])):
                inst._funcs.append(CGBF(tuple(shells.xyz[s]), comp, list(shells.expn[p0:p0 + k]),
                                        list(shells.coef[p0:p0 + k])))
        return inst

    def __len__(self) -> int:
        return len(self._funcs)

    def __getitem__(self, i: int) -> CGBF:
        return self._funcs[i]

    def __iter__(self):
        return iter(self._funcs)

    def __repr__(self):
        return f"Basis(nbf={len(self)})"


def _shells_of(basis):
    return basis.shells if isinstance(basis, Basis) else basis


class MolecularIntegrals:
    """The reference wrapper's high-level interface (python/molecular_integrals.py:348-490),
    computed on the GPU."""

    def coulomb_pgbf(self, a: PGBF, b: PGBF, c: PGBF, d: PGBF) -> float:
        """(ab|cd) of four primitives, each scaled by its own norm (the PGBF coulomb of
        src/ERI.jl:55-60)."""
        v = _quartet([(p.origin, p.powers, [p.expn], [1.0]) for p in (a, b, c, d)],
                     _engine.METHOD_AUTO, _engine.BOYS_EXACT)
        for p in (a, b, c, d):
            v *= p.norm / primitive_norm(p.expn, p.powers)
        return v

    def coulomb(self, a: CGBF, b: CGBF, c: CGBF, d: CGBF) -> float:
        """(ab|cd) of four normalised contracted functions (src/ERI.jl:102)."""
        return _quartet([f._spec() for f in (a, b, c, d)], _engine.METHOD_AUTO, _engine.BOYS_EXACT)

    def all_twoe_ints(self, basis, method: str = "default") -> np.ndarray:
        """Every unique (ij|kl) of the basis, packed in iindex order (src/ERI.jl:104-112);
        method "default", "hgp" or "rys".  ``basis`` is a Basis or a basis.Shells."""
        m = _method(method)
        return _engine.default_engine().eri_packed(_shells_of(basis), method=m,
                                                   boys=_engine.BOYS_EXACT)

    def all_twoe_ints_4d(self, basis, method: str = "default") -> np.ndarray:
        """The same integrals as an (n, n, n, n) array (python/molecular_integrals.py:442-482)."""
        sh = _shells_of(basis)
        return packed_to_4d(self.all_twoe_ints(basis, method), sh.nbf)

    def _one_e(self, a: CGBF, b: CGBF, which: int) -> float:
        lst = [(np.asarray(f.origin), int(sum(f.powers)), list(zip(f.exponents, f.coefficients)))
               for f in (a, b)]
        sh = _basis.Shells.from_list(lst)
        off = sh.fn_offsets()
        S, T, _ = _engine.default_engine().one_e(sh, np.zeros((0, 3)), np.zeros(0))
        mat = (S, T)[which]
        return float(mat[int(off[0]) + _component(a.powers), int(off[1]) + _component(b.powers)])

    def overlap(self, a: CGBF, b: CGBF) -> float:
        """<a|b> (src/OneInts.jl:11-52)."""
        return self._one_e(a, b, 0)

    def kinetic(self, a: CGBF, b: CGBF) -> float:
        """<a|-1/2 nabla^2|b> (src/OneInts.jl:120-135)."""
        return self._one_e(a, b, 1)
