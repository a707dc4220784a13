"""Basis sets as flat shell arrays, plus seeded generators for the benchmark molecules.

This mirrors the parts of MolecularIntegrals.jl that produce the ERI path's input:
``atom`` (src/Atoms.jl:11-17, Angstrom -> bohr by dividing by 0.52918), ``build_basis``
(src/Basis.jl:122-139: shells in atom order, components in ``shell_indices`` order) and the
STO-3G table (src/Data.jl:5-120, shipped as data/sto3g.json).  A basis is held the way the
C ABI takes it: one row per shell with its centre, angular momentum and a slice of the
primitive arrays (raw exponents and raw contraction coefficients, i.e. ``Shell.expns`` and
``Shell.coefs``).  Normalisation is applied by the engine, as ``build_basis`` does.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ANGSTROM_TO_BOHR_DIVISOR = 0.52918  # src/Atoms.jl:15
LVALUE = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}
_DATA = Path(__file__).resolve().parent / "data"


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def shell_components(l: int):
    """Cartesian powers of a shell in the reference order (src/Basis.jl:269-279).

    x-power descending then y-power descending, except that l=3 lists xzz before xyz."""
    comps = [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]
    if l == 3:
        comps[4], comps[5] = comps[5], comps[4]
    return comps


@dataclass
class Atom:
    atno: int
    xyz: np.ndarray  # bohr


def atom(atno: int, x: float, y: float, z: float, units: str = "Angstrom") -> Atom:
    """atom(atno,x,y,z) (src/Atoms.jl:12-17)."""
    xyz = np.array([x, y, z], dtype=np.float64)
    if units == "Angstrom":
        xyz = xyz / ANGSTROM_TO_BOHR_DIVISOR
    return Atom(atno, xyz)


@dataclass
class Shells:
    """Flat shell arrays: the engine's (and the C ABI's) basis descriptor."""
    xyz: np.ndarray        # [nshell, 3] bohr
    L: np.ndarray          # [nshell] int32
    nprim: np.ndarray      # [nshell] int32
    prim_off: np.ndarray   # [nshell] int32
    expn: np.ndarray       # [nprim_total]
    coef: np.ndarray       # [nprim_total], raw contraction coefficients
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nshell(self) -> int:
        return int(len(self.L))

    @property
    def nbf(self) -> int:
        return int(sum(ncart(int(l)) for l in self.L))

    @property
    def npacked(self) -> int:
        n = self.nbf
        return n * (n + 1) * (n * n + n + 2) // 8

    def fn_offsets(self) -> np.ndarray:
        off = np.zeros(self.nshell + 1, dtype=np.int64)
        off[1:] = np.cumsum([ncart(int(l)) for l in self.L])
        return off

    @staticmethod
    def from_list(shell_list, name: str = "") -> "Shells":
        """shell_list: iterable of (xyz_bohr, L, [(expn, coef), ...])."""
        xyz, L, nprim, poff, ex, co = [], [], [], [], [], []
        for center, l, prims in shell_list:
            xyz.append(np.asarray(center, dtype=np.float64))
            L.append(int(l))
            poff.append(len(ex))
            nprim.append(len(prims))
            for e, c in prims:
                ex.append(float(e))
                co.append(float(c))
        return Shells(np.array(xyz, dtype=np.float64).reshape(-1, 3),
                      np.array(L, dtype=np.int32), np.array(nprim, dtype=np.int32),
                      np.array(poff, dtype=np.int32), np.array(ex, dtype=np.float64),
                      np.array(co, dtype=np.float64), name)


def load_sto3g() -> dict:
    with open(_DATA / "sto3g.json") as fh:
        data = json.load(fh)["elements"]
    return {int(z): [(LVALUE[sym], prims) for sym, prims in shells] for z, shells in data.items()}


def build_basis(atoms, name: str = "sto3g") -> Shells:
    """build_basis(atoms, name) (src/Basis.jl:122-139) for the built-in STO-3G set."""
    if name != "sto3g":
        raise KeyError(f"basis {name!r} is not shipped; pass explicit shells instead")
    table = load_sto3g()
    lst = []
    for at in atoms:
        for l, prims in table[at.atno]:
            lst.append((at.xyz, l, prims))
    return Shells.from_list(lst, name)


# ----------------------------------------------------------------- sample molecules
def h2():
    """h2 (src/Data.jl:1188-1189)."""
    return [atom(1, 0.0, 0.0, 0.36628549), atom(1, 0.0, 0.0, -0.36628549)]


def ethane_staggered():
    """Staggered ethane: C-C 1.54 A along z, C-H 1.09 A, H-C-C 109.47 deg, ends 60 deg apart."""
    cc, ch, ang = 1.54, 1.09, math.radians(180.0 - 109.47)
    atoms = [atom(6, 0.0, 0.0, cc / 2), atom(6, 0.0, 0.0, -cc / 2)]
    for sign, phis in ((+1, (0.0, 120.0, 240.0)), (-1, (60.0, 180.0, 300.0))):
        for phi in phis:
            p = math.radians(phi)
            r = ch * math.sin(ang)
            atoms.append(atom(1, r * math.cos(p), r * math.sin(p),
                              sign * (cc / 2 + ch * math.cos(ang))))
    return atoms


# ----------------------------------------------------------------- synthetic shells
def _random_shell(rng, l: int, k: int, lo: float, hi: float):
    ex = np.sort(np.exp(rng.uniform(math.log(lo), math.log(hi), size=k)))[::-1]
    co = rng.normal(size=k)
    # renormalise the raw coefficients to a unit contracted function, as normalize! would
    s = 0.0
    for i in range(k):
        for j in range(k):
            s += co[i] * co[j] * (2 * math.sqrt(ex[i] * ex[j]) / (ex[i] + ex[j])) ** (l + 1.5)
    co = co / math.sqrt(s)
    return [(float(e), float(c)) for e, c in zip(ex, co)]


SPLIT_VALENCE_HEAVY = [(0, 6), (0, 3), (1, 3), (0, 1), (1, 1)]
SPLIT_VALENCE_H = [(0, 3), (0, 1)]
POLARISED_C = [(0, 7), (0, 7), (0, 1), (1, 3), (1, 1), (2, 1)]
POLARISED_H = [(0, 3), (0, 1), (1, 1)]


def _lattice_atoms(rng, nheavy: int, nh: int, spacing=1.4, jitter=0.3, dmin=0.9):
    """nheavy + nh atoms on a jittered cubic lattice (Angstrom), pairwise >= dmin apart."""
    ntot = nheavy + nh
    side = int(math.ceil(ntot ** (1 / 3))) + 1
    sites = [(i, j, k) for i in range(side) for j in range(side) for k in range(side)]
    while True:
        idx = rng.choice(len(sites), size=ntot, replace=False)
        pos = np.array([sites[i] for i in idx], dtype=np.float64) * spacing
        pos += rng.uniform(-jitter, jitter, size=pos.shape)
        d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
        np.fill_diagonal(d, 1e9)
        if d.min() >= dmin:
            return pos


def synthetic_molecule(seed: int, nheavy: int, nh: int, heavy_recipe, h_recipe,
                       lo: float, hi: float, name: str, heavy_extra=()) -> Shells:
    rng = np.random.default_rng(seed)
    pos = _lattice_atoms(rng, nheavy, nh)
    lst = []
    for a in range(nheavy + nh):
        xyz = pos[a] / ANGSTROM_TO_BOHR_DIVISOR
        recipe = list(heavy_recipe) + list(heavy_extra) if a < nheavy else h_recipe
        for l, k in recipe:
            lst.append((xyz, l, _random_shell(rng, l, k, lo, hi)))
    sh = Shells.from_list(lst, name)
    sh.meta = {"seed": seed, "natom": nheavy + nh, "nheavy": nheavy}
    return sh


def config0() -> Shells:
    """Staggered ethane in the built-in STO-3G basis (16 functions)."""
    sh = build_basis(ethane_staggered(), "sto3g")
    sh.name = "ethane_sto3g"
    return sh


def config1(seed: int = 1) -> Shells:
    """24-atom split-valence molecule (8 heavy + 16 H), l<=1, 104 functions."""
    return synthetic_molecule(seed, 8, 16, SPLIT_VALENCE_HEAVY, SPLIT_VALENCE_H, 0.1, 5e3,
                              "split_valence_24")


def config2(seed: int = 2) -> Shells:
    """Staggered ethane with a synthetic polarised basis (l<=2, 60 cartesian functions)."""
    rng = np.random.default_rng(seed)
    lst = []
    for at in ethane_staggered():
        recipe = POLARISED_C if at.atno == 6 else POLARISED_H
        for l, k in recipe:
            lst.append((at.xyz, l, _random_shell(rng, l, k, 0.1, 1e4)))
    sh = Shells.from_list(lst, "ethane_polarised")
    sh.meta = {"seed": seed}
    return sh


def config3_molecule(m: int) -> Shells:
    """Molecule m of the 256-molecule batch: 4-40 atoms, a third heavy, l<=2, K in {1,3,6,7}."""
    rng = np.random.default_rng(3000 + m)
    natom = int(rng.integers(4, 41))
    nheavy = max(1, natom // 3)
    if m % 2 == 0:
        return synthetic_molecule(3000 + m, nheavy, natom - nheavy, SPLIT_VALENCE_HEAVY,
                                  SPLIT_VALENCE_H, 0.1, 5e3, f"batch{m}")
    return synthetic_molecule(3000 + m, nheavy, natom - nheavy, POLARISED_C, POLARISED_H,
                              0.1, 1e4, f"batch{m}")


def config3(nmol: int = 256):
    return [config3_molecule(m) for m in range(nmol)]


def config4_request(r: int, with_f: bool = True) -> Shells:
    """Serving request r: 10-300 cartesian functions, l<=3 (heavy atoms may carry f)."""
    rng = np.random.default_rng(4_000_000 + r)
    natom = int(rng.integers(2, 26))
    nheavy = max(1, natom // 3)
    extra = [(3, 1)] if (with_f and rng.uniform() < 0.5) else []
    return synthetic_molecule(4_000_000 + r, nheavy, natom - nheavy, POLARISED_C, POLARISED_H,
                              0.1, 1e4, f"req{r}", heavy_extra=extra)


def config4_arrivals(rate: float = 200.0, window_s: float = 30.0, seed: int = 4):
    """Poisson arrival times (s) of the serving stream."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window_s:
            return out
        out.append(t)
