"""Algorithmic work of the ERI path, counted on the reference algorithm (not on the
generated kernels), for roofline figures.

Per shell quartet of class (la lb|lc ld) with K_abcd primitive quartets:

    FLOP = K_abcd * (V(e, f) + 2 nao(e) nao(f) + S(e+f+1)) + H(la, lb, lc, ld)

  * V: the VRR of vrr! (src/HGP.jl:180-240) for amax = e = la+lb, cmax = f = lc+ld, walking
    the reference's own loops: 3 FLOP per line (PA*v + WP*v), +4 for the a_i/2zeta(...) term
    of the a-build, +2 for the a_i/2(zeta+eta) cross term and +4 for the c_i/2eta(...) term
    of the c-build;
  * 2 nao(e) nao(f): the contraction cvrrs += c * vrrs (src/HGP.jl:62-64);
  * S = 20 + 3 mmax: prefactors and the Boys recursion per primitive quartet;
  * H: the HRR loops of chrr (src/HGP.jl:93-114) at 2 FLOP per element.
Bytes of a quartet are its packed stores (8 B per unique integral).
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np


def _tables(lmax):
    ao = []
    nao = []
    for l in range(lmax + 1):
        comps = [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]
        if l == 3:
            comps[4], comps[5] = comps[5], comps[4]
        ao.extend(comps)
        nao.append(len(ao))
    idx = {c: i for i, c in enumerate(ao)}
    return ao, nao, idx


AO, NAO, IDX = _tables(8)


def _shell(a):
    return sum(AO[a])


def _dir(a):
    m = AO[a]
    return max(range(3), key=lambda i: (m[i], -i))


def _minus(a, i):
    m = list(AO[a])
    if m[i] == 0:
        return -1
    m[i] -= 1
    return IDX[tuple(m)]


@lru_cache(maxsize=None)
def vrr_flops(amax: int, cmax: int) -> int:
    mmax = amax + cmax + 1
    f = 0
    for aplus in range(1, NAO[amax]):
        i = _dir(aplus)
        a = _minus(aplus, i)
        lim = mmax - _shell(aplus)
        f += lim * (7 if _minus(a, i) >= 0 else 3)
    for cplus in range(1, NAO[cmax]):
        i = _dir(cplus)
        c = _minus(cplus, i)
        cminus = _minus(c, i)
        for a in range(NAO[amax]):
            lim = mmax - _shell(cplus) - _shell(a)
            if lim <= 0:
                continue
            per = 3 + (2 if _minus(a, i) >= 0 else 0) + (4 if cminus >= 0 else 0)
            f += lim * per
    return f


@lru_cache(maxsize=None)
def hrr_flops(la: int, lb: int, lc: int, ld: int) -> int:
    n = 0
    ncc = NAO[lc + ld]
    for bplus in range(1, NAO[lb]):
        j = _dir(bplus)
        b = _minus(bplus, j)
        n += ncc * NAO[la + lb - _shell(b) - 1]
    for dplus in range(1, NAO[ld]):
        j = _dir(dplus)
        d = _minus(dplus, j)
        n += NAO[lc + ld - _shell(d) - 1] * NAO[lb] * NAO[la]
    return 2 * n


def per_prim_flops(la, lb, lc, ld) -> int:
    e, f = la + lb, lc + ld
    return vrr_flops(e, f) + 2 * NAO[e] * NAO[f] + 20 + 3 * (e + f + 1)


def class_of_pair(la, lb):
    return (la, lb) if la >= lb else (lb, la)


def workload(shells):
    """Algorithmic FLOPs, shell quartets and primitive quartets of one basis, per class
    pair (bra class >= ket class in the engine's order) and in total."""
    L = np.asarray(shells.L)
    K = np.asarray(shells.nprim)
    ns = len(L)
    order = sorted({class_of_pair(int(a), int(b)) for a in L for b in L},
                   key=lambda c: (c[0] + c[1], c[0]))
    groups = {c: [] for c in order}
    for i in range(ns):
        for j in range(i + 1):
            groups[class_of_pair(int(L[i]), int(L[j]))].append(int(K[i]) * int(K[j]))
    out = {}
    tot = {"flop": 0.0, "quartets": 0, "prim_quartets": 0}
    for xi, X in enumerate(order):
        kx = np.array(groups[X], dtype=np.float64)
        for Y in order[:xi + 1]:
            ky = np.array(groups[Y], dtype=np.float64)
            if X == Y:
                nq = len(kx) * (len(kx) + 1) // 2
                kq = (kx.sum() ** 2 + (kx ** 2).sum()) / 2
            else:
                nq = len(kx) * len(ky)
                kq = kx.sum() * ky.sum()
            bra, ket = (X, Y) if X[0] + X[1] >= Y[0] + Y[1] else (Y, X)
            fl = kq * per_prim_flops(*bra, *ket) + nq * hrr_flops(*bra, *ket)
            tag = "".join("spdfg"[l] for l in (*X, *Y))
            out[tag] = {"flop": fl, "quartets": nq, "prim_quartets": kq}
            tot["flop"] += fl
            tot["quartets"] += nq
            tot["prim_quartets"] += kq
    return out, tot
