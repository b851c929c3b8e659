"""Algorithmic work model of the Cholesky-ERI path.

GEMM-type work is counted with the closed formulas of the stages (M - L L^T:
2 NCand NBatch NChol_prev per macro iteration; pivot block: 2 N^3 / 3;
Inv_L products: 2 N^2 x columns; AO->MO: 2 N NA NAO^2 + 2 N NA NB NAO).  ERI
work is counted per canonical class (l_a >= l_b, l_c >= l_d, bra type >= ket
type) from the arithmetic of the reference's W-matrix algorithm
(auto2e_WMatrix_part*.f90: Boys, R_tuv recursion, ket and bra Hermite ->
Cartesian transforms per primitive quartet; HRR and spherical transforms per
contracted quartet), an FMA counted as two flops.  The counts of evaluated
quartets come from the library (gci_stats) or the oracle (orc_stats).
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np


def ncart(l):
    return (l + 1) * (l + 2) // 2


def cart_off(l):
    return l * (l + 1) * (l + 2) // 6


def herm_n(n):
    return (n + 1) * (n + 2) * (n + 3) // 6


def carts(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def pair_types(lmax):
    return [(hi, lo) for hi in range(lmax + 1) for lo in range(hi + 1)]


@lru_cache(maxsize=None)
def class_flops(la, lb, lc, ld, spher=True):
    """(flops per primitive quartet, flops per contracted quartet) of one class."""
    L1, L2 = la + lb, lc + ld
    LT = L1 + L2
    ebra = [c for l in range(la, L1 + 1) for c in carts(l)]
    fket = [c for l in range(lc, L2 + 1) for c in carts(l)]
    H1 = herm_n(L1)
    boys = 30 + 3 * LT
    pref = 25
    rrec = 3 * sum(herm_n(n) for n in range(1, LT + 1))
    s_build = 0
    for fx, fy, fz in fket:
        s_build += H1 * 2 * ((fx + 1) * (fy + 1) * (fz + 1) + (fy + 1) * (fz + 1) + (fz + 1))
    w_acc = len(fket) * sum(2 * ((ex + 1) * (ey + 1) * (ez + 1) + (ey + 1) * (ez + 1) + (ez + 1))
                            for ex, ey, ez in ebra)
    prim = boys + pref + rrec + s_build + w_acc
    nA, nB, nC, nD = ncart(la), ncart(lb), ncart(lc), ncart(ld)
    nf = (lambda l: 2 * l + 1) if spher else ncart
    fA, fB, fC, fD = nf(la), nf(lb), nf(lc), nf(ld)
    NE = len(ebra)
    hrr_k = NE * sum(4 * (dx + 1) * (dy + 1) * (dz + 1) for dx, dy, dz in carts(ld)) * nC
    t_d = 2 * NE * nC * fD * nD
    t_c = 2 * NE * fC * fD * nC
    hrr_b = fC * fD * nA * sum(4 * (bx + 1) * (by + 1) * (bz + 1) for bx, by, bz in carts(lb))
    t_b = 2 * nA * fB * fC * fD * nB
    t_a = 2 * fA * fB * fC * fD * nA
    epi = hrr_k + t_d + t_c + hrr_b + t_b + t_a
    return prim, epi


# Counter layouts: the library (gci_stats) keeps 6 counters per class over
# 10 pair types -- quartets, primitive quartets after the primitive-pair
# screen, integrals, primitive quartets before it, bra primitive pairs x
# quartets, ket primitive pairs x quartets; the oracle (orc_stats) keeps 3
# per class over 21 pair types and evaluates every primitive quartet.
LAYOUTS = {"lib": (10, 6), "oracle": (21, 3)}


def eri_flops(stats: np.ndarray, layout: str, spher=True, unscreened=False) -> float:
    """ERI flops from a work-counter array.  ``unscreened`` counts the primitive
    quartets the reference algorithm evaluates (no primitive screening)."""
    ntypes, nc = LAYOUTS[layout]
    types = pair_types({10: 3, 21: 5}[ntypes])
    col = 3 if (unscreened and nc == 6) else 1
    total = 0.0
    for tb in range(ntypes):
        for tk in range(ntypes):
            base = 8 + nc * (tb * ntypes + tk)
            q, pq = stats[base], stats[base + col]
            if q == 0:
                continue
            (la, lb), (lc, ld) = types[tb], types[tk]
            prim, epi = class_flops(la, lb, lc, ld, spher)
            total += pq * prim + q * epi
    return total


def job_flops(stats: np.ndarray, layout: str, spher=True) -> dict:
    """GEMM + ERI work of a job: ``total`` in the reference algorithm's terms
    (every primitive quartet), ``executed`` what was actually evaluated."""
    gemm = float(np.sum(stats[:5]))
    eri_ref = eri_flops(stats, layout, spher, unscreened=True)
    eri_run = eri_flops(stats, layout, spher, unscreened=False)
    return {"gemm": gemm, "eri": eri_ref, "eri_executed": eri_run, "total": gemm + eri_ref,
            "executed": gemm + eri_run, "integrals": float(stats[7]), "quartets": float(stats[5]),
            "prim_quartets": float(stats[6])}


def pair_supp_sum(la, lb):
    """Hermite products of all Cartesian pairs of shells (la, lb) (two-centre form)."""
    return sum((ax + bx + 1) * (ay + by + 1) * (az + bz + 1) for ax, ay, az in carts(la) for bx, by, bz in carts(lb))


@lru_cache(maxsize=None)
def kernel_class_flops(la, lb, lc, ld, variant, spher=True):
    """Arithmetic of this library's kernels for one class: (per primitive quartet,
    per bra primitive pair x quartet, per ket primitive pair x quartet, per quartet).
    variant 0: bra-first team kernel; 1..3: ket-first kernel (any team width)."""
    L1, L2 = la + lb, lc + ld
    LT = L1 + L2
    H1, H2 = herm_n(L1), herm_n(L2)
    ncb, nck = pair_supp_sum(la, lb), pair_supp_sum(lc, ld)
    nA, nB, nC, nD = ncart(la), ncart(lb), ncart(lc), ncart(ld)
    NE, NF = nA * nB, nC * nD
    boys = 30 + 3 * LT
    pref = 25
    rrec = 3 * sum(herm_n(n) for n in range(1, LT + 1))
    nf = (lambda l: 2 * l + 1) if spher else ncart
    fA, fB, fC, fD = nf(la), nf(lb), nf(lc), nf(ld)
    epi = 2 * NE * nC * fD * nD + 2 * NE * fC * fD * nC + 2 * nA * fB * fC * fD * nB + 2 * fA * fB * fC * fD * nA
    if variant == 0:
        return boys + pref + rrec + 2 * ncb * H2, 0, 2 * NE * nck, epi
    return boys + pref + rrec + 2 * H1 * nck, 2 * ncb * NF, 0, epi


def kernel_flops(stats: np.ndarray, variants: dict, spher=True) -> float:
    """FP64 arithmetic the library's ERI kernels executed, from gci_stats counters and the
    kernel variant of each class ({(tb, tk): variant})."""
    ntypes, nc = LAYOUTS["lib"]
    types = pair_types(3)
    total = 0.0
    for tb in range(ntypes):
        for tk in range(ntypes):
            base = 8 + nc * (tb * ntypes + tk)
            q = stats[base]
            if q == 0:
                continue
            pq, nbp, nkp = stats[base + 1], stats[base + 4], stats[base + 5]
            (la, lb), (lc, ld) = types[tb], types[tk]
            prim, perb, perk, epi = kernel_class_flops(la, lb, lc, ld, variants.get((tb, tk), 0), spher)
            total += pq * prim + nbp * perb + nkp * perk + q * epi
    return total


@lru_cache(maxsize=None)
def grad_class_flops(L1, L2):
    """Flops per primitive quartet of the adjoint potential kernel (grad_engine.cuh)
    for a bra pair of Hermite level L1 and a ket pair of level L2: Boys values
    and prefactor, the in-place R_tuv recursion to level N = L1 + 1 + L2, and
    the contraction V(t) += sum_tau h(tau) R(t + tau) over t <= L1 + 1,
    tau <= L2 (an FMA counted as two flops)."""
    N = L1 + 1 + L2
    boys = 30 + 3 * N
    pref = 25
    rrec = 3 * sum(herm_n(N - j) - 1 for j in range(N))
    contraction = 2 * herm_n(L1 + 1) * herm_n(L2)
    return boys + pref + rrec + contraction


def grad_flops(work: np.ndarray) -> float:
    """Total flops of one gci_coulomb_grad call from gci_coulomb_grad_work
    (primitive quartets per (L1, L2), 7 x 7)."""
    w = np.asarray(work).reshape(7, 7)
    return float(sum(w[a, b] * grad_class_flops(a, b) for a in range(7) for b in range(7)))
