"""ORACLE (test infrastructure only): an independent second algorithm for
contracted Cartesian ERIs -- Obara-Saika / Head-Gordon-Pople recursions on
the Boys function -- used to cross-check the Rys engines at the integral
level.  It shares no code with the Rys paths: the Boys function comes from
scipy's regularised incomplete gamma function and the recursions run over
Cartesian index tuples.  Slow (pure Python); meant for a handful of shell
quartets.  Normalisation follows libcint (s/p common factors applied, see
cuobc/lib/gint/pair_data.c:27-28), so results compare one-to-one with the
reference's Cartesian integrals.
"""
import math
from functools import lru_cache

import numpy as np
from scipy.special import gamma, gammainc

FAC_SP = {0: 0.282094791773878143, 1: 0.488602511902919921}


def boys(m, t):
    if t < 1e-13:
        return 1. / (2 * m + 1) - t / (2 * m + 3)
    a = m + .5
    return .5 * t ** (-a) * gamma(a) * gammainc(a, t)


def cart_list(l):
    return [(a, b, l - a - b) for a in range(l, -1, -1)
            for b in range(l - a, -1, -1)]


def _prim_eri(la, lb, lc, ld, a, b, c, d, A, B, C, D):
    p, q = a + b, c + d
    P = (a * A + b * B) / p
    Q = (c * C + d * D) / q
    W = (p * P + q * Q) / (p + q)
    rho = p * q / (p + q)
    T = rho * np.dot(P - Q, P - Q)
    kab = math.exp(-a * b / p * np.dot(A - B, A - B))
    kcd = math.exp(-c * d / q * np.dot(C - D, C - D))
    pre = 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * kab * kcd
    L = la + lb + lc + ld
    fm = [pre * boys(m, T) for m in range(L + 1)]
    PA, WP, QC, WQ = P - A, W - P, Q - C, W - Q

    @lru_cache(maxsize=None)
    def vrr(e, f, m):
        if min(e) < 0 or min(f) < 0:
            return 0.
        if sum(f) == 0:
            if sum(e) == 0:
                return fm[m]
            i = next(k for k in range(3) if e[k] > 0)
            em = list(e)
            em[i] -= 1
            em = tuple(em)
            em2 = list(em)
            em2[i] -= 1
            em2 = tuple(em2)
            v = PA[i] * vrr(em, f, m) + WP[i] * vrr(em, f, m + 1)
            if em[i] > 0:
                v += em[i] / (2 * p) * (vrr(em2, f, m)
                                        - rho / p * vrr(em2, f, m + 1))
            return v
        i = next(k for k in range(3) if f[k] > 0)
        fm1 = list(f)
        fm1[i] -= 1
        fm1 = tuple(fm1)
        fm2 = list(fm1)
        fm2[i] -= 1
        fm2 = tuple(fm2)
        v = QC[i] * vrr(e, fm1, m) + WQ[i] * vrr(e, fm1, m + 1)
        if fm1[i] > 0:
            v += fm1[i] / (2 * q) * (vrr(e, fm2, m)
                                     - rho / q * vrr(e, fm2, m + 1))
        if e[i] > 0:
            em = list(e)
            em[i] -= 1
            v += e[i] / (2 * (p + q)) * vrr(tuple(em), fm1, m + 1)
        return v

    AB, CD = A - B, C - D

    @lru_cache(maxsize=None)
    def hrr(ea, eb, ec, ed):
        if sum(eb) > 0:
            i = next(k for k in range(3) if eb[k] > 0)
            a1 = list(ea)
            a1[i] += 1
            b1 = list(eb)
            b1[i] -= 1
            return (hrr(tuple(a1), tuple(b1), ec, ed)
                    + AB[i] * hrr(ea, tuple(b1), ec, ed))
        if sum(ed) > 0:
            i = next(k for k in range(3) if ed[k] > 0)
            c1 = list(ec)
            c1[i] += 1
            d1 = list(ed)
            d1[i] -= 1
            return (hrr(ea, eb, tuple(c1), tuple(d1))
                    + CD[i] * hrr(ea, eb, ec, tuple(d1)))
        return vrr(ea, ec, 0)

    ca, cb, cc, cd = (cart_list(la), cart_list(lb), cart_list(lc),
                      cart_list(ld))
    out = np.empty((len(ca), len(cb), len(cc), len(cd)))
    for i, ea in enumerate(ca):
        for j, eb in enumerate(cb):
            for k, ec in enumerate(cc):
                for l, ed in enumerate(cd):
                    out[i, j, k, l] = hrr(ea, eb, ec, ed)
    return out


def eri_shells(mol, ish, jsh, ksh, lsh):
    """Contracted Cartesian (ij|kl) for one shell quartet of ``mol`` (first
    contraction of every shell), array (nfi, nfj, nfk, nfl)."""
    sh = [ish, jsh, ksh, lsh]
    ls = [mol.bas_angular(s) for s in sh]
    cen = [mol.atom_coords()[mol._bas[s, 0]] for s in sh]
    exps = [mol.bas_exp(s) for s in sh]
    cofs = [mol.bas_ctr_coeff(s)[:, 0] for s in sh]
    out = 0.
    for pa, ca in zip(exps[0], cofs[0]):
        for pb, cb in zip(exps[1], cofs[1]):
            for pc, cc in zip(exps[2], cofs[2]):
                for pd, cd in zip(exps[3], cofs[3]):
                    out = out + ca * cb * cc * cd * _prim_eri(
                        *ls, pa, pb, pc, pd, *cen)
    for l in ls:
        out = out * FAC_SP.get(l, 1.)
    return out
