"""ORACLE (test infrastructure only): the basis-function conventions that
the reference takes from PySCF/libcint (``cuobc/scf/hf.py:527`` calls
``gto.gto_norm``, ``:555`` calls ``mol.cart2sph_coeff()``; PySCF 2.5.0 is not
vendored), derived here independently of the product's ``byteqc_b200.gto``
so that a wrong normalisation or a wrong Cartesian-to-spherical matrix
cannot cancel between the product and the oracle:

  - ``gto_norm``: 1 / sqrt(int_0^inf r^(2l+2) exp(-2 a r^2) dr), from
    scipy's gamma function;
  - ``cart2sph``: the real spherical harmonics of scipy (``sph_harm_y``,
    which carries the Condon-Shortley phase) turned into libcint's real
    form (m = -l..l, sine terms for m < 0, no Condon-Shortley phase), and
    the Cartesian coefficients of r^l Y_lm obtained by a least-squares fit
    on points of the unit sphere (the degree-l monomials are linearly
    independent there); p shells keep libcint's (x, y, z) order;
  - ``overlap``: the overlap matrix of a molecule in its own (contracted,
    spherical or Cartesian) basis, from the C oracle's Cartesian overlap
    of the decontracted working basis and this module's transforms.
"""
import ctypes
import math

import numpy as np
from scipy import special

import oracle

ANG_OF, NPRIM_OF, NCTR_OF, PTR_COEFF = 1, 2, 3, 6


def gto_norm(l, expnt):
    expnt = np.asarray(expnt, dtype=np.float64)
    n = 2 * l + 2
    integral = special.gamma((n + 1) / 2.) / (2. * (2. * expnt) ** ((n + 1) / 2.))
    return 1. / np.sqrt(integral)


def _cart_powers(l):
    return [(a, b, l - a - b) for a in range(l, -1, -1)
            for b in range(l - a, -1, -1)]


def _real_ylm(l, m, theta, phi):
    if m == 0:
        return special.sph_harm_y(l, 0, theta, phi).real
    y = special.sph_harm_y(l, abs(m), theta, phi)
    part = y.real if m > 0 else y.imag
    return math.sqrt(2.) * (-1) ** abs(m) * part


_C2S = {}


def cart2sph(l):
    """(ncart(l), 2l+1) coefficients of r^l Y_lm over x^a y^b z^c."""
    if l in _C2S:
        return _C2S[l]
    if l == 0:
        c = np.ones((1, 1))
    elif l == 1:
        c = np.eye(3)
    else:
        rng = np.random.default_rng(12345 + l)
        npt = 40 * (l + 1) ** 2
        v = rng.normal(size=(npt, 3))
        v /= np.linalg.norm(v, axis=1)[:, None]
        theta = np.arccos(np.clip(v[:, 2], -1, 1))
        phi = np.arctan2(v[:, 1], v[:, 0])
        pows = _cart_powers(l)
        M = np.stack([v[:, 0] ** a * v[:, 1] ** b * v[:, 2] ** cc
                      for a, b, cc in pows], axis=1)
        Y = np.stack([_real_ylm(l, m, theta, phi) for m in range(-l, l + 1)],
                     axis=1)
        c, *_ = np.linalg.lstsq(M, Y, rcond=None)
        c[abs(c) < 1e-13] = 0.
    _C2S[l] = c
    return c


def cart2sph_coeff(mol):
    """Block-diagonal (nao_cart, nao_sph) transform over the shells of
    ``mol`` (every contraction of a shell gets its own block)."""
    bas = mol._bas
    ls = bas[:, ANG_OF]
    nctr = bas[:, NCTR_OF]
    nc = ((ls + 1) * (ls + 2) // 2 * nctr).sum()
    ns = ((2 * ls + 1) * nctr).sum()
    out = np.zeros((nc, ns))
    r = c = 0
    for l, n in zip(ls, nctr):
        blk = cart2sph(int(l))
        for _ in range(n):
            out[r:r + blk.shape[0], c:c + blk.shape[1]] = blk
            r += blk.shape[0]
            c += blk.shape[1]
    return out


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def overlap_working(pmol):
    """Cartesian overlap of a basis whose shells carry one contraction."""
    atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
    env = np.ascontiguousarray(pmol._env, dtype=np.float64)
    ls = bas[:, ANG_OF]
    ao_loc = np.append(0, np.cumsum((ls + 1) * (ls + 2) // 2)).astype(np.int32)
    n = int(ao_loc[-1])
    out = np.zeros((n, n))
    rc = oracle.lib().oracle_ovlp_cart(_ptr(atm), _ptr(bas), _ptr(env),
                                       ctypes.c_int(pmol.nbas), _ptr(ao_loc),
                                       _ptr(out))
    if rc:
        raise ValueError('oracle_ovlp_cart: unsupported shell')
    return out


def overlap(mol):
    """Overlap matrix of ``mol`` in its own basis: the decontracted working
    basis of the oracle's basis_seg_contraction (without the (l, nprim)
    sort), its Cartesian overlap, and the coefficient transform."""
    from oracle import hf_oracle
    pmol, coeff = hf_oracle.basis_seg_contraction(mol)
    s = overlap_working(pmol)
    return coeff.T @ s @ coeff
