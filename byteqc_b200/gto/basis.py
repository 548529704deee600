"""Basis-set sources.

Two sources are supported:

* real basis sets, read from NWChem-format text files in a directory named by
  ``BYTEQC_B200_BASIS_DIR`` (one file per basis, ``<name>.nw``; the ``SP``
  shell type is split into S and P).  The reference pulls these by name from
  PySCF's library (``cuobc/test/jk.py:7810``, ``cuobc/test/scf.py:125``);
  no basis data ships with this package;
* synthetic stand-ins ``standin-cc-pvdz``, ``standin-def2-tzvp`` and
  ``standin-6-31g*``.  Each has the shell structure of the named set as PySCF
  stores it -- the same angular momenta, primitive counts and numbers of
  (general) contractions per element, hence the same number of spherical
  functions (H2O: 24, 43 and 18) -- with even-tempered exponents over
  typical ranges and smooth synthetic contraction coefficients.  They
  exercise exactly the integral classes, contraction patterns and
  decontraction paths of the named sets; their energies are not those of
  the named sets.
"""
import os

import numpy as np

from byteqc_b200.gto.mole import charge

_L = {'S': 0, 'P': 1, 'D': 2, 'F': 3, 'G': 4, 'H': 5, 'I': 6}


def parse_nwchem(text, symb=None):
    """Parse NWChem-format basis text -> {symbol: [[l, [e, c...], ...]]}."""
    out = {}
    cur = None
    for raw in text.splitlines():
        line = raw.split('#')[0].strip()
        if not line or line.upper().startswith(('BASIS', 'END')):
            continue
        tok = line.split()
        if tok[0][0].isalpha():
            el = tok[0][0].upper() + tok[0][1:].lower()
            kind = tok[1].upper()
            shells = out.setdefault(el, [])
            if kind == 'SP':
                cur = ('SP', [[0], [1]])
                shells.append(cur[1][0])
                shells.append(cur[1][1])
            else:
                cur = (kind, [[_L[kind]]])
                shells.append(cur[1][0])
            continue
        vals = [float(v.replace('D', 'E').replace('d', 'e')) for v in tok]
        if cur[0] == 'SP':
            cur[1][0].append([vals[0], vals[1]])
            cur[1][1].append([vals[0], vals[2]])
        else:
            cur[1][0].append(vals)
    if symb is not None:
        return out[symb[0].upper() + symb[1:].lower()]
    return out


def _geom(amax, amin, n):
    if n == 1:
        return np.array([amax])
    return amax * (amin / amax) ** (np.arange(n) / (n - 1.))


def _bump(es, center, width=1.1):
    return np.exp(-(np.log(es) - np.log(center)) ** 2 / (2 * width ** 2))


def _contracted(l, es, cols):
    """Shell [l, [e, c0, c1, ...], ...] from exponents and coefficient
    columns."""
    cs = np.stack(cols, axis=1)
    return [l] + [[float(e)] + [float(c) for c in row]
                  for e, row in zip(es, cs)]


def _unit(n, i):
    v = np.zeros(n)
    v[i] = 1.
    return v


# per-element scale of the exponent ranges (roughly Z^2 at the core end)
_ZS = {'H': 1.0, 'C': 0.57, 'N': 0.77, 'O': 1.0}


def _standin_ccpvdz(symb):
    if symb == 'H':
        es = _geom(13.0, 0.122, 4)
        s = _contracted(0, es, [_bump(es, 1.0) * (np.arange(4) < 3),
                                _unit(4, 3)])
        return [s, [1, [0.73, 1.0]]]
    z = _ZS[symb]
    es = _geom(11700. * z, 0.30 * z ** .5, 9)
    core = _bump(es, 200. * z, 1.6)
    val = _bump(es, 1.0 * z, 1.0) - .35 * core
    s = _contracted(0, es, [core, val, _unit(9, 8)])
    ep = _geom(17.7 * z, .275 * z ** .5, 4)
    p = _contracted(1, ep, [_bump(ep, 2.0 * z, 1.2), _unit(4, 3)])
    return [s, p, [2, [1.19 * z ** .5, 1.0]]]


def _standin_def2tzvp(symb):
    if symb == 'H':
        es = _geom(34.1, 1.16, 3)
        return [_contracted(0, es, [_bump(es, 3.0)]),
                [0, [0.327, 1.0]], [0, [0.103, 1.0]], [1, [0.80, 1.0]]]
    z = _ZS[symb]
    e6 = _geom(27000. * z, 8.0 * z, 6)
    e2 = _geom(17.7 * z, 5.3 * z, 2)
    ep = _geom(49.2 * z, 0.70 * z ** .5, 4)
    return [_contracted(0, e6, [_bump(e6, 300. * z, 1.5)]),
            _contracted(0, e2, [np.array([.6, .45])]),
            [0, [0.94 * z ** .5, 1.0]], [0, [0.38 * z ** .5, 1.0]],
            [0, [0.15 * z ** .5, 1.0]],
            _contracted(1, ep, [_bump(ep, 4.0 * z, 1.2)]),
            [1, [0.27 * z ** .5, 1.0]], [1, [0.10 * z ** .5, 1.0]],
            [2, [2.31 * z ** .5, 1.0]], [2, [0.65 * z ** .5, 1.0]],
            [3, [1.43 * z ** .5, 1.0]]]


def _standin_631gs(symb):
    if symb == 'H':
        es = _geom(18.7, 0.64, 3)
        return [_contracted(0, es, [_bump(es, 2.5)]), [0, [0.161, 1.0]]]
    z = _ZS[symb]
    e6 = _geom(5480. * z, 4.0 * z, 6)
    e3 = _geom(15.8 * z, 0.90 * z ** .5, 3)
    return [_contracted(0, e6, [_bump(e6, 60. * z, 1.4)]),
            _contracted(0, e3, [np.array([-.11, .08, 1.0])]),
            _contracted(1, e3, [np.array([.24, .51, .55])]),
            [0, [0.27 * z ** .5, 1.0]], [1, [0.27 * z ** .5, 1.0]],
            [2, [0.80 * z ** .5, 1.0]]]


STANDINS = {
    'standin-cc-pvdz': _standin_ccpvdz,
    'standin-def2-tzvp': _standin_def2tzvp,
    'standin-6-31g*': _standin_631gs,
}


def load(name, symb):
    """Shells of element ``symb`` for basis ``name``."""
    key = name.lower()
    el = symb[0].upper() + symb[1:].lower()
    if key in STANDINS:
        if el not in _ZS:
            raise KeyError('stand-in basis %s has no element %s' % (name, el))
        return STANDINS[key](el)
    bdir = os.environ.get('BYTEQC_B200_BASIS_DIR')
    if bdir:
        for fname in (key + '.nw', key.replace('-', '') + '.nw',
                      key.replace('*', 's') + '.nw'):
            path = os.path.join(bdir, fname)
            if os.path.exists(path):
                with open(path) as f:
                    return parse_nwchem(f.read(), el)
    raise KeyError(
        'basis %r not found: set BYTEQC_B200_BASIS_DIR to a directory of '
        'NWChem-format files, or use one of %s' % (name, sorted(STANDINS)))


def n_spherical(name, symb):
    return sum((2 * s[0] + 1) * (len(s[1]) - 1) for s in load(name, symb))


__all__ = ['load', 'parse_nwchem', 'STANDINS', 'n_spherical', 'charge']
