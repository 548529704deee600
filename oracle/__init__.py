"""ORACLE -- test infrastructure only.

CPU restatement of the reference J/K path (ByteQC ``cuobc`` ``get_jk``):
``jk_oracle.c`` (OpenMP C: pair data, Rys recursion, J/K updates, bins,
Schwarz matrix), ``hf_oracle.py`` (the host orchestration of
``cuobc/scf/hf.py``), ``eri_os.py`` (an independent Obara-Saika ERI
algorithm).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg use this package, as the checker; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(['make', '-s', '-C', _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, 'liboracle.so')
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        _LIB.oracle_build_jk.restype = ctypes.c_long
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def rys_roots(n, x):
    s = np.zeros(n)
    w = np.zeros(n)
    err = lib().oracle_rys_roots(ctypes.c_int(n), ctypes.c_double(x), _p(s),
                                 _p(w))
    if err:
        raise ValueError('bad Rys request n=%d x=%g' % (n, x))
    return s, w


def eri_shells(mol, ish, jsh, ksh, lsh):
    """Contracted Cartesian (ij|kl) via the oracle's Rys engine,
    shape (nfi, nfj, nfk, nfl)."""
    from byteqc_b200.gto.mole import ncart
    ls = [mol.bas_angular(s) for s in (ish, jsh, ksh, lsh)]
    nf = [ncart(l) for l in ls]
    out = np.zeros(int(np.prod(nf)))
    lib().oracle_eri_shells(_p(mol._atm), _p(mol._bas), _p(mol._env),
                            ctypes.c_int(mol.nbas), ctypes.c_int(ish),
                            ctypes.c_int(jsh), ctypes.c_int(ksh),
                            ctypes.c_int(lsh), _p(out))
    return out.reshape(nf[::-1]).transpose(3, 2, 1, 0)


def q_cond(mol):
    q = np.zeros((mol.nbas, mol.nbas))
    lib().oracle_q_cond(_p(mol._atm), _p(mol._bas), _p(mol._env),
                        ctypes.c_int(mol.nbas), _p(q))
    return q
