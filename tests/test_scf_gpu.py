"""RHF on the GPU engine: the converged energy agrees with a plain SCF loop
built on the oracle's J/K, and the mixed-precision engine changes the energy
by far less than 1e-6 Eh."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu


def _oracle_scf(mol, tol=1e-10, max_cycle=80):
    from oracle import hf_oracle
    s = mol.intor('int1e_ovlp')
    h = mol.intor('int1e_kin') + mol.intor('int1e_nuc')
    nocc = mol.nelectron // 2
    w, v = np.linalg.eigh(s)
    x = v / np.sqrt(w)
    opt = hf_oracle.VHFOpt(mol).build()

    def solve(f):
        e, c = np.linalg.eigh(x.T @ f @ x)
        return x @ c

    c = solve(h)
    dm = 2 * c[:, :nocc] @ c[:, :nocc].T
    fs, es, e_last = [], [], None
    for _ in range(max_cycle):
        vj, vk = hf_oracle.get_jk(mol, dm, vhfopt=opt)
        f = h + vj - .5 * vk
        e = .5 * np.sum(dm * (h + f)) + mol.energy_nuc()
        if e_last is not None and abs(e - e_last) < tol:
            return e
        e_last = e
        err = x.T @ (f @ dm @ s - s @ dm @ f) @ x
        fs.append(f)
        es.append(err)
        fs, es = fs[-8:], es[-8:]
        n = len(fs)
        if n > 1:
            b = -np.ones((n + 1, n + 1))
            b[-1, -1] = 0
            for i in range(n):
                for j in range(n):
                    b[i, j] = np.sum(es[i] * es[j])
            rhs = np.zeros(n + 1)
            rhs[-1] = -1
            coef = np.linalg.lstsq(b, rhs, rcond=None)[0][:n]
            f = sum(ci * fi for ci, fi in zip(coef, fs))
        c = solve(f)
        dm = 2 * c[:, :nocc] @ c[:, :nocc].T
    raise RuntimeError('oracle SCF did not converge')


def test_rhf_matches_oracle_scf():
    from byteqc_b200.cuobc.scf import RHF
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
               basis='standin-cc-pvdz').build()
    mf = RHF(mol)
    e = mf.kernel()
    assert mf.converged
    e_ref = _oracle_scf(mol)
    assert abs(e - e_ref) < 1e-8, (e, e_ref)


def test_rhf_mixed_precision_energy_error():
    from byteqc_b200.cuobc.scf import RHF
    mol = Mole(atom=geom.water_cluster(4, box=7.0, seed=1),
               basis='standin-6-31g*').build()
    e64 = RHF(mol).kernel()
    mf = RHF(mol, fp32_cutoff=1e-6)
    e32 = mf.kernel()
    assert mf.converged
    assert abs(e32 - e64) < 1e-6, (e32, e64)
