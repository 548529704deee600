"""Three- and two-centre density-fitting integrals (byteqc_b200.cuobc.lib.
int3c, the counterpart of the reference's cuobc/lib/int3c.py) against the
oracle's shell quartets on the same concatenated basis (molecule, the
exponent-0 s shell, auxiliary basis).  Tolerance: 1e-10 max-abs relative to
max(1, max|block|)."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu

TOL = 1e-10

AUX = {'O': [[0, [8.0, 1.0]], [0, [2.0, 1.0]], [0, [0.5, 1.0]],
             [1, [3.0, 1.0]], [1, [0.8, 1.0]], [2, [1.5, 1.0]],
             [3, [1.1, 1.0]]],
       'H': [[0, [3.0, 1.0]], [0, [0.6, 1.0]], [1, [1.0, 1.0]]]}


def _setup():
    from byteqc_b200.cuobc.lib import int3c
    atoms = geom.water_cluster(2, box=5.0, seed=4)
    mol = Mole(atom=atoms, basis='standin-cc-pvdz').build()
    aux = Mole(atom=atoms, basis=AUX).build()
    opt = int3c.VHFOpt3c(mol, aux, 'int3c2e').build(diag_block_with_triu=True)
    return opt


def test_int3c_blocks_vs_oracle():
    import oracle
    from byteqc_b200.cuobc.lib import int3c
    opt = _setup()
    tot = opt.tot_mol
    nbas = opt.mol.nbas
    fake = nbas  # the exponent-0 shell follows the molecule's shells
    aux0 = nbas + 1
    ao = opt.ao_loc
    aao = opt.aux_ao_loc
    worst = 0.
    for cp in range(len(opt.log_qs)):
        for ca in range(len(opt.aux_log_qs)):
            for order in ('F', 'C'):
                si, sj, sk, blk = int3c.get_int3c(cp, ca, opt, order=order)
                blk = blk.cpu().numpy()
                cpi, cpj = int3c.ind2pair(cp)
                ish = range(opt.l_ctr_offsets[cpi], opt.l_ctr_offsets[cpi + 1])
                jsh = range(opt.l_ctr_offsets[cpj], opt.l_ctr_offsets[cpj + 1])
                ksh = range(opt.aux_l_ctr_offsets[ca], opt.aux_l_ctr_offsets[ca + 1])
                for i in ish:
                    for j in jsh:
                        for k in ksh:
                            ref = oracle.eri_shells(tot, i, j, aux0 + k, fake)[..., 0]
                            got = blk[ao[i] - si.start:ao[i + 1] - si.start,
                                      ao[j] - sj.start:ao[j + 1] - sj.start,
                                      aao[k] - sk.start:aao[k + 1] - sk.start]
                            worst = max(worst, abs(got - ref).max() / max(1., abs(ref).max()))
    assert worst <= TOL, worst


def test_int2c_metric_and_factor_vs_oracle():
    import oracle
    import torch
    from byteqc_b200.cuobc.lib import int3c
    opt = _setup()
    tot = opt.tot_mol
    nbas = opt.mol.nbas
    fake, aux0 = nbas, nbas + 1
    aao = opt.aux_ao_loc
    naux = opt.auxmol.nbas
    j2 = int3c.get_int2c_metric(opt).cpu().numpy()
    ref = np.zeros_like(j2)
    for p in range(naux):
        for q in range(naux):
            ref[aao[p]:aao[p + 1], aao[q]:aao[q + 1]] = oracle.eri_shells(
                tot, aux0 + p, fake, aux0 + q, fake)[:, 0, :, 0]
    assert abs(j2 - ref).max() <= TOL * max(1., abs(ref).max())
    # Cholesky factor of the metric in the input auxiliary basis
    L = int3c.get_int2c(opt).cpu().numpy()
    c = opt.auxcoeff
    m = c.T @ ref @ c
    assert abs(L @ L.T - m).max() <= 1e-9 * abs(m).max()
    # the eigenvector form spans the same inverse metric
    V = int3c.get_int2c(opt, j2c_eig_always=True).cpu().numpy()
    assert abs(V @ V.T @ m - np.eye(len(m))).max() <= 1e-6
