"""Parity against the reference's OWN kernels: ByteQC's cuobc J/K and
ERI-fill library compiled unmodified for sm_100a (oracle/ref/Makefile into
oracle/_ref/) and driven through its C-ABI (GINTbuild_jk, GINTfill_int2e)
by oracle/ref_jk.py in a child process.

Bar: 1e-10 max-abs in J/K elements (absolute), FP64.  The oracle (the CPU
restatement the other parity tests use) is held to the same bar against the
reference's kernels, which pins it to the reference's outputs."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom
from oracle import ref_jk

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_jk.available(),
                                 reason='oracle/_ref not built (needs the '
                                        'reference sources at build time)')]

TOL = 1e-10


def _water(nw, box, seed, basis):
    return Mole(atom=geom.water_cluster(nw, box=box, seed=seed),
                basis=basis).build()


def _scf_dm(mol, seed=1):
    from oracle import gto_oracle
    return geom.scf_like_density(gto_oracle.overlap(mol),
                                 nocc=mol.nelectron // 2, seed=seed)


def _assert_abs(a, b, what):
    err = abs(np.asarray(a) - np.asarray(b)).max()
    assert err <= TOL, '%s: max|diff| %.3e' % (what, err)
    return err


@pytest.mark.parametrize('case', ['h2o8-dz', 'h2o3-tzvp', 'h2o4-631gs'])
def test_get_jk_vs_reference_kernels(case):
    """get_jk against the reference's GINTbuild_jk task loop on the same
    molecule and density: (H2O)8 / cc-pVDZ (9 A cube, seed 0, SCF-like
    density) at full size, and smaller TZVP (f shells) and 6-31G* clusters.
    The oracle is checked against the reference on the same inputs."""
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    nw, box, seed, basis = {
        'h2o8-dz': (8, 9.0, 0, 'standin-cc-pvdz'),
        'h2o3-tzvp': (3, 6.0, 2, 'standin-def2-tzvp'),
        'h2o4-631gs': (4, 6.5, 5, 'standin-6-31g*')}[case]
    mol = _water(nw, box, seed, basis)
    dm = _scf_dm(mol)
    rj, rk, info = ref_jk.run('get_jk', mol, dm)
    vj, vk = hf.get_jk(mol, dm)
    _assert_abs(vj, rj, 'J engine vs reference')
    _assert_abs(vk, rk, 'K engine vs reference')
    oj, ok = hf_oracle.get_jk(mol, dm)
    _assert_abs(oj, rj, 'J oracle vs reference')
    _assert_abs(ok, rk, 'K oracle vs reference')


def test_get_jk_vs_reference_kernels_two_dms_unscreened():
    """Two densities in one call of the engine, no density screen and one
    bin (the reference test's settings, cuobc/test/jk.py:7824), J and K
    separately.  The reference is called once per density: its generic
    digestion does not restart its walk over the integral array for a
    second density (cuobc/lib/gvhf/contract_jk.cu:226-310 leaves idx and idy
    shifted after the first density), so with n_dm > 1 it reads outside that
    array; each density alone goes through its correct path."""
    from byteqc_b200.cuobc.scf import hf
    mol = _water(3, 6.0, 4, 'standin-cc-pvdz')
    rng = np.random.default_rng(3)
    d = rng.random((2, mol.nao, mol.nao))
    dm = d + d.transpose(0, 2, 1)
    ref = [ref_jk.run('get_jk', mol, dm[i], prescreen=False, nbins=1)
           for i in range(2)]
    rj = np.stack([r[0] for r in ref])
    rk = np.stack([r[1] for r in ref])
    opt = hf._VHFOpt(mol).build()
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt, prescreen=False, nbins=1)
    _assert_abs(vj, rj, 'J')
    _assert_abs(vk, rk, 'K')
    vj, _ = hf.get_jk(mol, dm, vhfopt=opt, with_k=False, prescreen=False,
                      nbins=1)
    _assert_abs(vj, rj, 'J only')
    _, vk = hf.get_jk(mol, dm, vhfopt=opt, with_j=False, prescreen=False,
                      nbins=1)
    _assert_abs(vk, rk, 'K only')


def test_get_jk_g_h_shells_vs_reference_kernels():
    """g and h shells (the reference's generic GINTint2e_jk_kernel<8..11>):
    water molecules in the cc-pVDZ stand-in plus uncontracted g and h and a
    contracted g on O, a g on H."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]],
                   [4, [3.0, 0.6], [0.7, 0.5]]],
             'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
           for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=1), basis=bas).build()
    rng = np.random.default_rng(5)
    d = rng.random((mol.nao, mol.nao))
    dm = d + d.T
    rj, rk, _ = ref_jk.run('get_jk', mol, dm)
    vj, vk = hf.get_jk(mol, dm)
    _assert_abs(vj, rj, 'J')
    _assert_abs(vk, rk, 'K')


def test_get_jk_h2o32_tzvp_vs_reference_kernels():
    """The (H2O)32 / def2-TZVP stand-in workload (14 A cube, seed 2; 1376
    functions, classes up to (ff|ff)) at full size."""
    from byteqc_b200.cuobc.scf import hf
    mol = _water(32, 14.0, 2, 'standin-def2-tzvp')
    dm = _scf_dm(mol)
    rj, rk, _ = ref_jk.run('get_jk', mol, dm)
    vj, vk = hf.get_jk(mol, dm)
    _assert_abs(vj, rj, 'J')
    _assert_abs(vk, rk, 'K')


@pytest.mark.parametrize('basis', ['standin-def2-tzvp', 'standin-cc-pvdz'])
def test_fill_int2e_vs_reference_kernels(basis):
    """Every class pair of the ERI tensor of two waters through
    jk_fill_int2e against the reference's GINTfill_int2e with the same
    strides, AO offsets and bins (cuobc/lib/int4c.py:73-127)."""
    from byteqc_b200.cuobc.lib import int4c
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _water(2, 5.0, 0, basis)
    opt = hf._VHFOpt(mol).build(diag_block_with_triu=True)
    ropt = hf_oracle.VHFOpt(mol).build(diag_block_with_triu=True)
    np.testing.assert_array_equal(opt.bas_pairs_locs, ropt.bas_pairs_locs)
    ncp = len(opt.log_qs)
    pairs = [(int(a), int(b)) for a, b in zip(*np.tril_indices(ncp))]
    ref = ref_jk.run('fill_blocks', ropt, pairs, cutoff=opt.direct_scf_tol)
    worst = 0.
    for (cp_ij, cp_kl), rblk in zip(pairs, ref):
        *_, blk = int4c.get_int4c_slice(cp_ij, cp_kl, opt)
        worst = max(worst, _assert_abs(blk.cpu().numpy(), rblk,
                                       'class pair (%d, %d)' % (cp_ij, cp_kl)))
