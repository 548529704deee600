"""Host-side logic that needs no GPU: the working-basis construction, the
stand-in basis sets, the geometry generators and the one-electron
integrals."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom, basis as gbasis
from byteqc_b200.gto.mole import cart2sph


@pytest.mark.parametrize('bname', ['standin-cc-pvdz', 'standin-6-31g*',
                                   'standin-def2-tzvp'])
def test_seg_contraction_matches_oracle(bname):
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = Mole(atom=geom.water_cluster(3, box=6.0, seed=1), basis=bname).build()
    pmol, c = hf.basis_seg_contraction(mol)
    rmol, rc = hf_oracle.basis_seg_contraction(mol)
    np.testing.assert_array_equal(pmol._bas, rmol._bas)
    # the oracle computes its primitive norms independently (scipy's gamma
    # function): equal to rounding
    np.testing.assert_allclose(pmol._env, rmol._env, rtol=1e-15, atol=0)
    np.testing.assert_allclose(c, rc, rtol=1e-14, atol=1e-15)
    # the working basis reproduces the contracted overlap
    s0 = mol.intor('int1e_ovlp')
    s1 = pmol.intor('int1e_ovlp')
    np.testing.assert_allclose(c.T @ s1 @ c, s0, atol=1e-12)


def test_standin_sizes():
    # spherical functions per water: cc-pVDZ 24, def2-TZVP 43, 6-31G* 18
    for b, n in (('standin-cc-pvdz', 24), ('standin-def2-tzvp', 43),
                 ('standin-6-31g*', 18)):
        assert gbasis.n_spherical(b, 'O') + 2 * gbasis.n_spherical(b, 'H') == n
    mol = Mole(atom=geom.water_cluster(8, box=9.0, seed=0),
               basis='standin-cc-pvdz').build()
    assert mol.nao == 192
    mol = Mole(atom=geom.water_cluster(32, box=14.0, seed=2),
               basis='standin-def2-tzvp').build()
    assert mol.nao == 1376


def test_water_cluster_constraints():
    atoms = geom.water_cluster(16, box=11.0, seed=5)
    xyz = np.array([a[1] for a in atoms])
    o = xyz[0::3]
    d = np.linalg.norm(o[:, None] - o[None], axis=-1)
    assert d[np.triu_indices(len(o), 1)].min() >= 2.6
    assert (o >= 0).all() and (o <= 11.0).all()
    for i in range(16):
        oh1 = np.linalg.norm(xyz[3 * i + 1] - xyz[3 * i])
        oh2 = np.linalg.norm(xyz[3 * i + 2] - xyz[3 * i])
        ang = np.degrees(np.arccos(np.dot(xyz[3 * i + 1] - xyz[3 * i],
                                          xyz[3 * i + 2] - xyz[3 * i])
                                   / (oh1 * oh2)))
        assert abs(oh1 - 0.957) < 1e-12 and abs(oh2 - 0.957) < 1e-12
        assert abs(ang - 104.5) < 1e-9


def test_random_walk_molecule():
    atoms = geom.random_walk_molecule(40, seed=4)
    xyz = np.array([a[1] for a in atoms])
    d = np.linalg.norm(xyz[:, None] - xyz[None], axis=-1)
    assert d[np.triu_indices(40, 1)].min() >= 1.2 - 1e-12
    z = {'H': 1, 'C': 6, 'N': 7, 'O': 8}
    assert sum(z[a[0]] for a in atoms) % 2 == 0


def test_cart2sph_orthonormal():
    # spherical functions are orthonormal on the unit sphere: check via the
    # overlap of one normalised shell per l
    for l in range(4):
        mol = Mole(atom=[('H', (0, 0, 0))], basis={'H': [[l, [1.1, 1.0]]]}).build()
        s = mol.intor('int1e_ovlp')
        np.testing.assert_allclose(s, np.eye(2 * l + 1), atol=1e-13)
    c = cart2sph(2)
    # d_{xy} is sqrt(15/4pi) xy and d_{x2-y2} is sqrt(15/16pi) (x2 - y2)
    assert abs(c[1, 0] - np.sqrt(15 / (4 * np.pi))) < 1e-14
    assert abs(c[0, 4] - np.sqrt(15 / (16 * np.pi))) < 1e-14


def test_scf_like_density():
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
               basis='standin-cc-pvdz').build()
    s = mol.intor('int1e_ovlp')
    d = geom.scf_like_density(s, nocc=10, seed=1)
    # idempotent in the S metric: (D S / 2)^2 = D S / 2, trace(D S) = 2 nocc
    ds = d @ s / 2
    np.testing.assert_allclose(ds @ ds, ds, atol=1e-10)
    assert abs(np.trace(d @ s) - 20) < 1e-10


def test_one_electron_analytic():
    a = 1.3
    mol = Mole(atom=[('H', (0, 0, 0))], basis={'H': [[0, [a, 1.0]]]}).build()
    assert abs(mol.intor('int1e_kin')[0, 0] - 1.5 * a) < 1e-13
    assert abs(mol.intor('int1e_nuc')[0, 0] + 2 * np.sqrt(2 * a / np.pi)) < 1e-13


def test_conc_mol_keeps_both_molecules():
    """conc_mol (the concatenated basis of the density-fitting integrals):
    the second molecule's shells keep their exponents, coefficients and
    centres after the pointer shift."""
    from byteqc_b200.gto import mole as gmole
    a = Mole(atom=geom.water_cluster(1, box=4.0, seed=1),
             basis='standin-cc-pvdz').build()
    b = Mole(atom=geom.water_cluster(2, box=5.0, seed=2),
             basis='standin-6-31g*').build()
    c = gmole.conc_mol(a, b)
    assert c.nbas == a.nbas + b.nbas and c.natm == a.natm + b.natm
    assert c.nao_nr(cart=True) == a.nao_nr(cart=True) + b.nao_nr(cart=True)
    coords = c.atom_coords()
    for ib in range(b.nbas):
        jb = a.nbas + ib
        assert np.array_equal(c.bas_exp(jb), b.bas_exp(ib))
        assert np.array_equal(c.bas_ctr_coeff(jb), b.bas_ctr_coeff(ib))
        assert c.bas_angular(jb) == b.bas_angular(ib)
        ia = c._bas[jb, gmole.ATOM_OF]
        assert np.array_equal(coords[ia], b.atom_coords()[b._bas[ib, gmole.ATOM_OF]])
    for ib in range(a.nbas):
        assert np.array_equal(c.bas_exp(ib), a.bas_exp(ib))


def test_df_basis_helpers():
    """Class-pair enumeration, the exponent-0 shell and the (l, nprim)
    grouping of the density-fitting basis."""
    from byteqc_b200.cuobc.lib import int3c, int4c
    for gi in range(12):
        for gj in range(gi + 1):
            assert int4c.ind2pair(gi * (gi + 1) // 2 + gj) == (gi, gj)
    fake = int3c.make_fake_mol()
    assert fake.nbas == 1 and fake.bas_angular(0) == 0
    assert fake.bas_exp(0)[0] == 0.0
    assert abs(fake.bas_ctr_coeff(0)[0, 0] * 0.282094791773878143 - 1.) < 1e-15
    mol = Mole(atom=geom.random_walk_molecule(8, seed=3),
               basis='standin-6-31g*').build()
    smol, coeff, counts = int3c.sort_mol(mol)
    assert counts.sum() == smol.nbas
    key = [(int(l), int(n)) for l, n in smol._bas[:, [1, 2]]]
    off = np.append(0, np.cumsum(counts))
    for g in range(len(counts)):
        assert len(set(key[off[g]:off[g + 1]])) == 1
    assert coeff.shape == (smol.nao_nr(cart=True), mol.nao)


def test_bins_and_group_split_match_oracle():
    """The host bin offsets and (l, nprim) group capping of the product path
    against the oracle's restatements of the same reference functions
    (cuobc/scf/hf.py:567-578, 581-606), and the bin invariants the
    class-pair entries rely on (monotone, starting at 0, covering the pairs
    above the cutoff)."""
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    rng = np.random.default_rng(2)
    for n in (1, 7, 300):
        lq = np.sort(np.log(rng.uniform(1e-12, 1., n)))[::-1]
        lq[lq > 0] = 0
        for nbins in (1, 4, 10):
            for cut in (1e-13, 1e-10):
                a = hf._make_s_index_offsets(lq, nbins, cut)
                b = hf_oracle.make_s_index_offsets(lq, nbins, cut)
                assert np.array_equal(a, b)
                assert a[0] == 0 and a[-1] <= n and np.all(np.diff(a) >= 0)
                # every pair above the cutoff falls in a bin
                assert a[-1] >= np.count_nonzero(lq >= np.log(cut))
    uniq = np.array([[0, 3], [1, 1], [2, 1]])
    counts = np.array([40, 25, 7])
    for gs in (8, 30, 100):
        x = hf._split_l_ctr_groups(uniq, counts, gs)
        y = hf_oracle._split_l_ctr_groups(uniq, counts, gs)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
        assert x[1].sum() == counts.sum()


def test_bench_reference_arm_ranks():
    """bench.py --impl reference under several ranks: rank 0 alone runs the
    CPU arm and prints one JSON line; other ranks exit 0 without output.
    The arm maps no engine library."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    base = [sys.executable, os.path.join(root, 'bench.py'), '--impl',
            'reference', '--gpus', '2', '--steps', '1', '--warmup', '0',
            '--ref-sample-s', '0.3', '--no-reference-gpu', '--workload',
            'h2o8-dz']
    env = dict(os.environ, WORLD_SIZE='2')
    p1 = subprocess.run(base, env=dict(env, RANK='1'), capture_output=True,
                        text=True, timeout=300)
    assert p1.returncode == 0 and p1.stdout.strip() == ''
    p0 = subprocess.run(base, env=dict(env, RANK='0'), capture_output=True,
                        text=True, timeout=600)
    assert p0.returncode == 0, p0.stderr[-2000:]
    lines = [x for x in p0.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference' and d['value'] > 0
    assert d['cpu_baseline']['kind'] == 'port'
    assert d['e2e']['h2d_bytes_per_step'] == 0


def test_serving_footprint_bound_covers_the_screened_basis():
    """The server admits a request by a footprint bound computed before
    anything is allocated: it is never below the footprint of the basis the
    Schwarz screen keeps (pair lists from the oracle's restatement of
    _VHFOpt.build), equals it when every shell pair is kept, and grows with
    the molecule."""
    from byteqc_b200.cuobc.scf.serve import _footprint, footprint_bound_bytes
    from oracle import hf_oracle
    prev = 0
    for n in (3, 5, 8):
        mol = Mole(atom=geom.random_walk_molecule(n, seed=60 + n),
                   basis='standin-6-31g*').build()
        opt = hf_oracle.VHFOpt(mol).build(1e-13)
        pm = opt.mol
        nbas = pm._bas.shape[0]
        nps = pm._bas[:, 2].astype(np.int64)
        i, j = opt.bas_pair2shls
        nao = int(pm.ao_loc_nr(cart=True)[-1])
        nao0 = opt.coeff.shape[1]
        exact = _footprint(nbas, nao, nao0, i.size, int((nps[i] * nps[j]).sum()))
        bound = footprint_bound_bytes(mol)
        assert 0 < exact <= bound
        all_pairs = nbas * (nbas + 1) // 2
        all_prim = int((nps.sum() ** 2 + (nps ** 2).sum()) // 2)
        assert _footprint(nbas, nao, nao0, all_pairs, all_prim) == bound
        assert bound > prev
        prev = bound
