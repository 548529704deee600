"""GPU parity of the J/K engine against the oracle (the CPU restatement of
the reference's get_jk, oracle/hf_oracle.py + oracle/jk_oracle.c).

Tolerance: 1e-10 max-abs in J/K elements, absolute (the FP64 parity bar).
Mixed precision: the J/K error is held to a small multiple of the FP32
cutoff (observed: about 2e-5 of the cutoff)."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _mol(nw, basis, box, seed=0):
    return Mole(atom=geom.water_cluster(nw, box=box, seed=seed),
                basis=basis).build()


def _rand_dm(n, seed=3, ndm=None):
    rng = np.random.default_rng(seed)
    shape = (n, n) if ndm is None else (ndm, n, n)
    d = rng.random(shape)
    return d + np.swapaxes(d, -1, -2)


def _close(a, b):
    err = abs(np.asarray(a) - np.asarray(b)).max()
    assert err <= TOL, 'max|diff| %.3e (max|ref| %.3g)' % (err, abs(b).max())


@pytest.mark.parametrize('basis', ['standin-cc-pvdz', 'standin-6-31g*',
                                   'standin-def2-tzvp'])
def test_get_jk_vs_oracle(basis):
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _mol(2, basis, 5.0)
    dm = _rand_dm(mol.nao)
    vj, vk = hf.get_jk(mol, dm)
    rj, rk = hf_oracle.get_jk(mol, dm)
    _close(vj, rj)
    _close(vk, rk)


def test_multi_dm_and_flags():
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _mol(3, 'standin-cc-pvdz', 6.0, seed=4)
    dm = _rand_dm(mol.nao, ndm=2)
    opt = hf._VHFOpt(mol).build()
    ropt = hf_oracle.VHFOpt(mol).build()
    rj, rk = hf_oracle.get_jk(mol, dm, vhfopt=ropt)
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
    _close(vj, rj)
    _close(vk, rk)
    vj2, vk2 = hf.get_jk(mol, dm, vhfopt=opt, with_k=False)
    assert vk2 is None
    _close(vj2, rj)
    vj3, vk3 = hf.get_jk(mol, dm, vhfopt=opt, with_j=False)
    assert vj3 is None
    _close(vk3, rk)
    # unscreened, single bin (the reference test's settings, jk.py:7824)
    rj, rk = hf_oracle.get_jk(mol, dm[0], vhfopt=ropt, prescreen=False,
                              nbins=1)
    vj, vk = hf.get_jk(mol, dm[0], vhfopt=opt, prescreen=False, nbins=1)
    _close(vj, rj)
    _close(vk, rk)


def test_pairs_and_qcond_vs_oracle():
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _mol(3, 'standin-def2-tzvp', 6.0, seed=2)
    opt = hf._VHFOpt(mol).build()
    ropt = hf_oracle.VHFOpt(mol).build()
    np.testing.assert_allclose(opt.q_cond, ropt.q_cond, rtol=1e-11,
                               atol=1e-16)
    np.testing.assert_array_equal(opt.bas_pairs_locs, ropt.bas_pairs_locs)
    np.testing.assert_allclose(opt.coeff, ropt.coeff, atol=1e-15)


def test_device_rys_tables_match_host():
    """Device evaluation (every kernel path) against the host evaluation of
    the tables; n = 1 is the Boys function on the device, the table on the
    host, so that case checks the two against each other."""
    import torch
    from byteqc_b200.cuobc import lib as jklib
    lib = jklib.load_library()
    rng = np.random.default_rng(1)
    xs = np.concatenate([[0., 1e-13, 0.5, 0.7499, 0.75, 1.0, 2.0, 41.9, 42.0,
                          97.9, 200., 1e5], rng.uniform(0, 120, 200)])
    dx = torch.as_tensor(xs, device='cuda')
    for n in range(1, 14):
        for mode in (0, 1, 2, 5):
            ds = torch.zeros(len(xs) * n, dtype=torch.float64, device='cuda')
            dw = torch.zeros_like(ds)
            assert lib.jk_rys_roots_device(n, dx.data_ptr(), len(xs),
                                           ds.data_ptr(), dw.data_ptr(), mode,
                                           None) == 0
            s = ds.cpu().numpy().reshape(-1, n)
            w = dw.cpu().numpy().reshape(-1, n)
            for i, x in enumerate(xs):
                hs, hw = np.zeros(n), np.zeros(n)
                lib.jk_rys_roots_host(n, x, hs.ctypes.data, hw.ctypes.data)
                np.testing.assert_allclose(s[i], hs, rtol=1e-14, atol=1e-300)
                np.testing.assert_allclose(w[i], hw, rtol=1e-14, atol=1e-300)


def test_device_rys_fp32_nodes():
    """Single-precision nodes and weights of the FP32 quartets (n <= 3):
    nodes s = t^2 in [0, 1) within 2e-6 absolute, weights within 2e-6 of
    their sum F0(x), against the double host evaluation."""
    import torch
    from byteqc_b200.cuobc import lib as jklib
    lib = jklib.load_library()
    rng = np.random.default_rng(2)
    xs = np.concatenate([[0., 1e-9, 0.5, 0.7499, 0.75, 1.0, 2.0, 41.9, 42.0,
                          47.99, 48.0, 53.99, 54.0, 200., 1e5],
                         rng.uniform(0, 60, 300)])
    dx = torch.as_tensor(xs, device='cuda')
    for n in range(1, 4):
        for mode in (3, 4):  # all roots at once (thread kernels), one at a time (teams)
            ds = torch.zeros(len(xs) * n, dtype=torch.float64, device='cuda')
            dw = torch.zeros_like(ds)
            assert lib.jk_rys_roots_device(n, dx.data_ptr(), len(xs),
                                           ds.data_ptr(), dw.data_ptr(), mode,
                                           None) == 0
            s = ds.cpu().numpy().reshape(-1, n)
            w = dw.cpu().numpy().reshape(-1, n)
            for i, x in enumerate(xs):
                hs, hw = np.zeros(n), np.zeros(n)
                lib.jk_rys_roots_host(n, x, hs.ctypes.data, hw.ctypes.data)
                assert abs(s[i] - hs).max() <= 2e-6, (n, mode, x, s[i], hs)
                assert abs(w[i] - hw).max() <= 2e-6 * hw.sum(), (n, mode, x, w[i], hw)
    # higher orders are not evaluated in single precision
    assert lib.jk_rys_roots_device(4, dx.data_ptr(), 1, ds.data_ptr(),
                                   dw.data_ptr(), 3, None) != 0


def test_mixed_precision_error_bounded():
    """FP32 recursion below the cutoff: J/K stay within a bound that scales
    with the cutoff, and fp32_cutoff=0 reproduces the FP64 engine exactly."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.gto import geom as g
    mol = _mol(4, 'standin-cc-pvdz', 7.0, seed=3)
    s = mol.intor('int1e_ovlp')
    dm = g.scf_like_density(s, nocc=mol.nelectron // 2, seed=1)
    opt = hf._VHFOpt(mol).build()
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
    vj0, vk0 = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=0.)
    assert abs(vj0 - vj).max() < 1e-11 and abs(vk0 - vk).max() < 1e-11
    for cut in (1e-8, 1e-6, 1e-4):
        mj, mk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=cut)
        err = max(abs(mj - vj).max(), abs(mk - vk).max())
        assert err < 1e-3 * cut + 1e-12, (cut, err)


@pytest.mark.parametrize('case', ['h2o12-dz', 'walk30-631gs', 'h2o6-tzvp'])
def test_device_screen_matches_class_pair_loop(case):
    """get_jk (screening on the device, pair-packed J side) against the
    reference's task loop over jk_build_class_pair (host bins, direct
    digestion): the same screened quartets, so the same J/K within the FP64
    bar, at sizes well beyond the oracle's reach; also J only, K only and two
    densities."""
    from byteqc_b200.cuobc.scf import hf
    if case == 'h2o12-dz':
        mol = _mol(12, 'standin-cc-pvdz', 9.0, seed=5)
    elif case == 'h2o6-tzvp':
        mol = _mol(6, 'standin-def2-tzvp', 7.5, seed=6)
    else:
        mol = Mole(atom=geom.random_walk_molecule(30, seed=7),
                   basis='standin-6-31g*').build()
    s = mol.intor('int1e_ovlp')
    dm = geom.scf_like_density(s, nocc=mol.nelectron // 2, seed=2)
    opt = hf._VHFOpt(mol).build()
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt, out='device')
    rj, rk = hf.get_jk_class_pairs(mol, dm, opt)
    _close(vj.cpu().numpy(), rj.cpu().numpy())
    _close(vk.cpu().numpy(), rk.cpu().numpy())
    j1, k1 = hf.get_jk(mol, dm, vhfopt=opt, with_k=False, out='device')
    assert k1 is None
    _close(j1.cpu().numpy(), rj.cpu().numpy())
    j2, k2 = hf.get_jk(mol, dm, vhfopt=opt, with_j=False, out='device')
    assert j2 is None
    _close(k2.cpu().numpy(), rk.cpu().numpy())
    dm2 = np.stack([dm, 0.5 * dm])
    vj2, vk2 = hf.get_jk(mol, dm2, vhfopt=opt, out='device')
    _close(vj2[1].cpu().numpy(), 0.5 * rj.cpu().numpy())
    _close(vk2[1].cpu().numpy(), 0.5 * rk.cpu().numpy())


def test_get_jk_vs_oracle_larger():
    """A five-water cluster (long kl rows, many class quartets) against the
    oracle."""
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _mol(5, 'standin-cc-pvdz', 6.5, seed=8)
    dm = _rand_dm(mol.nao, seed=9)
    vj, vk = hf.get_jk(mol, dm)
    rj, rk = hf_oracle.get_jk(mol, dm)
    _close(vj, rj)
    _close(vk, rk)


def test_get_jk_water8_dz_vs_oracle():
    """The (H2O)8 / cc-pVDZ workload (9 A cube, seed 0, SCF-like density) at
    full size against the oracle, in FP64 and in the mixed mode (its error
    bounded by the cutoff)."""
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _mol(8, 'standin-cc-pvdz', 9.0, seed=0)
    dm = geom.scf_like_density(mol.intor('int1e_ovlp'),
                               nocc=mol.nelectron // 2, seed=1)
    opt = hf._VHFOpt(mol).build()
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
    rj, rk = hf_oracle.get_jk(mol, dm)
    _close(vj, rj)
    _close(vk, rk)
    mj, mk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=1e-6)
    assert max(abs(mj - rj).max(), abs(mk - rk).max()) < 1e-9


@pytest.mark.parametrize('case', ['h2o-dz', 'h2o2-tzvp', 'walk6-631gs'])
def test_get_jk_vs_golden(case):
    """The engine against the committed golden J/K (tests/golden)."""
    import os
    from byteqc_b200.cuobc.scf import hf
    from tests.golden.make_golden import case_inputs
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'golden_jk.npz'))
    mol, dm = case_inputs(case)
    vj, vk = hf.get_jk(mol, dm)
    _close(vj, g[case + '/vj'])
    _close(vk, g[case + '/vk'])


def _high_l_mol(nw, seed=1):
    """Water molecules in the cc-pVDZ stand-in plus g and h shells (an
    uncontracted g and h and a two-primitive g on O, a g on H): every class
    above f runs the generic kernel, next to the templated ones."""
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]], [4, [3.0, 0.6], [0.7, 0.5]]],
             'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
           for s in ('O', 'H')}
    return Mole(atom=geom.water_cluster(nw, box=5.0, seed=seed),
                basis=bas).build()


@pytest.mark.parametrize('nw', [1, 2])
def test_get_jk_g_h_shells_vs_oracle(nw):
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol = _high_l_mol(nw)
    assert int(mol._bas[:, 1].max()) == 5
    opt = hf._VHFOpt(mol).build()
    ropt = hf_oracle.VHFOpt(mol).build()
    np.testing.assert_allclose(opt.q_cond, ropt.q_cond, rtol=1e-11,
                               atol=1e-16)
    dm = _rand_dm(mol.nao, ndm=2)
    rj, rk = hf_oracle.get_jk(mol, dm, vhfopt=ropt)
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
    _close(vj, rj)
    _close(vk, rk)
    # the reference's class-pair task loop reaches the same kernels
    cj, ck = hf.get_jk_class_pairs(mol, dm, opt)
    _close(cj.cpu().numpy(), rj)
    _close(ck.cpu().numpy(), rk)
    # mixed mode: the generic classes stay in FP64 in both parts
    mj, mk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=1e-6)
    assert max(abs(mj - vj).max(), abs(mk - vk).max()) < 1e-9


@pytest.mark.parametrize('name', ['h2o32-tzvp', 'h2o64-dz'])
def test_full_size_workloads_vs_oracle(name):
    """The (H2O)32 / def2-TZVP and (H2O)64 / cc-pVDZ stand-in workloads at
    full size, FP64, against a full oracle build on all host cores (about a
    minute each)."""
    import os
    import sys
    import time
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from byteqc_b200.cuobc.scf import hf
    from oracle import hf_oracle
    mol, dm = bench.make_workload(name)
    vj, vk = hf.get_jk(mol, dm)
    t = time.perf_counter()
    rj, rk = hf_oracle.get_jk(mol, dm)
    print('%s: oracle full build %.1f s' % (name, time.perf_counter() - t))
    _close(vj, rj)
    _close(vk, rk)


def _i_shell_mol(nw, seed=2):
    """Water molecules in the 6-31G* stand-in plus i shells (an uncontracted
    and a two-primitive i on O, an i on H) and a g on O: classes with an i
    shell run the generic kernel at its l = 6 sizes (13 Rys roots at
    (ii|ii)); the reference sends these quartets to PySCF on the CPU
    (cuobc/scf/hf.py:185-218)."""
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[6, [1.3, 1.0]], [6, [2.5, 0.7], [0.6, 0.5]],
                   [4, [1.0, 1.0]]],
             'H': [[6, [0.9, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-6-31g*', s)) + extra[s]
           for s in ('O', 'H')}
    return Mole(atom=geom.water_cluster(nw, box=5.0, seed=seed),
                basis=bas).build()


@pytest.mark.parametrize('nw', [1, 2])
def test_get_jk_i_shells_vs_oracle(nw):
    """i shells against the oracle: J/K at 1e-10 absolute for an SCF-like
    density (and half of it); the Schwarz diagonal within 1e-9 of its largest
    value (both codes evaluate (ii|ii) of distant i shells by the Rys
    recursion in double, whose cancellation at l = 6 leaves about 5e-9 of a
    small value; the oracle matches Obara-Saika to 1e-15 on (is|is))."""
    from byteqc_b200.cuobc.scf import hf
    from oracle import gto_oracle, hf_oracle
    mol = _i_shell_mol(nw)
    assert int(mol._bas[:, 1].max()) == 6
    opt = hf._VHFOpt(mol).build()
    ropt = hf_oracle.VHFOpt(mol).build()
    qmax = abs(ropt.q_cond).max()
    np.testing.assert_allclose(opt.q_cond, ropt.q_cond, rtol=1e-11,
                               atol=1e-9 * qmax)
    np.testing.assert_array_equal(opt.bas_pairs_locs, ropt.bas_pairs_locs)
    d = geom.scf_like_density(gto_oracle.overlap(mol),
                              nocc=mol.nelectron // 2, seed=4)
    dm = np.stack([d, 0.5 * d])
    rj, rk = hf_oracle.get_jk(mol, dm, vhfopt=ropt)
    vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
    _close(vj, rj)
    _close(vk, rk)
    cj, ck = hf.get_jk_class_pairs(mol, dm, opt)
    _close(cj.cpu().numpy(), rj)
    _close(ck.cpu().numpy(), rk)


def test_batch_and_fill_i_shells():
    """Batched builds with i shells match single builds, and the ERI-tensor
    fill of classes with an i shell matches the oracle's shell quartets."""
    from byteqc_b200.cuobc.lib import int4c
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    import oracle
    mols = [_i_shell_mol(1, seed=s) for s in (3, 4)]
    dms = [_rand_dm(m.nao, seed=5 + i) for i, m in enumerate(mols)]
    batch = JKBatch(mols)
    res = batch.get_jk(dms)
    for m, (mol, dm, opt) in enumerate(zip(mols, dms, batch.opts)):
        vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
        _close(res[m][0], vj)
        _close(res[m][1], vk)
    batch.close()
    mol = mols[0]
    opt = hf._VHFOpt(mol).build(diag_block_with_triu=True)
    pm = opt.mol
    ls = opt.uniq_l_ctr[:, 0]
    ngr = len(ls)
    ao_loc = pm.ao_loc_nr(cart=True)
    offs = opt.l_ctr_offsets
    cp_idx, cp_jdx = np.tril_indices(ngr)
    tested = 0
    for cp_ij in range(len(opt.log_qs)):
        for cp_kl in range(cp_ij + 1):
            g = (cp_idx[cp_ij], cp_jdx[cp_ij], cp_idx[cp_kl], cp_jdx[cp_kl])
            if 6 not in [int(ls[x]) for x in g] or tested >= 6:
                continue
            si, sj, sk, sl, blk = int4c.get_int4c_slice(cp_ij, cp_kl, opt)
            blk = blk.cpu().numpy()
            # every quartet of the first shell of each group (pair lists
            # keep them: all survive the Schwarz cutoff here)
            shells = [int(offs[x]) for x in g]
            ref = oracle.eri_shells(pm, *shells)
            a0 = [int(ao_loc[s]) - int(ao_loc[offs[x]]) for s, x in zip(shells, g)]
            n = ref.shape
            got = blk[a0[0]:a0[0] + n[0], a0[1]:a0[1] + n[1],
                      a0[2]:a0[2] + n[2], a0[3]:a0[3] + n[3]]
            assert abs(got - ref).max() <= 1e-10, (g, abs(got - ref).max())
            tested += 1
    assert tested > 0


def test_sharded_get_jk_two_ranks():
    """get_jk(..., group=...) split over two ranks (gloo, both on this GPU:
    their kernels never wait on each other, the all-reduce goes through the
    host) equals the unsharded build on every rank, FP64, two densities,
    mixed, J only."""
    import os
    import socket
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with socket.socket() as so:
        so.bind(('127.0.0.1', 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1',
           '--nproc-per-node=2', '--master-addr=127.0.0.1',
           '--master-port=%d' % port,
           os.path.join(root, 'tests', 'shard_worker.py')]
    p = subprocess.run(cmd, cwd=root, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, (p.stdout + p.stderr)[-3000:]
    assert 'rank 0 ok' in p.stdout and 'rank 1 ok' in p.stdout
