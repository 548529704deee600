"""Batched J/K over molecules of uneven size: identical (to rounding) to
building each molecule alone, in FP64, in mixed precision and when replayed
from a captured CUDA graph."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu


def _mols():
    out = []
    for i, n in enumerate((3, 7, 12, 5)):
        atoms = geom.random_walk_molecule(n, seed=40 + i)
        out.append(Mole(atom=atoms, basis='standin-6-31g*').build())
    return out


def _dms(mols, seed=0):
    rng = np.random.default_rng(seed)
    res = []
    for m in mols:
        d = rng.random((m.nao, m.nao))
        res.append(d + d.T)
    return res


def test_batch_matches_single_molecule_builds():
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols = _mols()
    dms = _dms(mols)
    batch = JKBatch(mols)
    res = batch.get_jk(dms)
    for m, (mol, dm, opt) in enumerate(zip(mols, dms, batch.opts)):
        vj, vk = hf.get_jk(mol, dm, vhfopt=opt)
        scale = max(1.0, abs(vj).max())
        assert abs(res[m][0] - vj).max() <= 1e-10
        assert abs(res[m][1] - vk).max() <= 1e-10
    # mixed precision in the batch equals mixed precision alone
    mres = batch.get_jk(dms, fp32_cutoff=1e-6)
    for m, (mol, dm, opt) in enumerate(zip(mols, dms, batch.opts)):
        vj, vk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=1e-6)
        assert abs(mres[m][0] - vj).max() <= 1e-9
        assert abs(mres[m][1] - vk).max() <= 1e-9


def test_batch_graph_replay():
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols = _mols()
    batch = JKBatch(mols)
    d0 = _dms(mols, seed=1)
    d1 = _dms(mols, seed=2)
    ref1 = batch.get_jk(d1)
    batch.capture(d0)
    for _ in range(2):
        got = batch.replay(d1)
    for (aj, ak), (bj, bk) in zip(ref1, got):
        assert abs(aj - bj).max() <= 1e-10
        assert abs(ak - bk).max() <= 1e-10


def test_batch_identical_molecules_keep_their_own_j():
    """Copies of one molecule in a batch: their segments of a class carry the
    same shell indices, so a warp that straddles two of them must not merge
    their J contributions (each copy has its own density)."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    atoms = geom.water_cluster(1, box=4.0, seed=3)
    mols = [Mole(atom=atoms, basis='standin-cc-pvdz').build() for _ in range(6)]
    dms = _dms(mols, seed=5)
    batch = JKBatch(mols)
    for cut in (None, 1e-6):
        res = batch.get_jk(dms, fp32_cutoff=cut)
        for m, (mol, dm, opt) in enumerate(zip(mols, dms, batch.opts)):
            vj, vk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=cut)
            scale = max(1.0, abs(vj).max())
            assert abs(res[m][0] - vj).max() <= 1e-10, (cut, m)
            assert abs(res[m][1] - vk).max() <= 1e-10, (cut, m)


def test_batch_g_h_shells():
    """Batched builds of molecules with g and h shells (the generic kernel's
    segment-table launch) match the single-molecule builds."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]]], 'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
           for s in ('O', 'H')}
    mols = [Mole(atom=geom.water_cluster(n, box=5.0, seed=s), basis=bas).build()
            for n, s in ((1, 1), (2, 2), (1, 3))]
    dms = _dms(mols, seed=5)
    batch = JKBatch(mols)
    for cut in (0., 1e-6):
        res = batch.get_jk(dms, fp32_cutoff=cut)
        for m, (mol, dm, opt) in enumerate(zip(mols, dms, batch.opts)):
            vj, vk = hf.get_jk(mol, dm, vhfopt=opt, fp32_cutoff=cut)
            scale = max(1.0, abs(vj).max())
            assert abs(res[m][0] - vj).max() <= 1e-10
            assert abs(res[m][1] - vk).max() <= 1e-10


def test_batch_molecules_vs_oracle():
    """The first eight molecules of the 256-molecule batched workload
    (random walks of 3-60 atoms, C:N:O:H = 3:1:1:5, 6-31G* stand-in, seed 4,
    SCF-like densities) built in one batch, each against the oracle at
    1e-10 absolute, FP64."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from byteqc_b200.cuobc.scf.batch import JKBatch
    from oracle import hf_oracle
    mols, dms = bench.batch_workload(8)
    batch = JKBatch(mols)
    res = batch.get_jk(dms)
    for m, (mol, dm) in enumerate(zip(mols, dms)):
        rj, rk = hf_oracle.get_jk(mol, dm)
        assert abs(res[m][0] - rj).max() <= 1e-10, m
        assert abs(res[m][1] - rk).max() <= 1e-10, m
    batch.close()


def test_batch_tune_keeps_results_and_cache(tmp_path):
    """The autotuner picks a launch shape per class launch (static chunks or
    a persistent grid with a device work counter); the batched J/K are the
    same before and after tuning, in FP64 and in the mixed mode, and a second
    tuning from the cache file times nothing again."""
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols = _mols()
    dms = _dms(mols, seed=9)
    batch = JKBatch(mols)
    ref = batch.get_jk(dms)
    ref32 = batch.get_jk(dms, fp32_cutoff=1e-6)
    cache = str(tmp_path / 'tune.txt')
    info = batch.tune(dms, fp32_cutoff=1e-6, cache=cache)
    assert info and all(k['fp64']['ms'] is not None for k in info)
    assert all(k['fp32']['ms'] is not None for k in info)
    got = batch.get_jk(dms)
    got32 = batch.get_jk(dms, fp32_cutoff=1e-6)
    for (aj, ak), (bj, bk) in zip(ref, got):
        assert abs(aj - bj).max() <= 1e-10
        assert abs(ak - bk).max() <= 1e-10
    for (aj, ak), (bj, bk) in zip(ref32, got32):
        assert abs(aj - bj).max() <= 1e-10
        assert abs(ak - bk).max() <= 1e-10
    # every persistent shape also gives the same result in a captured graph
    batch.capture(dms)
    rep = batch.replay(dms)
    for (aj, ak), (bj, bk) in zip(ref, rep):
        assert abs(aj - bj).max() <= 1e-10
        assert abs(ak - bk).max() <= 1e-10
    lines = open(cache).read().splitlines()
    assert len(lines) > 1
    b2 = JKBatch(mols, vhfopts=batch.opts)
    info2 = b2.tune(dms, fp32_cutoff=1e-6, cache=cache)
    shapes = {(k['class'], k['np_ij'], k['np_kl']): (k['fp64']['grab'],
              k['fp64']['grid_mul']) for k in info}
    for k in info2:
        assert shapes[(k['class'], k['np_ij'], k['np_kl'])] == (
            k['fp64']['grab'], k['fp64']['grid_mul'])
    b2.close()
    batch.close()


def test_batch_persistent_shapes_match_static():
    """Every persistent launch shape gives the static result: the batch's
    class launches forced to each candidate grab size (through a cache file
    written by hand) on molecules of uneven size."""
    import os
    import tempfile
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols = _mols()
    dms = _dms(mols, seed=10)
    batch = JKBatch(mols)
    ref = batch.get_jk(dms)
    info = batch.info()
    with tempfile.TemporaryDirectory() as d:
        for grab, gm in ((1, 1), (2, 2), (64, 1), (1024, 2)):
            path = os.path.join(d, 'c%d_%d.txt' % (grab, gm))
            with open(path, 'w') as f:
                for k in info:
                    lg = max(0, int(k['tasks']).bit_length() - 1)
                    f.write('%d %d %d 0 %d %d %d 1.0\n' % (
                        k['class'], k['np_ij'], k['np_kl'], lg, grab, gm))
            b = JKBatch(mols, vhfopts=batch.opts)
            b.tune(dms, cache=path)
            assert all(k['fp64']['grab'] == grab for k in b.info())
            got = b.get_jk(dms)
            for (aj, ak), (bj, bk) in zip(ref, got):
                assert abs(aj - bj).max() <= 1e-10, (grab, gm)
                assert abs(ak - bk).max() <= 1e-10, (grab, gm)
            b.close()
    batch.close()


def test_batch_solo_class_quartets():
    """Class quartets above the solo threshold run as their own launches
    (the single-molecule kernels), the rest merged: every split gives the
    single-molecule result, in FP64, in mixed precision and from a graph."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols = _mols()
    dms = _dms(mols, seed=20)
    base = JKBatch(mols, solo_tasks=0)
    assert base.nsolo == 0
    ref = [hf.get_jk(m, d, vhfopt=o) for m, d, o in zip(mols, dms, base.opts)]
    ref32 = [hf.get_jk(m, d, vhfopt=o, fp32_cutoff=1e-6)
             for m, d, o in zip(mols, dms, base.opts)]
    nsolos = []
    for solo in (1, 64, 4096):
        b = JKBatch(mols, vhfopts=base.opts, solo_tasks=solo)
        nsolos.append(b.nsolo)
        if solo == 1:
            assert b.info() == []      # everything on its own
        for cut, want, tol in ((None, ref, 1e-10), (1e-6, ref32, 1e-9)):
            got = b.get_jk(dms, fp32_cutoff=cut)
            for (aj, ak), (bj, bk) in zip(want, got):
                assert abs(aj - bj).max() <= tol, (solo, cut)
                assert abs(ak - bk).max() <= tol, (solo, cut)
        b.capture(dms, fp32_cutoff=1e-6)
        got = b.replay(dms)
        for (aj, ak), (bj, bk) in zip(ref32, got):
            assert abs(aj - bj).max() <= 1e-9
            assert abs(ak - bk).max() <= 1e-9
        b.close()
    assert nsolos[0] >= nsolos[1] >= nsolos[2] and nsolos[0] > nsolos[2]
    base.close()
