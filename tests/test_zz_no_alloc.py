"""jk_build_class_pair_noalloc, the entry point for callers that cannot
allocate device memory while running (their GPU memory is owned by their own
pool), must give the same J/K as jk_build_class_pair, whose scratch buffers
the library allocates.  Checked on every class pair of a small molecule, two
calls in a row (the second call reuses the fixed scratch array the first one
left filled).  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry():
    import torch
    from byteqc_b200.cuobc import lib as jklib
    from byteqc_b200.cuobc.scf import hf
    lib = jklib.load_library()
    mol = Mole(atom=geom.water_cluster(3, box=6.0, seed=6),
               basis='standin-def2-tzvp').build()
    opt = hf._VHFOpt(mol).build()
    nao = opt.nao
    rng = np.random.default_rng(11)
    d = rng.random((2, nao, nao))
    d = d + d.transpose(0, 2, 1)
    dd = torch.as_tensor(d, device='cuda').contiguous()
    locs = opt.bas_pairs_locs
    ncp = len(locs) - 1
    for rep in range(2):
        for cij in range(ncp):
            for ckl in range(cij + 1):
                nij, nkl = locs[cij + 1] - locs[cij], locs[ckl + 1] - locs[ckl]
                if nij == 0 or nkl == 0:
                    continue
                nb = 4
                lq_ij, lq_kl = opt.log_qs[cij], opt.log_qs[ckl]
                bij = hf._make_s_index_offsets(lq_ij, nb, 1e-11)
                bkl = hf._make_s_index_offsets(lq_kl, nb, 1e-11)
                out = []
                for fn in (lib.jk_build_class_pair,
                           lib.jk_build_class_pair_noalloc):
                    vj = torch.zeros_like(dd)
                    vk = torch.zeros_like(dd)
                    rc = fn(opt.handle, vj.data_ptr(), vk.data_ptr(),
                            dd.data_ptr(), nao, 2, bij.ctypes.data,
                            bkl.ctypes.data, nb, cij, ckl, None)
                    assert rc == 0, lib.jk_last_error()
                    torch.cuda.synchronize()
                    out.append((vj.cpu().numpy(), vk.cpu().numpy()))
                (aj, ak), (bj, bk) = out
                scale = max(1.0, abs(aj).max(), abs(ak).max())
                assert abs(aj - bj).max() <= 1e-10
                assert abs(ak - bk).max() <= 1e-10


def test_noalloc_rejects_oversized_requests():
    from byteqc_b200.cuobc import lib as jklib
    from byteqc_b200.cuobc.scf import hf
    lib = jklib.load_library()
    mol = Mole(atom=geom.water_cluster(1, box=3.0, seed=0),
               basis='standin-cc-pvdz').build()
    opt = hf._VHFOpt(mol).build()
    bins = np.zeros(2000, dtype=np.int32)
    rc = lib.jk_build_class_pair_noalloc(opt.handle, None, None, ctypes.c_void_p(8),
                                         opt.nao, 1, bins.ctypes.data,
                                         bins.ctypes.data, 1500, 0, 0, None)
    assert rc == 3
    assert b'1024' in lib.jk_last_error()


def test_noalloc_large_ij_class_allocates_nothing():
    """An ij class of more than 1024 shell pairs (several blocks of the
    row-offset scan, so the carry between them runs): (H2O)8 / cc-pVDZ, its
    largest class against itself and against the largest other class, two
    calls in a row.  A first call with vj = vk = NULL does the per-device
    set-up; afterwards the device's free memory does not change across
    calls."""
    import torch
    from byteqc_b200.cuobc import lib as jklib
    from byteqc_b200.cuobc.scf import hf
    lib = jklib.load_library()
    mol = Mole(atom=geom.water_cluster(8, box=9.0, seed=0),
               basis='standin-cc-pvdz').build()
    opt = hf._VHFOpt(mol).build()
    nao = opt.nao
    locs = opt.bas_pairs_locs
    sizes = locs[1:] - locs[:-1]
    order = np.argsort(sizes)[::-1]
    big = int(order[0])
    assert sizes[big] > 1024
    other = int(order[1])
    rng = np.random.default_rng(12)
    d = rng.random((nao, nao))
    dd = torch.as_tensor(d + d.T, device='cuda').contiguous()
    nb = 10
    assert lib.jk_build_class_pair_noalloc(opt.handle, None, None,
                                           dd.data_ptr(), nao, 1,
                                           np.zeros(nb + 1, np.int32).ctypes.data,
                                           np.zeros(nb + 1, np.int32).ctypes.data,
                                           nb, big, big, None) == 0
    torch.cuda.synchronize()
    for cij, ckl in ((big, big), (max(big, other), min(big, other))):
        bij = hf._make_s_index_offsets(opt.log_qs[cij], nb, 1e-13)
        bkl = hf._make_s_index_offsets(opt.log_qs[ckl], nb, 1e-13)
        ref_j = torch.zeros_like(dd)
        ref_k = torch.zeros_like(dd)
        assert lib.jk_build_class_pair(opt.handle, ref_j.data_ptr(),
                                       ref_k.data_ptr(), dd.data_ptr(), nao, 1,
                                       bij.ctypes.data, bkl.ctypes.data, nb,
                                       cij, ckl, None) == 0
        vj = torch.zeros_like(dd)
        vk = torch.zeros_like(dd)
        torch.cuda.synchronize()
        for rep in range(2):
            vj.zero_()
            vk.zero_()
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = lib.jk_build_class_pair_noalloc(
                opt.handle, vj.data_ptr(), vk.data_ptr(), dd.data_ptr(), nao,
                1, bij.ctypes.data, bkl.ctypes.data, nb, cij, ckl, None)
            assert rc == 0, lib.jk_last_error()
            assert torch.cuda.mem_get_info()[0] == free0
            scale = max(1.0, ref_j.abs().max().item(), ref_k.abs().max().item())
            assert (vj - ref_j).abs().max().item() <= 1e-10
            assert (vk - ref_k).abs().max().item() <= 1e-10
