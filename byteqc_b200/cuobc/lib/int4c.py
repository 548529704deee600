"""Dense two-electron integral tensor of the working basis on the GPU, the
counterpart of the reference's ``cuobc/lib/int4c.py`` (``get_int4c``,
``get_int4c_slice``): per class pair the screened shell quartets are filled
by ``jk_fill_int2e`` (libjk.so) into a block, and the eight index
permutations of each block fill the tensor.  The tensor is in the working
basis of the ``_VHFOpt`` (decontracted, Cartesian, shells sorted into
(l, nprim) groups), as the reference's; build the ``_VHFOpt`` with
``diag_block_with_triu=True`` (the default here, as in the reference's
int4c test) so that the diagonal shell pairs carry their full value."""
import ctypes

import numpy as np

from byteqc_b200.cuobc import lib as _lib


def ind2pair(ind):
    """Class-pair index -> (group i, group j), j <= i, of the lower-triangle
    enumeration (cuobc/lib/int3c.py:371-373)."""
    a = int(np.sqrt(2 * ind + 0.25) - 0.5)
    return a, ind - a * (a + 1) // 2


def _opt(mol, blksize=None, vhfopt=None):
    from byteqc_b200.cuobc.scf.hf import _VHFOpt
    if vhfopt is None:
        vhfopt = _VHFOpt(mol, 'int2e').build(group_size=blksize,
                                             diag_block_with_triu=True)
    return vhfopt


def get_int4c_slice(cp_ij_id, cp_kl_id, vhfopt, buf=None, nbins=1):
    """Integrals of one class pair (cuobc/lib/int4c.py:73-104): returns the
    four AO slices of the working basis and the (ni, nj, nk, nl) block (a
    float64 CUDA tensor; ``buf``, if given, a CUDA tensor it is carved
    from)."""
    from byteqc_b200.cuobc.scf.hf import _make_s_index_offsets, _torch
    torch = _torch()
    lib = _lib.load_library()
    cpi, cpj = ind2pair(cp_ij_id)
    cpk, cpl = ind2pair(cp_kl_id)
    ao_loc = vhfopt.mol.ao_loc_nr(cart=True)
    offs = vhfopt.l_ctr_offsets
    i0, i1 = ao_loc[offs[cpi]], ao_loc[offs[cpi + 1]]
    j0, j1 = ao_loc[offs[cpj]], ao_loc[offs[cpj + 1]]
    k0, k1 = ao_loc[offs[cpk]], ao_loc[offs[cpk + 1]]
    l0, l1 = ao_loc[offs[cpl]], ao_loc[offs[cpl + 1]]
    ni, nj, nk, nl = i1 - i0, j1 - j0, k1 - k0, l1 - l0
    n = ni * nj * nk * nl
    if buf is not None:
        blk = buf.reshape(-1)[:n].view(ni, nj, nk, nl)
        blk.zero_()
    else:
        blk = torch.zeros((ni, nj, nk, nl), dtype=torch.float64, device='cuda')
    ao_offsets = np.array([i0, j0, k0, l0], dtype=np.int32)
    strides = np.array([nj * nk * nl, nk * nl, nl, 1], dtype=np.int32)
    bins_ij = _make_s_index_offsets(vhfopt.log_qs[cp_ij_id], nbins,
                                    vhfopt.direct_scf_tol)
    bins_kl = _make_s_index_offsets(vhfopt.log_qs[cp_kl_id], nbins,
                                    vhfopt.direct_scf_tol)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.jk_fill_int2e(
        vhfopt.handle, ctypes.c_void_p(blk.data_ptr()), vhfopt.nao,
        strides.ctypes.data, ao_offsets.ctypes.data, bins_ij.ctypes.data,
        bins_kl.ctypes.data, nbins, cp_ij_id, cp_kl_id,
        ctypes.c_void_p(stream)), 'jk_fill_int2e')
    return (slice(i0, i1), slice(j0, j1), slice(k0, k1), slice(l0, l1), blk)


def get_int4c(mol, blksize=None, vhfopt=None, batch=1, buf_size=0, nbins=1):
    """The (nao, nao, nao, nao) tensor (ij|kl) of the working basis as a
    float64 CUDA tensor (cuobc/lib/int4c.py:44-70).  ``batch`` (the
    reference's multi-GPU task batching) and ``buf_size`` (a staging-buffer
    size of its basis set-up) are accepted for call compatibility; one GPU
    per process fills the whole tensor."""
    from byteqc_b200.cuobc.scf.hf import _torch
    torch = _torch()
    vhfopt = _opt(mol, blksize, vhfopt)
    nao = vhfopt.nao
    out = torch.zeros((nao, nao, nao, nao), dtype=torch.float64, device='cuda')
    for cp_ij, cp_kl in zip(*np.tril_indices(len(vhfopt.log_qs))):
        si, sj, sk, sl, b = get_int4c_slice(int(cp_ij), int(cp_kl), vhfopt,
                                            nbins=nbins)
        out[si, sj, sk, sl] = b
        out[sj, si, sk, sl] = b.permute(1, 0, 2, 3)
        out[si, sj, sl, sk] = b.permute(0, 1, 3, 2)
        out[sj, si, sl, sk] = b.permute(1, 0, 3, 2)
        out[sk, sl, si, sj] = b.permute(2, 3, 0, 1)
        out[sk, sl, sj, si] = b.permute(2, 3, 1, 0)
        out[sl, sk, si, sj] = b.permute(3, 2, 0, 1)
        out[sl, sk, sj, si] = b.permute(3, 2, 1, 0)
    return out


__all__ = ['get_int4c', 'get_int4c_slice', 'ind2pair']
