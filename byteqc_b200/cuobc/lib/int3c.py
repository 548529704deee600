"""Three- and two-centre Coulomb integrals for density fitting on the GPU,
the counterpart of the reference's ``cuobc/lib/int3c.py`` (``VHFOpt3c``,
``get_int3c``, ``get_int2c``).  As there, the working basis of the molecule,
one s function of exponent 0 (the "fake" shell, so that (ij|P) = (ij|P s0))
and the working basis of the auxiliary molecule are concatenated into one
basis handle; ``jk_fill_int2e`` (libjk.so) then fills (ij|P s0) for a class
pair of the molecule and a class of the auxiliary basis, and (P s0|Q s0) for
two auxiliary classes."""
import ctypes

import numpy as np

from byteqc_b200.cuobc import lib as _lib
from byteqc_b200.gto import mole as gmole
from byteqc_b200.cuobc.lib.int4c import ind2pair

# libcint's common factor of s functions, 1/sqrt(4 pi)
_FAC_S = 0.282094791773878143


def make_fake_mol():
    """One s shell of exponent 0 at the origin whose stored coefficient
    cancels the s common factor, so that its pair data with a shell P are
    those of P alone (cuobc/lib/int3c.py:49-62)."""
    from byteqc_b200.cuobc.scf.hf import basis_seg_contraction
    fake = gmole.Mole(atom=[('He', (0., 0., 0.))],
                      basis={'He': [[0, [100., 2.0]]]}).build()
    fake, _ = basis_seg_contraction(fake)
    fake._env[fake._bas[0, gmole.PTR_COEFF]] = 1.0 / _FAC_S
    fake._env[fake._bas[0, gmole.PTR_EXP]] = 0.0
    return fake


def sort_mol(mol, group_size=None):
    """Working basis of ``mol`` with its shells sorted into (l, nprim)
    groups (cuobc/lib/int3c.py:93-121): returns the sorted molecule, the
    coefficient rows in the sorted AO order, and the group counts."""
    from byteqc_b200.cuobc.scf.hf import (basis_seg_contraction,
                                          _split_l_ctr_groups)
    pmol, coeff = basis_seg_contraction(mol)
    l_ctrs = pmol._bas[:, [gmole.ANG_OF, gmole.NPRIM_OF]]
    uniq, inv, counts = np.unique(l_ctrs, return_inverse=True,
                                  return_counts=True, axis=0)
    inv = np.asarray(inv).ravel()
    if group_size is not None:
        uniq, counts = _split_l_ctr_groups(uniq, counts, group_size)
    sidx = np.argsort(inv, kind='stable')
    ao_loc = pmol.ao_loc_nr(cart=True)
    ao_idx = np.concatenate([np.arange(ao_loc[i], ao_loc[i + 1]) for i in sidx])
    pmol._bas = np.ascontiguousarray(pmol._bas[sidx])
    return pmol, coeff[ao_idx], np.asarray(counts)


class VHFOpt3c:
    """Basis handle of molecule + fake shell + auxiliary basis
    (cuobc/lib/int3c.py:185-264).  After ``build``: ``mol`` / ``auxmol``
    the sorted working bases, ``coeff`` / ``auxcoeff`` their maps to the
    input bases, ``log_qs`` the molecule's class pairs, ``aux_log_qs`` the
    (auxiliary class, fake) pairs, ``l_ctr_offsets`` / ``aux_l_ctr_offsets``
    the group shell offsets of the two bases."""

    def __init__(self, mol, auxmol, intor='int3c2e', prescreen='CVHFnoscreen',
                 qcondname='CVHFsetnr_direct_scf', dmcondname=None, aosym=True):
        self.mol0, self.auxmol0 = mol, auxmol
        self._intor = intor
        self.handle = None

    def build(self, cutoff=1e-13, group_size=None, aux_group_size=None,
              diag_block_with_triu=True, gpus=None):
        from byteqc_b200.cuobc.scf.hf import LMAX_ENGINE
        lib = _lib.load_library()
        smol, coeff, counts = sort_mol(self.mol0, group_size)
        saux, auxcoeff, acounts = sort_mol(self.auxmol0, aux_group_size)
        tot = gmole.conc_mol(smol, gmole.conc_mol(make_fake_mol(), saux))
        lmax = int(tot._bas[:, gmole.ANG_OF].max())
        if lmax > LMAX_ENGINE:
            raise NotImplementedError('shells with l=%d: this engine handles '
                                      'l <= %d' % (lmax, LMAX_ENGINE))
        groups = np.concatenate([counts, [1], acounts]).astype(np.int64)
        offsets = np.append(0, np.cumsum(groups)).astype(np.int32)
        handle = ctypes.c_void_p()
        atm = np.ascontiguousarray(tot._atm, dtype=np.int32)
        bas = np.ascontiguousarray(tot._bas, dtype=np.int32)
        env = np.ascontiguousarray(tot._env, dtype=np.float64)
        _lib.check(lib.jk_basis_create(
            atm.ctypes.data, tot.natm, bas.ctypes.data, tot.nbas,
            env.ctypes.data, env.size, offsets.ctypes.data, len(groups),
            cutoff, int(diag_block_with_triu), ctypes.byref(handle)),
            'jk_basis_create')
        self.handle = handle
        info = np.zeros(7, dtype=np.int32)
        _lib.check(lib.jk_basis_info(handle, info.ctypes.data), 'jk_basis_info')
        nbas, nao, ngroups, ncp, npairs = (int(v) for v in info[:5])
        pair2shls = np.zeros((2, max(npairs, 1)), dtype=np.int32)
        locs = np.zeros(ncp + 1, dtype=np.int32)
        log_q = np.zeros(max(npairs, 1))
        _lib.check(lib.jk_basis_pairs(handle, pair2shls.ctypes.data,
                                      locs.ctypes.data, log_q.ctypes.data,
                                      None), 'jk_basis_pairs')
        g = len(counts)  # molecule groups; the fake shell is group g
        self.log_qs = [log_q[locs[c]:locs[c + 1]] for c in range(g * (g + 1) // 2)]
        self.aux_cp = [(g + 1 + a) * (g + 2 + a) // 2 + g for a in range(len(acounts))]
        self.aux_log_qs = [log_q[locs[c]:locs[c + 1]] for c in self.aux_cp]
        self.mol, self.auxmol, self.tot_mol = smol, saux, tot
        self.coeff, self.auxcoeff = coeff, auxcoeff
        self.l_ctr_offsets = np.append(0, np.cumsum(counts)).astype(np.int32)
        self.aux_l_ctr_offsets = np.append(0, np.cumsum(acounts)).astype(np.int32)
        self.ao_loc = smol.ao_loc_nr(cart=True)
        self.aux_ao_loc = saux.ao_loc_nr(cart=True)
        self.nao_tot = nao
        self.direct_scf_tol = cutoff
        return self

    def clear(self):
        if self.handle is not None and self.handle.value:
            _lib.load_library().jk_basis_destroy(self.handle)
        self.handle = None
        return self

    def __del__(self):
        try:
            self.clear()
        except Exception:
            pass


def _fill(vhfopt, out, strides, ao_offsets, cp_ij, cp_kl, n_ij, n_kl):
    from byteqc_b200.cuobc.scf.hf import _torch
    torch = _torch()
    lib = _lib.load_library()
    bins_ij = np.array([0, n_ij], dtype=np.int32)
    bins_kl = np.array([0, n_kl], dtype=np.int32)
    strides = np.ascontiguousarray(strides, dtype=np.int32)
    ao_offsets = np.ascontiguousarray(ao_offsets, dtype=np.int32)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.jk_fill_int2e(
        vhfopt.handle, ctypes.c_void_p(out.data_ptr()), vhfopt.nao_tot,
        strides.ctypes.data, ao_offsets.ctypes.data, bins_ij.ctypes.data,
        bins_kl.ctypes.data, 1, cp_ij, cp_kl, ctypes.c_void_p(stream)),
        'jk_fill_int2e')


def get_int3c(cp_ij_id, cp_aux_id, vhfopt, bpcache=None, buf=None, order='F'):
    """(ij|P) of a class pair of the molecule and a class of the auxiliary
    basis (cuobc/lib/int3c.py:317-368): the slices of the two working bases
    and the (ni, nj, nk) block, a float64 CUDA tensor laid out column-major
    (order 'F') or row-major (order 'C')."""
    from byteqc_b200.cuobc.scf.hf import _torch
    torch = _torch()
    unao = int(vhfopt.ao_loc[-1])
    cpi, cpj = ind2pair(cp_ij_id)
    offs, aoffs = vhfopt.l_ctr_offsets, vhfopt.aux_l_ctr_offsets
    i0, i1 = (int(x) for x in vhfopt.ao_loc[offs[cpi:cpi + 2]])
    j0, j1 = (int(x) for x in vhfopt.ao_loc[offs[cpj:cpj + 2]])
    k0, k1 = (int(x) for x in vhfopt.aux_ao_loc[aoffs[cp_aux_id:cp_aux_id + 2]])
    ni, nj, nk = i1 - i0, j1 - j0, k1 - k0
    n = ni * nj * nk
    flat = (buf.reshape(-1)[:n] if buf is not None else
            torch.empty(n, dtype=torch.float64, device='cuda'))
    flat.zero_()
    if order == 'C':
        strides = [nj * nk, nk, 1, 1]
        blk = flat.view(ni, nj, nk)
    else:
        strides = [1, ni, ni * nj, 1]
        blk = flat.view(nk, nj, ni).permute(2, 1, 0)
    ao_offsets = [i0, j0, unao + 1 + k0, unao]
    _fill(vhfopt, flat, strides, ao_offsets, cp_ij_id,
          vhfopt.aux_cp[cp_aux_id], len(vhfopt.log_qs[cp_ij_id]),
          len(vhfopt.aux_log_qs[cp_aux_id]))
    return slice(i0, i1), slice(j0, j1), slice(k0, k1), blk


def get_int2c_metric(vhfopt):
    """(P|Q) over the auxiliary working basis, a float64 CUDA tensor."""
    from byteqc_b200.cuobc.scf.hf import _torch
    torch = _torch()
    unao = int(vhfopt.ao_loc[-1])
    unaux = int(vhfopt.aux_ao_loc[-1])
    flat = torch.zeros(unaux * unaux, dtype=torch.float64, device='cuda')
    # element (P, Q) at P + unaux Q (cuobc/lib/int3c.py:267-298)
    strides = [1, unaux, unaux, unaux * unaux]
    ao_offsets = [unao + 1, unao, unao + 1, unao]
    for k, lq_k in enumerate(vhfopt.aux_log_qs):
        for l, lq_l in enumerate(vhfopt.aux_log_qs):
            _fill(vhfopt, flat, strides, ao_offsets, vhfopt.aux_cp[k],
                  vhfopt.aux_cp[l], len(lq_k), len(lq_l))
    return flat.view(unaux, unaux).T


def get_int2c(vhfopt, j2c_eig_always=False, linear_dep_threshold=1e-13):
    """Factor of the inverse Coulomb metric in the input auxiliary basis
    (cuobc/lib/int3c.py:267-314): the Cholesky factor L of
    C^T (P|Q) C = L L^T, or, if that fails or ``j2c_eig_always``, the
    eigenvectors of the kept eigenvalues scaled by 1/sqrt(eigenvalue)."""
    from byteqc_b200.cuobc.scf.hf import _torch
    torch = _torch()
    c = torch.as_tensor(vhfopt.auxcoeff, dtype=torch.float64, device='cuda')
    j2c = c.T @ get_int2c_metric(vhfopt) @ c
    if not j2c_eig_always:
        L, info = torch.linalg.cholesky_ex(j2c)
        if int(info) == 0:
            return L
    e, v = torch.linalg.eigh(j2c)
    mask = e > linear_dep_threshold
    return v[:, mask] * torch.sqrt(1. / e[mask]).reshape(1, -1)


__all__ = ['VHFOpt3c', 'get_int3c', 'get_int2c', 'get_int2c_metric',
           'make_fake_mol', 'sort_mol']
