"""ORACLE (test infrastructure only): restatement of the reference's J/K host
orchestration, ByteQC ``cuobc/scf/hf.py``, driving the C oracle.

Follows, step by step:
  - ``basis_seg_contraction`` (hf.py:481-564): split generally contracted
    shells into primitive shells, Cartesian working basis, ``coeff`` maps the
    working basis to the contracted spherical (or Cartesian) basis;
  - ``_VHFOpt.build`` (hf.py:288-408): shells sorted by unique (l, nprim),
    optional group splitting (hf.py:581-606), Schwarz-sorted shell-pair
    lists per lower-triangular group pair, kept if q > cutoff, the upper
    triangle dropped in diagonal blocks, log(q) clipped at 0, diagonal pairs
    scaled by 0.5;
  - ``get_jk`` (hf.py:53-227): dms = C D C^T, per-group absmax condensation
    of dms, class-pair tasks decoded from the lower triangle, class-level
    density screen, log-Schwarz bins (``_make_s_index_offsets``,
    hf.py:567-578), the per-task kernel call, then J = 2 C^T (V + V^T) C and
    K = C^T (V + V^T) C.
The Schwarz matrix is the oracle's own (C, same definition as PySCF's
CVHFsetnr_direct_scf); the radial normalisation and the Cartesian-to-spherical
transform are the oracle's own too (``gto_oracle``), so they do not share
code with the product's ``byteqc_b200.gto``.
"""
import ctypes

import numpy as np

import oracle
from byteqc_b200.gto import mole as gmole  # libcint slot indices only
from oracle import gto_oracle

LMAX_ON_GPU = 5  # the reference's GPU limit, used by the group split
LMAX_ORACLE = 6


def basis_seg_contraction(mol):
    bas_templates = {}
    _bas = []
    _env = mol._env.copy()
    contr_coeff = []
    for ia, (ib0, ib1) in enumerate(mol.aoslice_by_atom()[:, :2]):
        key = tuple(mol._bas[ib0:ib1, gmole.PTR_EXP])
        if key in bas_templates:
            bas_of_ia, coeff = bas_templates[key]
            bas_of_ia = bas_of_ia.copy()
            bas_of_ia[:, gmole.ATOM_OF] = ia
        else:
            coeff = []
            bas_of_ia = []
            for shell in mol._bas[ib0:ib1]:
                l = shell[gmole.ANG_OF]
                nf = (l + 1) * (l + 2) // 2
                nctr = shell[gmole.NCTR_OF]
                if nctr == 1:
                    bas_of_ia.append(shell[None])
                    coeff.append(np.eye(nf))
                    continue
                nprim = shell[gmole.NPRIM_OF]
                pcoeff = shell[gmole.PTR_COEFF]
                pexp = shell[gmole.PTR_EXP]
                exps = _env[pexp:pexp + nprim]
                norm = gto_oracle.gto_norm(l, exps)
                c = _env[pcoeff:pcoeff + nprim * nctr].reshape(nctr, nprim)
                c = np.einsum('ip,p,ef->iepf', c, 1 / norm, np.eye(nf))
                coeff.append(c.reshape(nf * nctr, nf * nprim).T)
                _env[pcoeff:pcoeff + nprim] = norm
                bs = np.repeat(shell[None], nprim, axis=0)
                bs[:, gmole.NPRIM_OF] = 1
                bs[:, gmole.NCTR_OF] = 1
                bs[:, gmole.PTR_EXP] = np.arange(pexp, pexp + nprim)
                bs[:, gmole.PTR_COEFF] = np.arange(pcoeff, pcoeff + nprim)
                bas_of_ia.append(bs)
            bas_of_ia = np.vstack(bas_of_ia)
            bas_templates[key] = (bas_of_ia, coeff)
        _bas.append(bas_of_ia)
        contr_coeff.extend(coeff)
    pmol = mol.copy()
    pmol.cart = True
    pmol._bas = np.asarray(np.vstack(_bas), dtype=np.int32)
    pmol._env = _env
    if mol.cart:
        n0 = sum(c.shape[0] for c in contr_coeff)
        n1 = sum(c.shape[1] for c in contr_coeff)
        out = np.zeros((n0, n1))
        r = cc = 0
        for c in contr_coeff:
            out[r:r + c.shape[0], cc:cc + c.shape[1]] = c
            r += c.shape[0]
            cc += c.shape[1]
        return pmol, out
    c2s = gto_oracle.cart2sph_coeff(mol)
    cols = np.cumsum([0] + [c.shape[0] for c in contr_coeff])
    rows = np.cumsum([0] + [c.shape[1] for c in contr_coeff])
    out = np.empty((cols[-1], c2s.shape[1]))
    for i, c in enumerate(contr_coeff):
        out[cols[i]:cols[i + 1]] = c.dot(c2s[rows[i]:rows[i + 1]])
    return pmol, out


def _split_l_ctr_groups(uniq_l_ctr, l_ctr_counts, group_size):
    ls, counts = [], []
    for l_ctr, cnt in zip(uniq_l_ctr, l_ctr_counts):
        l = l_ctr[0]
        nf = (l + 1) * (l + 2) // 2
        max_shells = max(group_size // nf, 2)
        if l > LMAX_ON_GPU or cnt <= max_shells:
            ls.append(l_ctr)
            counts.append(cnt)
            continue
        nsub, rest = divmod(cnt, max_shells)
        ls.extend([l_ctr] * nsub)
        counts.extend([max_shells] * nsub)
        if rest > 0:
            ls.append(l_ctr)
            counts.append(rest)
    return np.vstack(ls), np.hstack(counts)


class VHFOpt:
    def __init__(self, mol):
        self.mol, self.coeff = basis_seg_contraction(mol)

    def build(self, cutoff=1e-13, group_size=None, diag_block_with_triu=False):
        mol = self.mol
        l_ctrs = mol._bas[:, [gmole.ANG_OF, gmole.NPRIM_OF]]
        uniq_l_ctr, _, inv_idx, l_ctr_counts = np.unique(
            l_ctrs, return_index=True, return_inverse=True,
            return_counts=True, axis=0)
        inv_idx = np.asarray(inv_idx).ravel()
        # the reference computes quartets with a shell above h on the CPU
        # through PySCF (hf.py:185-218); the oracle keeps them in the same
        # screened loop as the rest, up to i shells
        if uniq_l_ctr[:, 0].max() > LMAX_ORACLE:
            raise NotImplementedError('l > 6 shells')
        if group_size is not None:
            uniq_l_ctr, l_ctr_counts = _split_l_ctr_groups(
                uniq_l_ctr, l_ctr_counts, group_size)
        sorted_idx = np.argsort(inv_idx, kind='stable').astype(np.int32)
        ao_loc = mol.ao_loc_nr(cart=True)
        nao = ao_loc[-1]
        ao_idx = np.array_split(np.arange(nao), ao_loc[1:-1])
        ao_idx = np.hstack([ao_idx[i] for i in sorted_idx])
        self.coeff = self.coeff[ao_idx]
        mol._bas = mol._bas[sorted_idx]
        self.direct_scf_tol = cutoff
        q_cond = oracle.q_cond(mol)
        self.q_cond = q_cond
        log_qs, pair2bra, pair2ket = [], [], []
        l_ctr_offsets = np.append(0, np.cumsum(l_ctr_counts))
        for i, (p0, p1) in enumerate(zip(l_ctr_offsets[:-1],
                                         l_ctr_offsets[1:])):
            for q0, q1 in zip(l_ctr_offsets[:i], l_ctr_offsets[1:i + 1]):
                q_sub = q_cond[p0:p1, q0:q1].ravel()
                idx = q_sub.argsort(axis=None)[::-1]
                q_sorted = q_sub[idx]
                mask = q_sorted > cutoff
                idx = idx[mask]
                ishs, jshs = np.unravel_index(idx, (p1 - p0, q1 - q0))
                pair2bra.append(ishs + p0)
                pair2ket.append(jshs + q0)
                log_q = np.log(q_sorted[mask])
                log_q[log_q > 0] = 0
                log_qs.append(log_q)
            q_sub = q_cond[p0:p1, p0:p1].ravel()
            idx = q_sub.argsort(axis=None)[::-1]
            q_sorted = q_sub[idx]
            ishs, jshs = np.unravel_index(idx, (p1 - p0, p1 - p0))
            mask = q_sorted > cutoff
            if not diag_block_with_triu:
                mask &= ishs >= jshs
            pair2bra.append(ishs[mask] + p0)
            pair2ket.append(jshs[mask] + p0)
            log_q = np.log(q_sorted[mask])
            log_q[log_q > 0] = 0
            log_qs.append(log_q)
        self.uniq_l_ctr = uniq_l_ctr
        self.l_ctr_offsets = l_ctr_offsets
        self.bas_pair2shls = np.hstack(pair2bra + pair2ket).astype(
            np.int32).reshape(2, -1)
        self.bas_pairs_locs = np.append(
            0, np.cumsum([x.size for x in pair2bra])).astype(np.int32)
        self.log_qs = log_qs
        self.diag_fac = 1. if diag_block_with_triu else .5
        return self


def make_s_index_offsets(log_q, nbins=10, cutoff=1e-12):
    scale = nbins / np.log(min(cutoff, .1))
    s_index = np.floor(scale * log_q).astype(np.int32)
    bins = np.bincount(s_index)
    if bins.size < nbins:
        bins = np.append(bins, np.zeros(nbins - bins.size, dtype=np.int32))
    else:
        bins = bins[:nbins]
    if bins.max() >= 65536 * 8:
        raise RuntimeError('bin too large')
    return np.append(0, np.cumsum(bins)).astype(np.int32)


def condense_absmax(x, loc):
    n = len(loc) - 1
    out = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            blk = x[loc[i]:loc[i + 1], loc[j]:loc[j + 1]]
            out[i, j] = np.abs(blk).max() if blk.size else 0.
    return out


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True,
           prescreen=True, nbins=None, stats=None, ij_stride=1, ij_offset=0,
           count_only=False):
    """Oracle J/K.  Returns numpy (vj, vk) shaped like ``dm``; a disabled
    matrix is None.  ``ij_stride``/``ij_offset`` evaluate only the rows
    ij = ij_offset mod ij_stride of every class pair (a subsample for timing);
    ``count_only`` evaluates nothing and only counts the quartets (in
    ``stats['quartets']``)."""
    if hermi != 1:
        raise NotImplementedError('JK-builder only supports hermitian '
                                  'density matrix')
    if vhfopt is None:
        vhfopt = VHFOpt(mol).build()
    coeff = vhfopt.coeff
    nao, nao0 = coeff.shape
    dm0 = np.asarray(dm)
    dms = dm0.reshape(-1, nao0, nao0)
    n_dm = dms.shape[0]
    dms = np.einsum('pi,nij,qj->npq', coeff, dms, coeff, optimize=True)
    dms = np.ascontiguousarray(dms)
    vj = np.zeros(n_dm * nao * nao) if with_j else None
    vk = np.zeros(n_dm * nao * nao) if with_k else None
    pmol = vhfopt.mol
    log_qs = vhfopt.log_qs
    locs = vhfopt.bas_pairs_locs
    tol = vhfopt.direct_scf_tol
    if nbins is None:
        pairs_max = (locs[1:] - locs[:-1]).max()
        nbins = max(10, int(pairs_max // 100000))
    ncptype = len(log_qs)
    cp_idx, cp_jdx = np.tril_indices(ncptype)
    l_ctr_ao_loc = pmol.ao_loc_nr(cart=True)[vhfopt.l_ctr_offsets]
    dm_cond = np.max([condense_absmax(x, l_ctr_ao_loc) for x in dms], axis=0)
    p2b = np.ascontiguousarray(vhfopt.bas_pair2shls[0])
    p2k = np.ascontiguousarray(vhfopt.bas_pair2shls[1])
    ao_loc = pmol.ao_loc_nr(cart=True)
    lib = oracle.lib()
    nquartets = 0
    if not count_only and lib.oracle_jk_begin(
            ctypes.c_int(nao), ctypes.c_int(n_dm), ctypes.c_int(int(with_j)),
            ctypes.c_int(int(with_k))):
        raise MemoryError('oracle J/K accumulators')
    for n in range(ncptype * (ncptype + 1) // 2):
        cp_ij = int(np.floor(np.sqrt(2 * n)))
        if cp_ij * (cp_ij + 1) // 2 > n:
            cp_ij -= 1
        cp_kl = n - cp_ij * (cp_ij + 1) // 2
        lq_ij, lq_kl = log_qs[cp_ij], log_qs[cp_kl]
        cpi, cpj = cp_idx[cp_ij], cp_jdx[cp_ij]
        cpk, cpl = cp_idx[cp_kl], cp_jdx[cp_kl]
        if lq_ij.size == 0 or lq_kl.size == 0:
            continue
        sub = max(dm_cond[cpi, cpj], dm_cond[cpk, cpl], dm_cond[cpi, cpk],
                  dm_cond[cpj, cpk], dm_cond[cpi, cpl], dm_cond[cpj, cpl])
        if prescreen and sub < tol:
            continue
        with np.errstate(divide='ignore'):
            cutoff = tol / sub
        bins_ij = make_s_index_offsets(lq_ij, nbins, cutoff)
        bins_kl = make_s_index_offsets(lq_kl, nbins, cutoff)
        nquartets += lib.oracle_build_jk(
            _ptr(pmol._atm), _ptr(pmol._bas), _ptr(pmol._env),
            ctypes.c_int(pmol.nbas), _ptr(ao_loc), _ptr(p2b), _ptr(p2k),
            _ptr(locs), ctypes.c_double(vhfopt.diag_fac), _ptr(dms),
            ctypes.c_int(nao), ctypes.c_int(n_dm),
            _ptr(vj) if with_j else None, _ptr(vk) if with_k else None,
            _ptr(bins_ij), _ptr(bins_kl), ctypes.c_int(nbins),
            ctypes.c_int(cp_ij), ctypes.c_int(cp_kl), ctypes.c_int(ij_stride),
            ctypes.c_int(ij_offset), ctypes.c_int(int(count_only)))
    if not count_only:
        lib.oracle_jk_end(_ptr(vj) if with_j else None,
                          _ptr(vk) if with_k else None)
    if stats is not None:
        stats['quartets'] = nquartets
        stats['nbins'] = nbins
    out = []
    for v, fac in ((vj, 2.), (vk, 1.)):
        if v is None:
            out.append(None)
            continue
        V = v.reshape(n_dm, nao, nao).transpose(0, 2, 1)
        W = np.einsum('pi,npq,qj->nij', coeff, V + V.transpose(0, 2, 1),
                      coeff, optimize=True) * fac
        out.append(W.reshape(dm0.shape) if dm0.ndim == 2 else W)
    if dm0.ndim == 2:
        out = [o[0] if o is not None and o.ndim == 3 else o for o in out]
    return out[0], out[1]
