"""Direct-SCF J/K on the B200: the host side of ByteQC's ``cuobc`` J/K path.

Same call as the reference (``cuobc/scf/hf.py:53-55``)::

    vj, vk = get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True)

``mol`` is a :class:`byteqc_b200.gto.Mole` (the libcint-layout subset of a
PySCF ``Mole`` the path reads), ``dm`` a numpy array or a CUDA tensor of
shape (nao, nao) or (n_dm, nao, nao).  The result has ``dm``'s shape and
comes back as numpy float64 arrays, as in the reference (``hf.py:176,181``),
or as CUDA tensors with ``out='device'``.  A disabled matrix is returned as
``None``.

Everything after the argument checks runs on the GPU through libjk.so: the
AO transforms, the density condensation, the screening, the Rys J/K kernels
and the symmetrisation.  There is no CPU fallback.
"""
import ctypes
import math

import numpy as np

from byteqc_b200.cuobc import lib as _lib
from byteqc_b200.gto import mole as gmole

LMAX_ON_GPU = 5  # h functions: the reference's GPU limit (group splitting)
# Shells up to i (l = 6) run on the GPU here; the reference hands quartets
# with an i shell to PySCF on the CPU (cuobc/scf/hf.py:185-218).
LMAX_ENGINE = 6
ANGULAR = 'spdfghik'


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError('the J/K engine needs a CUDA device')
    return torch


def _stream_ptr(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def basis_seg_contraction(mol):
    """Working basis of the J/K kernels (cuobc/scf/hf.py:481-564): every
    generally contracted shell (nctr > 1) is split into its primitive shells,
    functions are Cartesian, and ``coeff`` (nao_working, nao) maps the
    working basis back to ``mol``'s contracted (spherical or Cartesian)
    functions.  Shells with one contraction are kept as they are."""
    env = mol._env.copy()
    new_bas = []
    blocks = []  # (rows, cols) transform block per original shell
    for shell in mol._bas:
        l, nprim, nctr = (int(shell[gmole.ANG_OF]), int(shell[gmole.NPRIM_OF]),
                          int(shell[gmole.NCTR_OF]))
        nf = gmole.ncart(l)
        if nctr == 1:
            new_bas.append(shell.copy())
            blocks.append(np.eye(nf))
            continue
        pexp, pcoeff = int(shell[gmole.PTR_EXP]), int(shell[gmole.PTR_COEFF])
        exps = mol._env[pexp:pexp + nprim]
        norm = gmole.gto_norm(l, exps)
        # atoms of one element share env slots: read the original
        # coefficients, not the copy already rewritten for an earlier atom
        c = mol._env[pcoeff:pcoeff + nprim * nctr].reshape(nctr, nprim) / norm
        # rows: (primitive p, component f); cols: (contraction i, component f)
        blk = np.kron(c.T, np.eye(nf))
        env[pcoeff:pcoeff + nprim] = norm
        for p in range(nprim):
            s = shell.copy()
            s[gmole.NPRIM_OF] = 1
            s[gmole.NCTR_OF] = 1
            s[gmole.PTR_EXP] = pexp + p
            s[gmole.PTR_COEFF] = pcoeff + p
            new_bas.append(s)
        blocks.append(blk)
    pmol = mol.copy()
    pmol.cart = True
    pmol._bas = np.asarray(new_bas, dtype=np.int32).reshape(-1, gmole.BAS_SLOTS)
    pmol._env = env
    nrow = sum(b.shape[0] for b in blocks)
    ncol = sum(b.shape[1] for b in blocks)
    contr = np.zeros((nrow, ncol))
    r = c0 = 0
    for b in blocks:
        contr[r:r + b.shape[0], c0:c0 + b.shape[1]] = b
        r += b.shape[0]
        c0 += b.shape[1]
    if mol.cart:
        return pmol, contr
    return pmol, contr @ mol.cart2sph_coeff()


def _split_l_ctr_groups(uniq_l_ctr, l_ctr_counts, group_size):
    """Cap the AOs per (l, nprim) group (cuobc/scf/hf.py:581-606)."""
    ls, counts = [], []
    for l_ctr, cnt in zip(uniq_l_ctr, l_ctr_counts):
        nf = gmole.ncart(int(l_ctr[0]))
        max_shells = max(group_size // nf, 2)
        full, rest = divmod(int(cnt), max_shells) if cnt > max_shells else (0, int(cnt))
        ls.extend([l_ctr] * (full + (rest > 0)))
        counts.extend([max_shells] * full + ([rest] if rest else []))
    return np.vstack(ls), np.asarray(counts)


def _make_s_index_offsets(log_q, nbins=10, cutoff=1e-12):
    """Log-Schwarz bin offsets of a Schwarz-sorted pair list
    (cuobc/scf/hf.py:567-578); for callers of the per-class-pair entry."""
    scale = nbins / np.log(min(cutoff, .1))
    s_index = np.floor(scale * log_q).astype(np.int32)
    bins = np.bincount(s_index, minlength=nbins)[:nbins]
    return np.append(0, np.cumsum(bins)).astype(np.int32)


class _VHFOpt:
    """Per-geometry J/K setup, the counterpart of the reference's _VHFOpt
    (cuobc/scf/hf.py:277-448).  ``build`` sorts the working basis into
    (l, nprim) groups and creates the device-side basis: Schwarz matrix,
    Schwarz-sorted pair lists and the primitive-pair cache."""

    def __init__(self, mol, intor='int2e', prescreen='CVHFnoscreen',
                 qcondname='CVHFsetnr_direct_scf', dmcondname=None):
        self.mol, self.coeff = basis_seg_contraction(mol)
        self._intor = intor
        self.handle = None

    def build(self, cutoff=1e-13, group_size=None, diag_block_with_triu=False,
              gpus=None):
        if gpus not in (None, 1, [0], (0,)) and not isinstance(gpus, int):
            pass  # one GPU per process; replicas scale out (see bench.py)
        torch = _torch()
        lib = _lib.load_library()
        mol = self.mol
        l_ctrs = mol._bas[:, [gmole.ANG_OF, gmole.NPRIM_OF]]
        uniq_l_ctr, inv_idx, l_ctr_counts = np.unique(
            l_ctrs, return_inverse=True, return_counts=True, axis=0)
        inv_idx = np.asarray(inv_idx).ravel()
        lmax = int(uniq_l_ctr[:, 0].max())
        if lmax > LMAX_ENGINE:
            raise NotImplementedError(
                'shells with l=%d: this engine handles l <= %d'
                % (lmax, LMAX_ENGINE))
        if group_size is not None:
            uniq_l_ctr, l_ctr_counts = _split_l_ctr_groups(
                uniq_l_ctr, l_ctr_counts, group_size)
        sorted_idx = np.argsort(inv_idx, kind='stable').astype(np.int32)
        ao_loc = mol.ao_loc_nr(cart=True)
        ao_idx = np.concatenate([np.arange(ao_loc[i], ao_loc[i + 1])
                                 for i in sorted_idx])
        self.coeff = self.coeff[ao_idx]
        mol._bas = np.ascontiguousarray(mol._bas[sorted_idx])
        self.direct_scf_tol = cutoff
        self.uniq_l_ctr = uniq_l_ctr
        self.l_ctr_offsets = np.append(0, np.cumsum(l_ctr_counts)).astype(
            np.int32)
        self.diag_fac = 1. if diag_block_with_triu else .5
        self.h_shls = []
        self.g_shls = []

        handle = ctypes.c_void_p()
        atm = np.ascontiguousarray(mol._atm, dtype=np.int32)
        bas = np.ascontiguousarray(mol._bas, dtype=np.int32)
        env = np.ascontiguousarray(mol._env, dtype=np.float64)
        _lib.check(lib.jk_basis_create(
            atm.ctypes.data, mol.natm, bas.ctypes.data, mol.nbas,
            env.ctypes.data, env.size, self.l_ctr_offsets.ctypes.data,
            len(uniq_l_ctr), cutoff, int(diag_block_with_triu),
            ctypes.byref(handle)), 'jk_basis_create')
        self.handle = handle
        info = np.zeros(7, dtype=np.int32)
        _lib.check(lib.jk_basis_info(handle, info.ctypes.data), 'jk_basis_info')
        nbas, nao, ngroups, ncp, npairs = (int(v) for v in info[:5])
        self.nao = nao
        pair2shls = np.zeros((2, max(npairs, 1)), dtype=np.int32)
        locs = np.zeros(ncp + 1, dtype=np.int32)
        log_q = np.zeros(max(npairs, 1))
        q_cond = np.zeros((nbas, nbas))
        _lib.check(lib.jk_basis_pairs(handle, pair2shls.ctypes.data,
                                      locs.ctypes.data, log_q.ctypes.data,
                                      q_cond.ctypes.data), 'jk_basis_pairs')
        self.bas_pair2shls = pair2shls[:, :npairs]
        self.bas_pairs_locs = locs
        self.log_qs = [log_q[locs[i]:locs[i + 1]] for i in range(ncp)]
        self.q_cond = q_cond
        self.coeff_dev = torch.as_tensor(self.coeff, dtype=torch.float64,
                                         device='cuda').contiguous()
        return self

    def get_q_cond(self):
        return self.q_cond

    def default_nbins(self):
        """cuobc/scf/hf.py:96-100."""
        locs = self.bas_pairs_locs
        pairs_max = int((locs[1:] - locs[:-1]).max()) if len(locs) > 1 else 0
        return max(10, pairs_max // 100000)

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


def get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True,
           omega=None, verbose=None, group_size=None, gpus=None,
           prescreen=True, nbins=None, out='host', fp32_cutoff=None,
           group=None):
    """Coulomb and exchange matrices of the density matrices ``dm``.

    ``fp32_cutoff``: mixed precision -- contracted quartets whose screened
    bound q_ij q_kl max|D| is below it run the Rys recursion and products in
    FP32 (roots, weights, prefactors and all J/K accumulation stay FP64);
    None or 0 keeps everything in FP64 (the reference's arithmetic).

    ``group``: a ``torch.distributed`` process group, one rank per GPU (the
    reference's multi-GPU task farm, cuobc/scf/hf.py:147-169 with
    lib/multigpu.py:136-329): every rank builds its share of the class
    quartets (``jk_shard_plan`` on their cost, the same plan on every rank)
    and the partial J and K are summed by one all-reduce each, so every rank
    returns the full result.  Every rank of the group must call with the
    same molecule and density."""
    if hermi != 1:
        raise NotImplementedError(
            'JK-builder only supports hermitian density matrix')
    torch = _torch()
    lib = _lib.load_library()
    if vhfopt is None:
        vhfopt = _VHFOpt(mol, 'int2e').build(gpus=gpus, group_size=group_size)
    nao, nao0 = vhfopt.coeff.shape
    is_tensor = isinstance(dm, torch.Tensor)
    shape = tuple(dm.shape)
    if shape[-1] != nao0 or shape[-2] != nao0 or len(shape) not in (2, 3):
        raise ValueError('dm of shape %s does not match nao=%d' % (shape, nao0))
    d = torch.as_tensor(dm, dtype=torch.float64, device='cuda')
    d = d.reshape(-1, nao0, nao0).contiguous()
    n_dm = d.shape[0]
    vj = torch.empty_like(d) if with_j else None
    vk = torch.empty_like(d) if with_k else None
    if not with_j and not with_k:
        return None, None
    opts = _lib.JKOpts()
    opts.direct_scf_tol = vhfopt.direct_scf_tol
    opts.nbins = nbins if nbins is not None else vhfopt.default_nbins()
    opts.prescreen = int(bool(prescreen))
    opts.fp32_cutoff = float(fp32_cutoff or 0.)
    if group is not None:
        import torch.distributed as dist
        opts.shard = dist.get_rank(group)
        opts.nshards = dist.get_world_size(group)
    _lib.check(lib.jk_get_jk(
        vhfopt.handle, vhfopt.coeff_dev.data_ptr(), nao0, d.data_ptr(), n_dm,
        vj.data_ptr() if with_j else None, vk.data_ptr() if with_k else None,
        ctypes.byref(opts), _stream_ptr(torch)), 'jk_get_jk')
    if group is not None and opts.nshards > 1:
        import torch.distributed as dist
        for v in (vj, vk):
            if v is not None:
                dist.all_reduce(v, group=group)
    res = []
    for v in (vj, vk):
        if v is None:
            res.append(None)
            continue
        v = v.reshape(shape)
        res.append(v if (out == 'device' or (out == 'same' and is_tensor))
                   else v.cpu().numpy())
    return res[0], res[1]


def get_jk_class_pairs(mol, dm, vhfopt, with_j=True, with_k=True,
                       prescreen=True, nbins=None):
    """J/K through the reference's own task loop (cuobc/scf/hf.py:104-166):
    per-group absmax condensation of the densities, the class-level density
    screen, log-Schwarz bins per class pair (``_make_s_index_offsets``) and
    one ``jk_build_class_pair`` call per class quartet -- the GINTbuild_jk
    contract (cuobc/lib/gvhf/nr_jk_driver.cu:227-284) on the per-class-pair
    kernels.  Same result as :func:`get_jk` (which screens on the device and
    runs the tiled kernels) up to rounding; returns CUDA tensors."""
    torch = _torch()
    lib = _lib.load_library()
    nao, nao0 = vhfopt.coeff.shape
    C = vhfopt.coeff_dev
    d = torch.as_tensor(dm, dtype=torch.float64, device='cuda')
    shape = tuple(d.shape)
    d = d.reshape(-1, nao0, nao0)
    n_dm = d.shape[0]
    dms = (C @ d @ C.T).contiguous()
    vj = torch.zeros(n_dm, nao, nao, dtype=torch.float64, device='cuda')
    vk = torch.zeros_like(vj)
    gao = vhfopt.mol.ao_loc_nr(cart=True)[vhfopt.l_ctr_offsets]
    ng = len(gao) - 1
    a = dms.abs().amax(0)
    dm_cond = np.zeros((ng, ng))
    for gi in range(ng):
        rows = a[gao[gi]:gao[gi + 1]]
        for gj in range(ng):
            dm_cond[gi, gj] = float(rows[:, gao[gj]:gao[gj + 1]].max())
    tol = vhfopt.direct_scf_tol
    nbins = nbins if nbins is not None else vhfopt.default_nbins()
    log_qs = vhfopt.log_qs
    cp_idx, cp_jdx = np.tril_indices(ng)
    sp = _stream_ptr(torch)
    for cp_ij in range(len(log_qs)):
        for cp_kl in range(cp_ij + 1):
            lq_ij, lq_kl = log_qs[cp_ij], log_qs[cp_kl]
            if lq_ij.size == 0 or lq_kl.size == 0:
                continue
            i, j, k, l = cp_idx[cp_ij], cp_jdx[cp_ij], cp_idx[cp_kl], cp_jdx[cp_kl]
            sub = max(dm_cond[i, j], dm_cond[k, l], dm_cond[i, k],
                      dm_cond[j, k], dm_cond[i, l], dm_cond[j, l])
            if prescreen and sub < tol:
                continue
            with np.errstate(divide='ignore'):
                cutoff = tol / sub
            bij = _make_s_index_offsets(lq_ij, nbins, cutoff)
            bkl = _make_s_index_offsets(lq_kl, nbins, cutoff)
            _lib.check(lib.jk_build_class_pair(
                vhfopt.handle, vj.data_ptr() if with_j else None,
                vk.data_ptr() if with_k else None, dms.data_ptr(), nao, n_dm,
                bij.ctypes.data, bkl.ctypes.data, nbins, cp_ij, cp_kl, sp),
                'jk_build_class_pair')
    out = []
    for v, fac, on in ((vj, 2., with_j), (vk, 1., with_k)):
        if not on:
            out.append(None)
            continue
        w = fac * (C.T @ (v + v.transpose(1, 2)) @ C)
        out.append(w.reshape(shape))
    return out[0], out[1]


def _get_jk(mf, mol=None, dm=None, hermi=1, with_j=True, with_k=True,
            omega=None):
    """RHF.get_jk of the reference (cuobc/scf/hf.py:230-250): builds and
    caches the _VHFOpt on first use."""
    if omega is not None:
        raise NotImplementedError('Range separated Coulomb integrals')
    if mol is None:
        mol = mf.mol
    if getattr(mf, '_opt_gpu', None) is None:
        mf._opt_gpu = _VHFOpt(mol, 'int2e').build(mf.direct_scf_tol)
    return get_jk(mol, dm, hermi, mf._opt_gpu, with_j, with_k)


def eig(h, s):
    """Generalised eigenproblem h C = s C e through Loewdin orthogonalisation
    on the GPU (cuobc/scf/hf.py:253-265): functions with overlap eigenvalue
    below 1e-15 are dropped."""
    torch = _torch()
    s = torch.as_tensor(s, dtype=torch.float64, device='cuda')
    h = torch.as_tensor(h, dtype=torch.float64, device='cuda')
    seig, t = torch.linalg.eigh(s)
    keep = seig >= 1e-15
    t = t[:, keep] / torch.sqrt(seig[keep])
    e, c = torch.linalg.eigh(t.T @ h @ t)
    return e, t @ c


class RHF:
    """Restricted Hartree-Fock driver around the J/K engine.

    The reference's ``RHF`` (cuobc/scf/hf.py:272-274) overrides ``get_jk`` and
    ``_eigh`` of PySCF's ``hf.RHF``; PySCF is not a dependency here, so this
    class provides the loop itself: core-Hamiltonian guess, DIIS on the
    orthogonalised commutator F D S - S D F, and direct-SCF incremental Fock
    builds (J/K of the density change added to the previous ones, rebuilt from
    scratch every ``rebuild_every`` cycles), all on the GPU.  ``fp32_cutoff``
    switches on the mixed-precision engine.
    """

    def __init__(self, mol, fp32_cutoff=None):
        self.mol = mol
        self.conv_tol = 1e-9
        self.conv_tol_grad = None
        self.max_cycle = 60
        self.direct_scf = True
        self.direct_scf_tol = 1e-13
        self.diis_space = 8
        self.rebuild_every = 8
        self.fp32_cutoff = fp32_cutoff
        self.converged = False
        self.e_tot = None
        self.cycles = 0
        self.jk_builds = 0
        self._opt_gpu = None

    def get_jk(self, mol=None, dm=None, hermi=1, with_j=True, with_k=True,
               omega=None):
        if omega is not None:
            raise NotImplementedError('Range separated Coulomb integrals')
        if mol is None:
            mol = self.mol
        if self._opt_gpu is None:
            self._opt_gpu = _VHFOpt(mol, 'int2e').build(self.direct_scf_tol)
        self.jk_builds += 1
        return get_jk(mol, dm, hermi, self._opt_gpu, with_j, with_k,
                      out='device', fp32_cutoff=self.fp32_cutoff)

    def eig(self, h, s):
        return eig(h, s)

    def kernel(self, dm0=None):
        torch = _torch()
        mol = self.mol
        dev = dict(dtype=torch.float64, device='cuda')
        s = torch.as_tensor(mol.intor('int1e_ovlp'), **dev)
        h = torch.as_tensor(mol.intor('int1e_kin') + mol.intor('int1e_nuc'),
                            **dev)
        e_nuc = mol.energy_nuc()
        nocc = mol.nelectron // 2
        if dm0 is None:
            _, c = self.eig(h, s)
            dm = 2. * c[:, :nocc] @ c[:, :nocc].T
        else:
            dm = torch.as_tensor(dm0, **dev)
        seig, t = torch.linalg.eigh(s)
        x = t[:, seig >= 1e-15] / torch.sqrt(seig[seig >= 1e-15])
        vj = vk = None
        dm_last = None
        fs, es = [], []
        e_last = None
        self.converged = False
        for cycle in range(1, self.max_cycle + 1):
            if (self.direct_scf and dm_last is not None
                    and cycle % self.rebuild_every != 0):
                dj, dk = self.get_jk(mol, dm - dm_last)
                vj, vk = vj + dj, vk + dk
            else:
                vj, vk = self.get_jk(mol, dm)
            f = h + vj - .5 * vk
            e_tot = float(.5 * torch.sum(dm * (h + f))) + e_nuc
            err = x.T @ (f @ dm @ s - s @ dm @ f) @ x
            fs.append(f)
            es.append(err)
            if len(fs) > self.diis_space:
                fs.pop(0)
                es.pop(0)
            n = len(fs)
            if n > 1:
                b = torch.empty(n + 1, n + 1, **dev)
                b[-1, :] = -1
                b[:, -1] = -1
                b[-1, -1] = 0
                for i in range(n):
                    for j in range(i + 1):
                        b[i, j] = b[j, i] = torch.sum(es[i] * es[j])
                rhs = torch.zeros(n + 1, **dev)
                rhs[-1] = -1
                coef = torch.linalg.lstsq(b, rhs[:, None]).solution[:n, 0]
                f = sum(ci * fi for ci, fi in zip(coef, fs))
            mo_e, c = self.eig(f, s)
            dm_last = dm
            dm = 2. * c[:, :nocc] @ c[:, :nocc].T
            grad = float(err.abs().max())
            self.cycles = cycle
            if e_last is not None and abs(e_tot - e_last) < self.conv_tol and (
                    self.conv_tol_grad is None or grad < self.conv_tol_grad):
                self.converged = True
                self.e_tot = e_tot
                break
            e_last = e_tot
        # final energy of the converged density with a full (non-incremental) build
        vj, vk = self.get_jk(mol, dm)
        f = h + vj - .5 * vk
        self.e_tot = float(.5 * torch.sum(dm * (h + f))) + e_nuc
        self.mo_energy, self.mo_coeff = mo_e.cpu().numpy(), c.cpu().numpy()
        self.make_rdm1 = lambda: dm.cpu().numpy()
        return self.e_tot
