"""ORACLE (test infrastructure only): drives the reference's OWN J/K and
ERI-fill library -- ByteQC ``cuobc/lib/gint`` and ``cuobc/lib/gvhf``,
compiled unmodified for sm_100a into ``oracle/_ref/`` by
``oracle/ref/Makefile`` -- through its ctypes C-ABI, the way the
reference's Python layer does:

  - ``BasisProdCache`` / ``ContractionProdType`` mirrored as ctypes
    structures (``cuobc/scf/hf.py:451-478``, ``gint/gint.h:110-147``);
  - ``GINTinit_basis_prod_cpu`` then ``GINTinit_basis_prod_gpu`` over
    device copies of ``ao_loc``, the shell coordinates, ``aexyz`` and the
    pair lists (``hf.py:410-437``, ``gint/nr_fill_ao_ints.cu:452-491``);
    the pair lists, (l, nprim) groups and log-Schwarz values come from the
    oracle's restatement of ``_VHFOpt.build`` (``oracle/hf_oracle.py``);
  - the ``get_jk`` task loop (``hf.py:67-181``): dms = C D C^T, per-group
    absmax condensation, class-level density screen, log-Schwarz bins,
    ``GINTbuild_jk`` per class pair (``gvhf/nr_jk_driver.cu:227-284``), then
    J = 2 C^T (V + V^T) C and K = C^T (V + V^T) C;
  - ``GINTfill_int2e`` (``nr_fill_ao_ints.cu:493-549``) per class pair, with
    the slice set-up of ``cuobc/lib/int4c.py:73-127``.

Device buffers are torch tensors (the reference uses CuPy, absent here).
The reference's allocation helpers call ``exit`` on a CUDA error
(``gint/cuda_alloc.cuh:21-31``), so callers run this module in a child
process: ``python -m oracle.ref_jk <in.pkl> <out.pkl>``; ``run()`` does that.
"""
import ctypes
import os
import pickle
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, '_ref')


class ContractionProdType(ctypes.Structure):
    _fields_ = [('l_bra', ctypes.c_int), ('l_ket', ctypes.c_int),
                ('nprim_12', ctypes.c_int), ('npairs', ctypes.c_int)]


class BasisProdCache(ctypes.Structure):
    _fields_ = [
        ('nbas', ctypes.c_int), ('ncptype', ctypes.c_int),
        ('cptype', ctypes.POINTER(ContractionProdType)),
        ('bas_pairs_locs', ctypes.POINTER(ctypes.c_int)),
        ('primitive_pairs_locs', ctypes.POINTER(ctypes.c_int)),
        ('bas_pair2shls', ctypes.POINTER(ctypes.c_int)),
        ('aexyz', ctypes.POINTER(ctypes.c_double)),
        ('bas_coords', ctypes.POINTER(ctypes.c_double)),
        ('bas_pair2bra', ctypes.POINTER(ctypes.c_int)),
        ('bas_pair2ket', ctypes.POINTER(ctypes.c_int)),
        ('ao_loc', ctypes.POINTER(ctypes.c_int)),
        ('a12', ctypes.POINTER(ctypes.c_double)),
        ('e12', ctypes.POINTER(ctypes.c_double)),
        ('x12', ctypes.POINTER(ctypes.c_double)),
        ('y12', ctypes.POINTER(ctypes.c_double)),
        ('z12', ctypes.POINTER(ctypes.c_double)),
    ]


def available():
    return all(os.path.exists(os.path.join(REF_DIR, f))
               for f in ('libgint.so', 'libgvhf.so'))


_LIBS = None


def libs():
    global _LIBS
    if _LIBS is None:
        gint = ctypes.CDLL(os.path.join(REF_DIR, 'libgint.so'),
                           mode=ctypes.RTLD_GLOBAL)
        gvhf = ctypes.CDLL(os.path.join(REF_DIR, 'libgvhf.so'))
        P = ctypes.POINTER(BasisProdCache)
        gvhf.GINTbuild_jk.restype = ctypes.c_int
        gvhf.GINTbuild_jk.argtypes = [
            P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        gint.GINTfill_int2e.restype = ctypes.c_int
        gint.GINTfill_int2e.argtypes = [
            P, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _LIBS = (gint, gvhf)
    return _LIBS


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefBasis:
    """The reference's BasisProdCache over the oracle's VHFOpt, with its
    device arrays held as torch tensors (hf.py:410-437)."""

    def __init__(self, vhfopt):
        import torch
        gint, _ = libs()
        self.opt = vhfopt
        pmol = vhfopt.mol
        self._atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
        self._bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
        self._env = np.ascontiguousarray(pmol._env, dtype=np.float64)
        self._p2s = np.ascontiguousarray(vhfopt.bas_pair2shls, dtype=np.int32)
        self._locs = np.ascontiguousarray(vhfopt.bas_pairs_locs,
                                          dtype=np.int32)
        ncptype = len(vhfopt.log_qs)
        ao_loc = np.asarray(pmol.ao_loc_nr(cart=True), dtype=np.int32)
        bas_coords = np.empty(pmol.nbas * 3)
        cpu = ctypes.POINTER(BasisProdCache)()
        gint.GINTinit_basis_prod_cpu(
            ctypes.byref(cpu), ctypes.c_double(vhfopt.diag_fac),
            _ptr(bas_coords), _ptr(self._p2s), _ptr(self._locs),
            ctypes.c_int(ncptype), _ptr(self._atm), ctypes.c_int(pmol.natm),
            _ptr(self._bas), ctypes.c_int(pmol.nbas), _ptr(self._env))
        nprim = cpu.contents.primitive_pairs_locs[ncptype]
        aexyz = np.ctypeslib.as_array(cpu.contents.aexyz, (nprim * 5,))
        dev = torch.device('cuda')
        self.d_ao_loc = torch.as_tensor(ao_loc, device=dev)
        self.d_coords = torch.as_tensor(bas_coords, device=dev)
        self.d_aexyz = torch.as_tensor(aexyz.copy(), device=dev)
        self.d_p2s = torch.as_tensor(self._p2s.ravel(), device=dev)
        self.gpu = ctypes.POINTER(BasisProdCache)()
        gint.GINTinit_basis_prod_gpu(
            ctypes.byref(cpu), ctypes.byref(self.gpu),
            ctypes.c_void_p(self.d_ao_loc.data_ptr()),
            ctypes.c_void_p(self.d_coords.data_ptr()),
            ctypes.c_void_p(self.d_aexyz.data_ptr()),
            ctypes.c_void_p(self.d_p2s.data_ptr()))
        self.ncptype = ncptype
        self.nao = int(ao_loc[-1])

    def close(self):
        # the reference frees the GPU copy only (hf.py:439-441); the host
        # arrays it shares with the CPU copy go with it
        if self.gpu:
            libs()[0].GINTdel_basis_prod(ctypes.byref(self.gpu))
            self.gpu = None


def _tasks(rb, dms_host, nbins, prescreen):
    """The task list of get_jk (hf.py:104-166): (cp_ij, cp_kl, bins_ij,
    bins_kl) of every class pair that survives the density screen."""
    from oracle import hf_oracle
    opt = rb.opt
    log_qs = opt.log_qs
    locs = opt.bas_pairs_locs
    if nbins is None:
        pairs_max = (locs[1:] - locs[:-1]).max()
        nbins = max(10, int(pairs_max // 100000))
    ncp = len(log_qs)
    cp_idx, cp_jdx = np.tril_indices(ncp)
    l_ctr_ao_loc = opt.mol.ao_loc_nr(cart=True)[opt.l_ctr_offsets]
    dm_cond = np.max([hf_oracle.condense_absmax(x, l_ctr_ao_loc)
                      for x in dms_host], axis=0)
    tol = opt.direct_scf_tol
    out = []
    for n in range(ncp * (ncp + 1) // 2):
        cp_ij = int(np.floor(np.sqrt(2 * n)))
        if cp_ij * (cp_ij + 1) // 2 > n:
            cp_ij -= 1
        cp_kl = n - cp_ij * (cp_ij + 1) // 2
        lq_ij, lq_kl = log_qs[cp_ij], log_qs[cp_kl]
        if lq_ij.size == 0 or lq_kl.size == 0:
            continue
        cpi, cpj, cpk, cpl = (cp_idx[cp_ij], cp_jdx[cp_ij], cp_idx[cp_kl],
                              cp_jdx[cp_kl])
        sub = max(dm_cond[cpi, cpj], dm_cond[cpk, cpl], dm_cond[cpi, cpk],
                  dm_cond[cpj, cpk], dm_cond[cpi, cpl], dm_cond[cpj, cpl])
        if prescreen and sub < tol:
            continue
        with np.errstate(divide='ignore'):
            cutoff = tol / sub
        out.append((cp_ij, cp_kl,
                    hf_oracle.make_s_index_offsets(lq_ij, nbins, cutoff),
                    hf_oracle.make_s_index_offsets(lq_kl, nbins, cutoff)))
    return nbins, out


def get_jk(mol, dm, with_j=True, with_k=True, nbins=None, prescreen=True,
           timing=None, vhfopt=None):
    """J, K of ``dm`` through the reference's GINTbuild_jk.  ``timing``
    (warmup, reps) also times the launch loop with CUDA events (density
    already on the device, task bins precomputed): returns ms per build.

    One density only: for n_dm > 1 the reference's generic digestion
    (cuobc/lib/gvhf/contract_jk.cu:226-310) does not restart its index walk
    over the local integral array for the second density and reads below
    that array, so more densities are refused here rather than run."""
    import torch
    from oracle import hf_oracle
    _, gvhf = libs()
    opt = vhfopt or hf_oracle.VHFOpt(mol).build()
    rb = RefBasis(opt)
    try:
        coeff = np.asarray(opt.coeff)
        nao, nao0 = coeff.shape
        dm0 = np.asarray(dm)
        dms = dm0.reshape(-1, nao0, nao0)
        n_dm = dms.shape[0]
        if n_dm != 1:
            raise ValueError('the reference kernels are run with one density '
                             'per call (see the docstring)')
        dms = np.ascontiguousarray(
            np.einsum('pi,nij,qj->npq', coeff, dms, coeff, optimize=True))
        nbins, tasks = _tasks(rb, dms, nbins, prescreen)
        dev = torch.device('cuda')
        d_dm = torch.as_tensor(dms, device=dev)
        vj = torch.zeros((n_dm, nao, nao), dtype=torch.float64, device=dev) \
            if with_j else None
        vk = torch.zeros_like(vj if vj is not None else d_dm) \
            if with_k else None
        stream = torch.cuda.current_stream()

        def loop():
            for cp_ij, cp_kl, bij, bkl in tasks:
                err = gvhf.GINTbuild_jk(
                    rb.gpu, None if vj is None else vj.data_ptr(),
                    None if vk is None else vk.data_ptr(), d_dm.data_ptr(),
                    nao, n_dm, _ptr(bij), _ptr(bkl), nbins, cp_ij, cp_kl,
                    stream.cuda_stream)
                if err:
                    raise RuntimeError('GINTbuild_jk(%d, %d) returned %d'
                                       % (cp_ij, cp_kl, err))

        loop()
        torch.cuda.synchronize()
        out = []
        for v, fac in ((vj, 2.), (vk, 1.)):
            if v is None:
                out.append(None)
                continue
            V = v.cpu().numpy().transpose(0, 2, 1)
            W = np.einsum('pi,npq,qj->nij', coeff, V + V.transpose(0, 2, 1),
                          coeff, optimize=True) * fac
            out.append(W[0] if dm0.ndim == 2 else W.reshape(dm0.shape))
        ms = None
        if timing:
            warm, reps = timing
            for _ in range(warm):
                loop()
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                loop()
            t1.record(stream)
            torch.cuda.synchronize()
            ms = t0.elapsed_time(t1) / reps
        return out[0], out[1], {'ms_per_build': ms, 'launch_calls': len(tasks),
                                'nbins': nbins}
    finally:
        rb.close()


def fill_blocks(vhfopt, pairs, nbins=1, cutoff=None):
    """Blocks of the ERI tensor, one per class pair (cp_ij, cp_kl) of
    ``pairs``, through GINTfill_int2e with the slice set-up of
    ``cuobc/lib/int4c.py:73-127``: the (ni, nj, nk, nl) block of the four
    (l, nprim) groups, strides (nj nk nl, nk nl, nl, 1), AO offsets of the
    groups, bins from ``_make_s_index_offsets`` at ``cutoff`` (default the
    VHFOpt's direct_scf_tol).  Returns numpy blocks."""
    import torch
    from oracle import hf_oracle
    gint, _ = libs()
    rb = RefBasis(vhfopt)
    cutoff = vhfopt.direct_scf_tol if cutoff is None else cutoff
    ao_loc = vhfopt.mol.ao_loc_nr(cart=True)
    offs = vhfopt.l_ctr_offsets
    cp_idx, cp_jdx = np.tril_indices(len(offs) - 1)
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    try:
        for cp_ij, cp_kl in pairs:
            g = (cp_idx[cp_ij], cp_jdx[cp_ij], cp_idx[cp_kl], cp_jdx[cp_kl])
            a0 = [int(ao_loc[offs[x]]) for x in g]
            n = [int(ao_loc[offs[x + 1]]) - a for x, a in zip(g, a0)]
            eri = torch.zeros(n, dtype=torch.float64, device='cuda')
            st = np.array([n[1] * n[2] * n[3], n[2] * n[3], n[3], 1],
                          dtype=np.int32)
            of = np.array(a0, dtype=np.int32)
            bij = hf_oracle.make_s_index_offsets(vhfopt.log_qs[cp_ij], nbins,
                                                 cutoff)
            bkl = hf_oracle.make_s_index_offsets(vhfopt.log_qs[cp_kl], nbins,
                                                 cutoff)
            err = gint.GINTfill_int2e(rb.gpu, eri.data_ptr(), rb.nao,
                                      _ptr(st), _ptr(of), _ptr(bij),
                                      _ptr(bkl), nbins, cp_ij, cp_kl, stream)
            if err:
                raise RuntimeError('GINTfill_int2e(%d, %d) returned %d'
                                   % (cp_ij, cp_kl, err))
            out.append(eri.cpu().numpy())
        return out
    finally:
        rb.close()


def get_int4c_timing(vhfopt, nbins=1, reps=3):
    """CUDA-event time of the reference's ``get_int4c`` flow
    (``cuobc/lib/int4c.py:44-70``) on one GPU: for every class pair a zeroed
    block, ``GINTfill_int2e`` into it, then the eight permuted copies into
    the dense (nao, nao, nao, nao) tensor; one untimed pass first.  Returns
    {'ms': mean ms of the whole tensor, 'ms_fill_calls': the fill calls
    alone (blocks allocated and zeroed beforehand), 'pairs': class pairs}."""
    import torch
    from oracle import hf_oracle
    gint, _ = libs()
    rb = RefBasis(vhfopt)
    cutoff = vhfopt.direct_scf_tol
    ao_loc = vhfopt.mol.ao_loc_nr(cart=True)
    offs = vhfopt.l_ctr_offsets
    ncp = len(offs) - 1
    cp_idx, cp_jdx = np.tril_indices(ncp)
    npair = len(vhfopt.log_qs)
    pairs = list(zip(*np.tril_indices(npair)))
    nao = int(ao_loc[offs[-1]])
    stream = torch.cuda.current_stream().cuda_stream
    setup = []
    for cp_ij, cp_kl in pairs:
        g = (cp_idx[cp_ij], cp_jdx[cp_ij], cp_idx[cp_kl], cp_jdx[cp_kl])
        a0 = [int(ao_loc[offs[x]]) for x in g]
        n = [int(ao_loc[offs[x + 1]]) - a for x, a in zip(g, a0)]
        st = np.array([n[1] * n[2] * n[3], n[2] * n[3], n[3], 1], dtype=np.int32)
        of = np.array(a0, dtype=np.int32)
        bij = hf_oracle.make_s_index_offsets(vhfopt.log_qs[cp_ij], nbins, cutoff)
        bkl = hf_oracle.make_s_index_offsets(vhfopt.log_qs[cp_kl], nbins, cutoff)
        sl = [slice(a, a + m) for a, m in zip(a0, n)]
        setup.append((int(cp_ij), int(cp_kl), n, st, of, bij, bkl, sl))

    def fill(blk, cp_ij, cp_kl, st, of, bij, bkl):
        err = gint.GINTfill_int2e(rb.gpu, blk.data_ptr(), nao, _ptr(st),
                                  _ptr(of), _ptr(bij), _ptr(bkl), nbins,
                                  cp_ij, cp_kl, stream)
        if err:
            raise RuntimeError('GINTfill_int2e(%d, %d) returned %d'
                               % (cp_ij, cp_kl, err))

    def whole():
        out = torch.zeros((nao,) * 4, dtype=torch.float64, device='cuda')
        for cp_ij, cp_kl, n, st, of, bij, bkl, (si, sj, sk, sl) in setup:
            b = torch.zeros(n, dtype=torch.float64, device='cuda')
            fill(b, cp_ij, cp_kl, st, of, bij, bkl)
            out[si, sj, sk, sl] = b
            out[sj, si, sk, sl] = b.permute(1, 0, 2, 3)
            out[si, sj, sl, sk] = b.permute(0, 1, 3, 2)
            out[sj, si, sl, sk] = b.permute(1, 0, 3, 2)
            out[sk, sl, si, sj] = b.permute(2, 3, 0, 1)
            out[sk, sl, sj, si] = b.permute(2, 3, 1, 0)
            out[sl, sk, si, sj] = b.permute(3, 2, 0, 1)
            out[sl, sk, sj, si] = b.permute(3, 2, 1, 0)
        return out

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    try:
        ms = timed(whole)
        blks = [torch.zeros(x[2], dtype=torch.float64, device='cuda') for x in setup]

        def calls():
            for b, (cp_ij, cp_kl, n, st, of, bij, bkl, _) in zip(blks, setup):
                fill(b, cp_ij, cp_kl, st, of, bij, bkl)
        ms_calls = timed(calls)
        return {'ms': ms, 'ms_fill_calls': ms_calls, 'pairs': len(pairs),
                'nao': nao}
    finally:
        rb.close()


def run(func, *args, timeout=1800, **kwargs):
    """Call ``func`` (a name in this module) in a child process."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        fin = os.path.join(d, 'in.pkl')
        fout = os.path.join(d, 'out.pkl')
        with open(fin, 'wb') as f:
            pickle.dump((func, args, kwargs), f)
        root = os.path.dirname(_HERE)
        env = dict(os.environ)
        env['PYTHONPATH'] = root + os.pathsep + env.get('PYTHONPATH', '')
        p = subprocess.run([sys.executable, '-m', 'oracle.ref_jk', fin, fout],
                           cwd=root, env=env, capture_output=True, text=True,
                           timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError('reference child failed (%d): %s'
                               % (p.returncode, (p.stdout + p.stderr)[-2000:]))
        with open(fout, 'rb') as f:
            return pickle.load(f)


if __name__ == '__main__':
    with open(sys.argv[1], 'rb') as f:
        name, args, kwargs = pickle.load(f)
    import torch
    torch.cuda.set_device(0)
    res = globals()[name](*args, **kwargs)
    with open(sys.argv[2], 'wb') as f:
        pickle.dump(res, f)
