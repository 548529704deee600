"""Batched J/K over many molecules in one pass on one GPU.

``JKBatch(mols)`` builds a _VHFOpt per molecule and one engine batch; then
``get_jk(dms)`` returns [(vj, vk), ...] for all molecules from a single
sequence of launches (one per class shared by the molecules; a class
quartet of at least ``solo_tasks`` unscreened tasks keeps a launch of its
own), and
``capture(dms)`` / ``replay()`` record that sequence in a CUDA graph so an SCF
iteration of the whole batch is one graph launch.  ``tune(dms)`` runs the
engine's autotuner (``jk_batch_tune``): every class launch of the batch is
timed in its candidate shapes (static chunks, or persistent grids taking
chunks from a device counter) and the fastest is kept, optionally through a
cache file.  Densities and results use the layout of the single-molecule
``get_jk`` (``cuobc/scf/hf.py:53-227``).
"""
import ctypes

import numpy as np

from byteqc_b200.cuobc import lib as _lib
from byteqc_b200.cuobc.scf import hf


def _ptrs(seq):
    arr = (ctypes.c_void_p * len(seq))()
    for i, p in enumerate(seq):
        arr[i] = p
    return arr


class JKBatch:
    def __init__(self, mols, cutoff=1e-13, vhfopts=None, solo_tasks=None):
        torch = hf._torch()
        self.lib = _lib.load_library()
        self.mols = list(mols)
        self.opts = vhfopts or [hf._VHFOpt(m).build(cutoff) for m in self.mols]
        self.nmol = len(self.mols)
        handles = _ptrs([o.handle.value for o in self.opts])
        self.handle = ctypes.c_void_p()
        if solo_tasks is None:
            _lib.check(self.lib.jk_batch_create(handles, self.nmol,
                                                ctypes.byref(self.handle)),
                       'jk_batch_create')
        else:
            _lib.check(self.lib.jk_batch_create_ex(handles, self.nmol,
                                                   int(solo_tasks),
                                                   ctypes.byref(self.handle)),
                       'jk_batch_create_ex')
        n = ctypes.c_int()
        _lib.check(self.lib.jk_batch_nsolo(self.handle, ctypes.byref(n)),
                   'jk_batch_nsolo')
        self.nsolo = n.value
        self.nao0 = [o.coeff.shape[1] for o in self.opts]
        self._coeffs = _ptrs([o.coeff_dev.data_ptr() for o in self.opts])
        self._nao0 = (ctypes.c_int * self.nmol)(*self.nao0)
        self._buffers = None
        self._graph = None
        self.torch = torch

    def _opts(self, prescreen, nbins, fp32_cutoff):
        o = _lib.JKOpts()
        o.direct_scf_tol = self.opts[0].direct_scf_tol
        o.nbins = nbins if nbins is not None else max(
            op.default_nbins() for op in self.opts)
        o.prescreen = int(bool(prescreen))
        o.fp32_cutoff = float(fp32_cutoff or 0.)
        return o

    def _ensure_buffers(self, n_dm):
        torch = self.torch
        if self._buffers is None or self._buffers[0] != n_dm:
            dm = [torch.zeros(n_dm, n, n, dtype=torch.float64, device='cuda')
                  for n in self.nao0]
            vj = [torch.zeros_like(d) for d in dm]
            vk = [torch.zeros_like(d) for d in dm]
            self._buffers = (n_dm, dm, vj, vk)
        return self._buffers

    def _load(self, dms):
        torch = self.torch
        shapes = [tuple(np.shape(d)) for d in dms]
        n_dm = 1 if len(shapes[0]) == 2 else shapes[0][0]
        _, bdm, bvj, bvk = self._ensure_buffers(n_dm)
        for b, d, n in zip(bdm, dms, self.nao0):
            b.copy_(torch.as_tensor(d, dtype=torch.float64).reshape(n_dm, n, n),
                    non_blocking=False)
        return n_dm, shapes

    def _run(self, n_dm, with_j, with_k, o):
        _, bdm, bvj, bvk = self._buffers
        stream = ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        _lib.check(self.lib.jk_batch_get_jk(
            self.handle, self._coeffs, self._nao0,
            _ptrs([b.data_ptr() for b in bdm]),
            _ptrs([b.data_ptr() for b in bvj]) if with_j else None,
            _ptrs([b.data_ptr() for b in bvk]) if with_k else None,
            n_dm, ctypes.byref(o), stream), 'jk_batch_get_jk')

    def _results(self, shapes, with_j, with_k, out):
        _, _, bvj, bvk = self._buffers
        res = []
        for m, shp in enumerate(shapes):
            pair = []
            for use, b in ((with_j, bvj[m]), (with_k, bvk[m])):
                if not use:
                    pair.append(None)
                    continue
                v = b.reshape(shp)
                pair.append(v.clone() if out == 'device' else v.cpu().numpy())
            res.append(tuple(pair))
        return res

    def get_jk(self, dms, with_j=True, with_k=True, prescreen=True, nbins=None,
               fp32_cutoff=None, out='host'):
        """J/K of every molecule; ``dms[m]`` has molecule m's (n_dm, nao,
        nao) or (nao, nao) shape, numpy or CUDA tensor."""
        if len(dms) != self.nmol:
            raise ValueError('one density per molecule expected')
        n_dm, shapes = self._load(dms)
        self._run(n_dm, with_j, with_k, self._opts(prescreen, nbins,
                                                   fp32_cutoff))
        return self._results(shapes, with_j, with_k, out)

    # -- autotuner -----------------------------------------------------------
    def tune(self, dms, prescreen=True, nbins=None, fp32_cutoff=None,
             cache=None):
        """Choose the launch shape of every class launch of the batch by
        timing the candidates on these densities (FP64 part, and the FP32
        part when ``fp32_cutoff`` > 0).  ``cache``: path of a text file of
        earlier choices, read first and rewritten.  A captured graph is
        dropped (it holds the old shapes).  Returns ``info()``."""
        torch = self.torch
        n_dm, _ = self._load(dms)
        _, bdm, _, _ = self._buffers
        w, vj, vk = [], [], []
        for b, op in zip(bdm, self.opts):
            C = op.coeff_dev
            w.append(torch.stack([C @ b[d] @ C.T for d in range(n_dm)])
                     .contiguous())
            vj.append(torch.zeros_like(w[-1]))
            vk.append(torch.zeros_like(w[-1]))
        o = self._opts(prescreen, nbins, fp32_cutoff)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(self.lib.jk_batch_tune(
            self.handle, _ptrs([x.data_ptr() for x in w]),
            _ptrs([x.data_ptr() for x in vj]),
            _ptrs([x.data_ptr() for x in vk]), n_dm, ctypes.byref(o),
            cache.encode() if cache else None, stream), 'jk_batch_tune')
        self._graph = None
        return self.info()

    def info(self):
        """Launch shape of every class launch: class index, primitive
        counts (-1: any), task bound, and per part (FP64, FP32) the grab
        (0: static chunks), grid multiple, tuned time (ms, None if not
        tuned) and segment count."""
        n = ctypes.c_int()
        _lib.check(self.lib.jk_batch_info(self.handle, ctypes.byref(n), None),
                   'jk_batch_info')
        out = np.zeros((max(n.value, 1), 12), dtype=np.int32)
        _lib.check(self.lib.jk_batch_info(self.handle, ctypes.byref(n),
                                          out.ctypes.data), 'jk_batch_info')
        res = []
        for r in out[:n.value]:
            parts = []
            for p in range(2):
                g, gm, us, ns = (int(v) for v in r[4 + 4 * p:8 + 4 * p])
                parts.append({'grab': g, 'grid_mul': gm,
                              'ms': us / 1e3 if us >= 0 else None,
                              'segments': ns})
            res.append({'class': int(r[0]), 'np_ij': int(r[1]),
                        'np_kl': int(r[2]), 'tasks': int(r[3]),
                        'fp64': parts[0], 'fp32': parts[1]})
        return res

    # -- CUDA graph of one batched build ----------------------------------
    def capture(self, dms, with_j=True, with_k=True, prescreen=True,
                nbins=None, fp32_cutoff=None):
        """Record one batched build in a CUDA graph; ``replay(dms)`` then
        copies new densities into the captured input buffers and launches
        the graph."""
        torch = self.torch
        n_dm, shapes = self._load(dms)
        o = self._opts(prescreen, nbins, fp32_cutoff)
        self._run(n_dm, with_j, with_k, o)  # warm-up: tables, attributes
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self._run(n_dm, with_j, with_k, o)
        torch.cuda.current_stream().wait_stream(s)
        self._graph = (g, shapes, with_j, with_k, o)
        return self

    def replay(self, dms=None, out='host'):
        g, shapes, with_j, with_k, _ = self._graph
        if dms is not None:
            self._load(dms)
        g.replay()
        return self._results(shapes, with_j, with_k, out)

    def close(self):
        if getattr(self, 'handle', None) is not None and self.handle.value:
            self.lib.jk_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
