"""Continuous-batching J/K server: many SCF calculations share the GPU.

Requests (a molecule, optionally a starting density) arrive over time; each
runs ``n_iter`` SCF iterations (or fewer, once its energy change falls below
``conv_tol``) whose J/K builds the server executes.  The scheduler loop

* admits waiting requests while a slot is free and their device footprint,
  bounded from the basis sizes before anything is allocated, fits the HBM
  budget (setup -- Schwarz screening and pair cache -- then runs at admission
  and stays on the device with the request's density, Fock history and
  orbitals until it finishes; the exact footprint replaces the bound);
* runs ONE batched J/K pass for all admitted requests (each request's
  iteration k), so requests that arrived at different times overlap on the
  device; the engine batch is kept while the set of active requests does
  not change and rebuilt when one joins or leaves;
* advances every request's SCF state (Fock matrix, DIIS, eigensolver, all on
  the device) and retires finished requests, freeing their slot and memory.

Recorded per request: the latency of each of its J/K builds (issue to
completion of the batched pass that carries it: all builds of a pass
complete together), of each of its iterations (step start to the end of
its own SCF update), and of the whole request (arrival to last iteration);
``stats()`` reports their p50/p99 and the builds/s.  The result of a request
does not depend on what it was batched with: every J/K build is the same
computation with the same screening as a build of that molecule alone.
"""
import collections
import time

import numpy as np

from byteqc_b200.cuobc.scf import hf
from byteqc_b200.cuobc.scf.batch import JKBatch


def _footprint(nbas, nao, nao0, npairs, nprim):
    """Device bytes of an admitted request from its basis sizes: shell-pair
    Schwarz matrix, pair lists and primitive-pair cache (basis handle),
    density / J / K work buffers in the working basis and the back
    transform, and the SCF state (S, H, orthogonaliser, density, DIIS
    history) in the caller's basis."""
    words = (nbas * nbas + 4 * npairs + 6 * nprim + 6 * npairs  # basis
             + 6 * nao * nao + nao * nao0                       # work buffers
             + 16 * nao0 * nao0)                                # SCF state
    return 8 * words


def footprint_bound_bytes(mol):
    """Upper bound of footprint_bytes(opt) from the basis alone (no device
    work, nothing allocated): every shell pair counted as kept by the
    Schwarz screen."""
    pmol, coeff = hf.basis_seg_contraction(mol)
    bas = pmol._bas
    nbas = int(bas.shape[0])
    ls = bas[:, 1]
    nps = bas[:, 2].astype(np.int64)
    nao = int(((ls + 1) * (ls + 2) // 2).sum())
    nprim = int((nps.sum() ** 2 + (nps ** 2).sum()) // 2)
    return _footprint(nbas, nao, coeff.shape[1], nbas * (nbas + 1) // 2, nprim)


def footprint_bytes(opt):
    """Device bytes a request holds while admitted, from the sizes of its
    basis handle (the shell pairs the Schwarz screen kept)."""
    from byteqc_b200.cuobc import lib as _lib
    info = np.zeros(7, dtype=np.int32)
    _lib.load_library().jk_basis_info(opt.handle, info.ctypes.data)
    nbas, nao, ngroups, ncp, npairs, nprim, ncq = (int(v) for v in info)
    return _footprint(nbas, nao, opt.coeff.shape[1], npairs, nprim)


class _Request:
    def __init__(self, rid, mol, arrival, n_iter, dm0, conv_tol):
        self.rid = rid
        self.mol = mol
        self.arrival = arrival
        self.n_iter = n_iter
        self.dm0 = dm0
        self.conv_tol = conv_tol
        self.iter = 0
        self.energies = []
        self.build_lat = []
        self.iter_lat = []
        self.done_time = None
        self.converged = False


class _SCFState:
    """Device-resident RHF state of one request (core guess, DIIS, optional
    level shift of the virtual space: F + shift (S - S D S / 2), which
    damps oscillations and leaves the converged energy unchanged)."""

    def __init__(self, req, opt, torch, level_shift=0.):
        mol = req.mol
        dev = dict(dtype=torch.float64, device='cuda')
        self.torch = torch
        self.s = torch.as_tensor(mol.intor('int1e_ovlp'), **dev)
        self.h = torch.as_tensor(mol.intor('int1e_kin') + mol.intor('int1e_nuc'), **dev)
        self.e_nuc = mol.energy_nuc()
        self.nocc = mol.nelectron // 2
        seig, t = torch.linalg.eigh(self.s)
        keep = seig >= 1e-15
        self.x = t[:, keep] / torch.sqrt(seig[keep])
        if req.dm0 is not None:
            self.dm = torch.as_tensor(req.dm0, **dev)
        else:
            _, c = hf.eig(self.h, self.s)
            self.dm = 2. * c[:, :self.nocc] @ c[:, :self.nocc].T
        self.fs, self.es = [], []
        self.level_shift = level_shift

    def update(self, vj, vk):
        torch = self.torch
        f = self.h + vj - .5 * vk
        e = float(.5 * torch.sum(self.dm * (self.h + f))) + self.e_nuc
        err = self.x.T @ (f @ self.dm @ self.s - self.s @ self.dm @ f) @ self.x
        self.fs.append(f)
        self.es.append(err)
        self.fs, self.es = self.fs[-8:], self.es[-8:]
        n = len(self.fs)
        if n > 1:
            b = torch.empty(n + 1, n + 1, dtype=torch.float64, device='cuda')
            b[-1, :] = -1
            b[:, -1] = -1
            b[-1, -1] = 0
            for i in range(n):
                for j in range(i + 1):
                    b[i, j] = b[j, i] = torch.sum(self.es[i] * self.es[j])
            rhs = torch.zeros(n + 1, dtype=torch.float64, device='cuda')
            rhs[-1] = -1
            coef = torch.linalg.lstsq(b, rhs[:, None]).solution[:n, 0]
            f = sum(ci * fi for ci, fi in zip(coef, self.fs))
        if self.level_shift:
            sds = self.s @ self.dm @ self.s
            f = f + self.level_shift * (self.s - 0.5 * sds)
        _, c = hf.eig(f, self.s)
        self.dm = 2. * c[:, :self.nocc] @ c[:, :self.nocc].T
        return e


class JKServer:
    def __init__(self, hbm_budget_bytes=40 << 30, max_slots=64,
                 fp32_cutoff=None, n_iter=15, cutoff=1e-13, conv_tol=None,
                 level_shift=0.):
        self.torch = hf._torch()
        self.budget = hbm_budget_bytes
        self.max_slots = max_slots
        self.fp32_cutoff = fp32_cutoff
        self.n_iter = n_iter
        self.cutoff = cutoff
        self.conv_tol = conv_tol
        self.level_shift = level_shift
        self.waiting = collections.deque()
        self.active = []  # (request, opt, state, bytes)
        self.finished = []
        self.used = 0
        self.builds = 0
        self.steps = 0
        self._next_id = 0
        self._batch = None
        self._batch_ids = None
        self.batch_builds = 0  # engine batches created

    def submit(self, mol, arrival=None, dm0=None, n_iter=None):
        rid = self._next_id
        self._next_id += 1
        self.waiting.append(_Request(rid, mol, time.perf_counter() if arrival is None else arrival,
                                     n_iter or self.n_iter, dm0, self.conv_tol))
        return rid

    def _admit(self):
        while self.waiting and len(self.active) < self.max_slots:
            req = self.waiting[0]
            bound = footprint_bound_bytes(req.mol)
            if bound > self.budget:
                raise MemoryError('request %d may need %d bytes, over the '
                                  'budget' % (req.rid, bound))
            if self.active and self.used + bound > self.budget:
                break
            self.waiting.popleft()
            opt = hf._VHFOpt(req.mol).build(self.cutoff)
            need = footprint_bytes(opt)
            self.active.append((req, opt, _SCFState(req, opt, self.torch,
                                                    self.level_shift), need))
            self.used += need

    def _engine_batch(self):
        ids = tuple(a[0].rid for a in self.active)
        if ids != self._batch_ids:
            if self._batch is not None:
                self._batch.close()
            self._batch = JKBatch([a[0].mol for a in self.active],
                                  vhfopts=[a[1] for a in self.active])
            self._batch_ids = ids
            self.batch_builds += 1
        return self._batch

    def step(self):
        """Admit, run one batched J/K pass for every active request, advance
        their SCF states, retire finished ones.  Returns the number of
        builds done."""
        torch = self.torch
        self._admit()
        if not self.active:
            return 0
        t0 = time.perf_counter()
        batch = self._engine_batch()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        res = batch.get_jk([a[2].dm for a in self.active], out='device',
                           fp32_cutoff=self.fp32_cutoff)
        ev1.record()
        ev1.synchronize()
        lat = ev0.elapsed_time(ev1) * 1e-3
        still = []
        for (req, opt, st, nbytes), (vj, vk) in zip(self.active, res):
            req.energies.append(st.update(vj, vk))
            torch.cuda.current_stream().synchronize()
            req.build_lat.append(lat)
            req.iter_lat.append(time.perf_counter() - t0)
            req.iter += 1
            conv = (req.conv_tol is not None and len(req.energies) > 1 and
                    abs(req.energies[-1] - req.energies[-2]) < req.conv_tol)
            if conv or req.iter >= req.n_iter:
                req.converged = conv
                req.done_time = time.perf_counter()
                req.dm_final = st.dm
                self.finished.append(req)
                self.used -= nbytes
                opt.clear()
            else:
                still.append((req, opt, st, nbytes))
        if len(still) != len(self.active) and self._batch is not None:
            self._batch.close()  # its molecules change: rebuilt next step
            self._batch, self._batch_ids = None, None
        self.active = still
        self.builds += len(res)
        self.steps += 1
        return len(res)

    def run_until_empty(self):
        while self.waiting or self.active:
            self.step()

    def stats(self):
        lat = np.array([x for r in self.finished for x in r.build_lat])
        itl = np.array([x for r in self.finished for x in r.iter_lat])
        req = np.array([r.done_time - r.arrival for r in self.finished])
        out = {'requests': len(self.finished), 'builds': int(lat.size),
               'engine_batches': self.batch_builds, 'steps': self.steps}
        if lat.size:
            out.update(build_p50_ms=float(np.percentile(lat, 50) * 1e3),
                       build_p99_ms=float(np.percentile(lat, 99) * 1e3),
                       iteration_p50_ms=float(np.percentile(itl, 50) * 1e3),
                       iteration_p99_ms=float(np.percentile(itl, 99) * 1e3))
        if req.size:
            out.update(request_p50_s=float(np.percentile(req, 50)),
                       request_p99_s=float(np.percentile(req, 99)))
        return out


def single_build_seconds(mol, cutoff=1e-13, fp32_cutoff=None):
    """Seconds of one J/K build of ``mol`` alone on the GPU at the density
    its request starts from (the core guess), after one untimed build: the
    service time a request's iteration costs without batching, for sizing
    an arrival rate.  (A diagonal or otherwise sparse density would let the
    density screen drop most quartets and overstate the capacity.)"""
    torch = hf._torch()
    opt = hf._VHFOpt(mol).build(cutoff)
    try:
        st = _SCFState(_Request(-1, mol, 0., 1, None, None), opt, torch)
        for _ in range(2):
            torch.cuda.synchronize()
            t = time.perf_counter()
            hf.get_jk(mol, st.dm, vhfopt=opt, out='device',
                      fp32_cutoff=fp32_cutoff)
            torch.cuda.synchronize()
        return time.perf_counter() - t
    finally:
        opt.clear()


def poisson_serve(mols, rate_per_s, duration_s=None, seed=5, **server_kw):
    """Drive a JKServer with Poisson arrivals of ``mols`` (in order) at
    ``rate_per_s``; returns (server, wall seconds)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=len(mols))
    srv = JKServer(**server_kw)
    t0 = time.perf_counter()
    arrivals = t0 + np.cumsum(gaps)
    i = 0
    while i < len(mols) or srv.waiting or srv.active:
        now = time.perf_counter()
        while i < len(mols) and arrivals[i] <= now:
            srv.submit(mols[i], arrival=arrivals[i])
            i += 1
        if srv.waiting or srv.active:
            srv.step()
        elif i < len(mols):
            time.sleep(max(0., min(arrivals[i] - now, 0.01)))
    return srv, time.perf_counter() - t0
