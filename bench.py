#!/usr/bin/env python
"""J/K build throughput on one B200 (or N independent replicas).

A step is one direct-SCF J/K build (FP64 J and K of one density) of the
workload, through the engine's entry jk_get_jk with the density resident on
the device (``value``), and end to end through the public get_jk call with
host numpy input and output (``e2e``).  Default workload: a seeded (H2O)32
cluster in a 14 A cube with the def2-TZVP stand-in basis (s-f shells, 1376
spherical functions), density D = 2 C C^T with C^T S C = 1.

Timing: CUDA events on the launching stream around each step, L2 flushed
(a 512 MiB buffer written) before every timed step, max over ranks.
The CPU baseline is the oracle (the OpenMP restatement of the reference's
algorithm) on the host cores, timed on a uniform subsample of shell-pair rows
and scaled to a full build.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nwater, cube A, seed, basis)
    'h2o32-tzvp': (32, 14.0, 2, 'standin-def2-tzvp'),
    'h2o8-dz': (8, 9.0, 0, 'standin-cc-pvdz'),
    'h2o64-dz': (64, 18.0, 3, 'standin-cc-pvdz'),
    'h2o12-tzvp': (12, 10.5, 2, 'standin-def2-tzvp'),  # small case for ncu captures
    # a 60-atom random-walk molecule (the kind of the batched workload)
    'walk60-631gs': ('walk', 60, 11, 'standin-6-31g*'),
}


def make_workload(name, oracle_overlap=False):
    """Molecule and density of a named workload.  ``oracle_overlap`` takes
    the overlap matrix for the density from the oracle's own integrals
    instead of the engine's one-electron code (the reference arm maps no
    engine library); the two agree to 1e-13."""
    from byteqc_b200.gto import Mole, geom
    nw, box, seed, basis = WORKLOADS[name]
    if nw == 'walk':
        mol = Mole(atom=geom.random_walk_molecule(box, seed=seed),
                   basis=basis).build()
    else:
        mol = Mole(atom=geom.water_cluster(nw, box=box, seed=seed),
                   basis=basis).build()
    if oracle_overlap:
        from oracle import gto_oracle
        s = gto_oracle.overlap(mol)
    else:
        s = mol.intor('int1e_ovlp')
    dm = geom.scf_like_density(s, nocc=mol.nelectron // 2, seed=1)
    return mol, dm


# DRAM bytes (read + write) of one build's class-quartet launches, summed
# from an ncu launch list of `bench.py --profile-builds 2` on the workload
PROFILED_TRAFFIC = {'h2o32-tzvp': 78.9e6, 'h2o12-tzvp': 5.7e6}


def batch_workload(nmol=256, seed=4, basis='standin-6-31g*'):
    """Seeded molecules of 3-60 atoms grown by a random walk (elements
    C:N:O:H = 3:1:1:5), each with a D = 2 C C^T density.  A molecule with an
    odd electron count is taken as its cation (charge +1), so that every
    molecule is closed-shell for the RHF runs."""
    from byteqc_b200.gto import Mole, geom
    rng = np.random.default_rng(seed)
    mols, dms = [], []
    for i in range(nmol):
        natm = int(rng.integers(3, 61))
        atoms = geom.random_walk_molecule(natm, seed=seed * 100003 + i)
        m = Mole(atom=atoms, basis=basis).build()
        if m.nelectron % 2:
            m = Mole(atom=atoms, basis=basis, charge=1).build()
        s = m.intor('int1e_ovlp')
        mols.append(m)
        dms.append(geom.scf_like_density(s, nocc=m.nelectron // 2, seed=i))
    return mols, dms


def bench_batch(args, torch, timed):
    """Builds of the 256-molecule workload: per-molecule launches in FP64 (the
    plain engine), and the batch (one launch per shared class) replayed from a
    captured CUDA graph in FP64 and in mixed precision, first with static
    chunks, then with the launch shapes the autotuner picks; then an RHF of
    every molecule through the batched server, FP64 and mixed, and the
    energy difference of each.  Returns the 'batch' sub-object of the bench
    line."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.batch import JKBatch
    mols, dms = batch_workload(args.batch_mols)
    t = time.perf_counter()
    batch = JKBatch(mols)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t
    nbf = [m.nao for m in mols]
    d_dms = [torch.as_tensor(d, device='cuda') for d in dms]

    def per_molecule():
        for m, d, o in zip(mols, d_dms, batch.opts):
            hf.get_jk(m, d, vhfopt=o, out='device')

    ref = batch.get_jk(d_dms, out='device')
    # first-order energy error of the mixed mode at each molecule's density:
    # 1/2 tr(D (dJ - dK/2)) -- the SCF energy is stationary in the density,
    # so this is the SCF energy difference to first order
    mix = batch.get_jk(d_dms, out='device', fp32_cutoff=args.fp32_cutoff)
    de_fixed = [0.5 * float((d * ((mj - rj) - 0.5 * (mk - rk))).sum())
                for d, (rj, rk), (mj, mk) in zip(d_dms, ref, mix)]

    def err_vs_ref():
        got = batch._results(batch._graph[1] if batch._graph else
                             [tuple(d.shape) for d in d_dms], True, True, 'device')
        return max(max((a[0] - b[0]).abs().max().item(),
                       (a[1] - b[1]).abs().max().item())
                   for a, b in zip(ref, got))
    batch._load(d_dms)
    res = {}
    per_molecule()
    ms = timed(per_molecule, args.batch_steps)
    res['per_molecule_fp64'] = {'ms': ms, 'builds_per_s': len(mols) * 1e3 / ms}

    def graphs(suffix):
        for name, cut in (('graph_fp64', 0.), ('graph_mixed', args.fp32_cutoff)):
            batch.capture(d_dms, fp32_cutoff=cut)
            g = batch._graph[0]
            g.replay()
            ms = timed(g.replay, args.batch_steps)
            res[name + suffix] = {'ms': ms, 'builds_per_s': len(mols) * 1e3 / ms,
                                  'max_abs_err_jk_vs_fp64': err_vs_ref()}
    graphs('')
    t = time.perf_counter()
    info = batch.tune(d_dms, fp32_cutoff=args.fp32_cutoff)
    tune_s = time.perf_counter() - t
    batch._load(d_dms)
    graphs('_tuned')
    res['graph_mixed']['fp32_cutoff'] = args.fp32_cutoff
    res['graph_mixed_tuned']['fp32_cutoff'] = args.fp32_cutoff
    base = res['per_molecule_fp64']['builds_per_s']
    shapes = {'launches': len(info),
              'persistent_fp64': sum(1 for k in info if k['fp64']['grab'] > 0),
              'persistent_fp32': sum(1 for k in info if k['fp32']['grab'] > 0),
              'tune_s': tune_s}
    batch.close()
    out = {'molecules': len(mols), 'basis': 'standin-6-31g*',
           'nbf_min': min(nbf), 'nbf_max': max(nbf), 'nbf_mean': float(np.mean(nbf)),
           'setup_s': setup, 'variants': res, 'tuned_shapes': shapes,
           'speedup_graph_mixed_tuned_vs_per_molecule_fp64':
               res['graph_mixed_tuned']['builds_per_s'] / base,
           'speedup_graph_fp64_tuned_vs_per_molecule_fp64':
               res['graph_fp64_tuned']['builds_per_s'] / base,
           'speedup_graph_mixed_vs_graph_fp64':
               res['graph_mixed']['builds_per_s'] / res['graph_fp64']['builds_per_s'],
           'energy_error_fixed_density': {
               'what': '1/2 tr(D (dJ - dK/2)), mixed minus FP64, every molecule at its density',
               'fp32_cutoff': args.fp32_cutoff,
               'max_abs_eh': float(np.abs(de_fixed).max()),
               'mean_abs_eh': float(np.abs(de_fixed).mean())}}
    if args.batch_scf > 0:
        out['scf'] = bench_batch_scf(args, mols[:args.batch_scf])
    return out


def bench_batch_scf(args, mols):
    """RHF of molecules of the batched workload through the batched server
    (all requests admitted at once, one batched J/K pass per iteration,
    level shift 0.5 Eh against the oscillations of these random geometries,
    converged when the energy changes by less than 1e-9 Eh), in FP64 and in
    mixed precision: the energy difference of every molecule that converged
    in both."""
    from byteqc_b200.cuobc.scf.serve import JKServer
    res = {}
    for name, cut in (('fp64', None), ('mixed', args.fp32_cutoff)):
        t = time.perf_counter()
        srv = JKServer(n_iter=args.batch_scf_iters, conv_tol=1e-9,
                       fp32_cutoff=cut, max_slots=len(mols),
                       hbm_budget_bytes=150 << 30, level_shift=0.5)
        for m in mols:
            srv.submit(m)
        srv.run_until_empty()
        fin = sorted(srv.finished, key=lambda r: r.rid)
        res[name] = {'wall_s': time.perf_counter() - t, 'steps': srv.steps,
                     'energies': [r.energies[-1] for r in fin],
                     'iterations': [len(r.energies) for r in fin],
                     'conv': [r.converged for r in fin],
                     'converged': sum(1 for r in fin if r.converged)}
    both = np.array(res['fp64']['conv']) & np.array(res['mixed']['conv'])
    de = (np.array(res['mixed']['energies']) - np.array(res['fp64']['energies']))[both]
    return {'molecules': len(mols), 'conv_tol': 1e-9, 'level_shift': 0.5,
            'fp32_cutoff': args.fp32_cutoff,
            'converged_fp64': res['fp64']['converged'],
            'converged_mixed': res['mixed']['converged'],
            'compared': int(both.sum()),
            'max_abs_de': float(np.abs(de).max()) if de.size else None,
            'mean_abs_de': float(np.abs(de).mean()) if de.size else None,
            'de_per_molecule': [float(x) for x in de],
            'iterations_fp64_mean': float(np.mean(res['fp64']['iterations'])),
            'iterations_mixed_mean': float(np.mean(res['mixed']['iterations'])),
            'wall_s_fp64': res['fp64']['wall_s'], 'wall_s_mixed': res['mixed']['wall_s']}


def bench_sweep(args, torch, timed):
    """Mixed-precision sweep on the (H2O)64 / cc-pVDZ workload: for each
    fp32_cutoff the build time, the J/K max-abs error against the FP64
    engine on the workload density, and the converged RHF energy against the
    FP64 RHF energy."""
    from byteqc_b200.cuobc.scf import RHF, hf
    mol, dm = make_workload('h2o64-dz')
    opt = hf._VHFOpt(mol).build()
    d = torch.as_tensor(dm, device='cuda')
    rj, rk = hf.get_jk(mol, d, vhfopt=opt, out='device')
    ms64 = timed(lambda: hf.get_jk(mol, d, vhfopt=opt, out='device'), args.steps)
    t = time.perf_counter()
    mf = RHF(mol)
    mf._opt_gpu = opt
    e64 = mf.kernel()
    scf64 = {'e_tot': e64, 'converged': mf.converged, 'cycles': mf.cycles,
             'jk_builds': mf.jk_builds, 'wall_s': time.perf_counter() - t}
    rows = []
    for cut in args.sweep_cutoffs:
        mj, mk = hf.get_jk(mol, d, vhfopt=opt, out='device', fp32_cutoff=cut)
        err = max((mj - rj).abs().max().item(), (mk - rk).abs().max().item())
        ms = timed(lambda: hf.get_jk(mol, d, vhfopt=opt, out='device',
                                     fp32_cutoff=cut), args.steps)
        t = time.perf_counter()
        mf = RHF(mol, fp32_cutoff=cut)
        mf._opt_gpu = opt
        e = mf.kernel()
        rows.append({'fp32_cutoff': cut, 'ms_per_build': ms,
                     'speedup_vs_fp64': ms64 / ms, 'max_abs_err_jk': err,
                     'scf_de': e - e64, 'converged': mf.converged,
                     'cycles': mf.cycles, 'scf_wall_s': time.perf_counter() - t})
    opt.clear()
    return {'workload': 'h2o64-dz', 'nao': int(mol.nao), 'ms_per_build_fp64': ms64,
            'scf_fp64': scf64, 'rows': rows}


def bench_rhf(args, mol, opt):
    """Full RHF of the headline workload to |dE| < 1e-9 Eh (DIIS,
    incremental Fock builds) in FP64, and in mixed precision at the bench's
    FP32 cutoff: energies, cycles, J/K builds and wall time."""
    from byteqc_b200.cuobc.scf import RHF
    out = {'workload': args.workload, 'conv_tol': 1e-9}
    for name, cut in (('fp64', None), ('mixed', args.fp32_cutoff or None)):
        t = time.perf_counter()
        mf = RHF(mol, fp32_cutoff=cut)
        mf._opt_gpu = opt
        e = mf.kernel()
        out[name] = {'e_tot': e, 'converged': mf.converged, 'cycles': mf.cycles,
                     'jk_builds': mf.jk_builds, 'wall_s': time.perf_counter() - t}
    if out['mixed']['e_tot'] is not None:
        out['de_mixed'] = out['mixed']['e_tot'] - out['fp64']['e_tot']
    return out


def serve_workload(nreq, seed=5, max_nbf=2000, min_nbf=50):
    """Requests of the serving stream: seeded random-walk molecules sized
    log-uniform in [min_nbf, max_nbf] basis functions, the basis drawn from
    6-31G*, cc-pVDZ and def2-TZVP (stand-ins)."""
    from byteqc_b200.gto import Mole, geom
    rng = np.random.default_rng(seed)
    per_atom = {'standin-6-31g*': 8.5, 'standin-cc-pvdz': 9.5,
                'standin-def2-tzvp': 18.5}
    bases = sorted(per_atom)
    mols = []
    for i in range(nreq):
        basis = bases[int(rng.integers(len(bases)))]
        nbf = float(np.exp(rng.uniform(np.log(min_nbf), np.log(max_nbf))))
        natm = max(3, int(round(nbf / per_atom[basis])))
        mols.append(Mole(atom=geom.random_walk_molecule(natm, seed=seed * 7919 + i),
                         basis=basis).build())
    return mols


def bench_serve(args, torch):
    """Continuous-batching server on a Poisson stream: the capacity is
    estimated from one FP64 build of every request alone at its starting
    (core-guess) density (sequential, so a lower bound of the batched
    capacity), then requests arrive at 80 % of that rate, in FP64 and in
    mixed precision; per-build and per-iteration p50/p99 latency,
    per-request latency and builds/s."""
    from byteqc_b200.cuobc.scf.serve import (JKServer, poisson_serve,
                                             single_build_seconds)
    mols = serve_workload(args.serve_requests, max_nbf=args.serve_max_nbf)
    nbf = [m.nao for m in mols]
    kw = dict(n_iter=args.serve_iters)
    # warm-up: one batched pass over every request in both precisions, so
    # that the timed streams do not pay the first (lazy) load of a kernel,
    # its attributes or the allocator's first blocks
    for cut in (None, args.fp32_cutoff):
        warm = JKServer(n_iter=1, fp32_cutoff=cut)
        for m in mols:
            warm.submit(m)
        warm.run_until_empty()
    build_s = sum(single_build_seconds(m) for m in mols)
    cap_builds = len(mols) / build_s
    rate = 0.8 * cap_builds / args.serve_iters  # requests per second
    out = {'requests': len(mols), 'iters_per_request': args.serve_iters,
           'nbf_min': min(nbf), 'nbf_max': max(nbf), 'nbf_median': float(np.median(nbf)),
           'capacity_builds_per_s_sequential': cap_builds,
           'poisson_rate_req_per_s': rate}
    for name, cut in (('fp64', None), ('mixed', args.fp32_cutoff)):
        srv, wall = poisson_serve(mols, rate, seed=5, fp32_cutoff=cut, **kw)
        st = srv.stats()
        st.update(builds_per_s=srv.builds / wall, wall_s=wall)
        if cut:
            st['fp32_cutoff'] = cut
        out[name] = st
    return out


def bench_int4c(args, torch, timed):
    """The dense ERI tensor of (H2O)2 / cc-pVDZ in the working basis through
    int4c.get_int4c (the fill kernels of every class pair plus the eight
    permuted block copies), CUDA-event timed."""
    from byteqc_b200.cuobc.lib import int4c
    from byteqc_b200.cuobc.scf.hf import _VHFOpt
    from byteqc_b200.gto import Mole, geom
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
               basis='standin-cc-pvdz').build()
    opt = _VHFOpt(mol).build(diag_block_with_triu=True)
    int4c.get_int4c(mol, vhfopt=opt)
    ms = timed(lambda: int4c.get_int4c(mol, vhfopt=opt), 2)
    # the fill calls alone: every class pair into a preallocated zeroed block
    from byteqc_b200.cuobc import lib as _lib
    from byteqc_b200.cuobc.scf.hf import _make_s_index_offsets
    lib = _lib.load_library()
    calls = []
    for cp_ij, cp_kl in zip(*np.tril_indices(len(opt.log_qs))):
        si, sj, sk, sl, b = int4c.get_int4c_slice(int(cp_ij), int(cp_kl), opt)
        shp = b.shape
        calls.append((int(cp_ij), int(cp_kl), b,
                      np.array([shp[1] * shp[2] * shp[3], shp[2] * shp[3], shp[3], 1], dtype=np.int32),
                      np.array([si.start, sj.start, sk.start, sl.start], dtype=np.int32),
                      _make_s_index_offsets(opt.log_qs[cp_ij], 1, opt.direct_scf_tol),
                      _make_s_index_offsets(opt.log_qs[cp_kl], 1, opt.direct_scf_tol)))
    stream = torch.cuda.current_stream().cuda_stream

    def fill_calls():
        for cp_ij, cp_kl, b, st, of, bij, bkl in calls:
            _lib.check(lib.jk_fill_int2e(
                opt.handle, ctypes.c_void_p(b.data_ptr()), opt.nao, st.ctypes.data,
                of.ctypes.data, bij.ctypes.data, bkl.ctypes.data, 1, cp_ij, cp_kl,
                ctypes.c_void_p(stream)), 'jk_fill_int2e')
    fill_calls()
    ms_calls = timed(fill_calls, 3)
    n = opt.nao
    npair = n * (n + 1) // 2
    return {'workload': '(H2O)2 standin-cc-pvdz, working basis',
            'nao': n, 'ms': ms, 'fill_calls_ms': ms_calls,
            'class_pairs': len(calls), 'tensor_gb': 8. * n ** 4 / 1e9,
            'unique_integrals_per_s': npair * (npair + 1) // 2 / (ms * 1e-3),
            'tensor_write_gbs': 8. * n ** 4 / (ms * 1e-3) / 1e9}


# even-tempered stand-in auxiliary basis for the density-fitting measurement
# (no fitting basis data is available offline)
DF_AUX = {'O': [[0, [8.0, 1.0]], [0, [2.0, 1.0]], [0, [0.5, 1.0]],
                [1, [3.0, 1.0]], [1, [0.8, 1.0]], [2, [1.5, 1.0]],
                [3, [1.1, 1.0]]],
          'H': [[0, [3.0, 1.0]], [0, [0.6, 1.0]], [1, [1.0, 1.0]]]}


def bench_df(args, torch, timed):
    """Density-fitting integrals of (H2O)8 / cc-pVDZ with the stand-in
    auxiliary basis: every (ij|P) block of int3c.get_int3c plus the metric
    factor of get_int2c, CUDA-event timed."""
    from byteqc_b200.cuobc.lib import int3c
    from byteqc_b200.gto import Mole, geom
    atoms = geom.water_cluster(8, box=9.0, seed=0)
    mol = Mole(atom=atoms, basis='standin-cc-pvdz').build()
    aux = Mole(atom=atoms, basis=DF_AUX).build()
    opt = int3c.VHFOpt3c(mol, aux, 'int3c2e').build()

    def run():
        for cp in range(len(opt.log_qs)):
            for ca in range(len(opt.aux_log_qs)):
                int3c.get_int3c(cp, ca, opt)
        int3c.get_int2c(opt)
    run()
    ms = timed(run, 2)
    nao, naux = int(opt.ao_loc[-1]), int(opt.aux_ao_loc[-1])
    return {'workload': '(H2O)8 standin-cc-pvdz, even-tempered stand-in '
                        'auxiliary basis, working bases',
            'nao': nao, 'naux': naux, 'ms': ms,
            'int3c_per_s': nao * (nao + 1) // 2 * naux / (ms * 1e-3)}


def ncart(l):
    return (l + 1) * (l + 2) // 2


def class_flops(li, lj, lk, ll, nprim_ij, nprim_kl, n_dm=1, with_j=True,
                with_k=True):
    """Algorithmic FLOPs of one contracted quartet of the class: the fixed
    cost model used for the roofline (identical for every engine)."""
    n = (li + lj + lk + ll) // 2 + 1
    nm, mm = li + lj, lk + ll
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    vrr = 4 * nm + 6 * (nm + 1) * mm
    hrr = 2 * sum((nm - j + 1) * (mm + 1) for j in range(1, lj + 1))
    hrr += 2 * (li + 1) * (lj + 1) * sum(mm - l + 1 for l in range(1, ll + 1))
    per_root = 56 + 20 + 3 * (vrr + hrr) + 3 * nf
    prim = 30 + n * per_root
    dig = (4 * nf if with_j else 0) + (8 * nf if with_k else 0)
    return nprim_ij * nprim_kl * prim + dig * n_dm


class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons while running."""

    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._th = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ['nvidia-smi', '-i', str(self.index),
                     '--query-gpu=' + self.FIELDS,
                     '--format=csv,noheader,nounits'],
                    capture_output=True, text=True, timeout=5).stdout
                self.samples.append([v.strip() for v in out.split(',')])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._th = threading.Thread(target=self._run, daemon=True)
        self._th.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [],
                    'samples': 0}
        sm = [float(s[0]) for s in self.samples if s[0].replace('.', '').isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.strip().lower() == 'active':
                    reasons.add(n)
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': max(mx) if mx else None,
                'reasons': sorted(reasons), 'samples': len(self.samples)}


def cpu_baseline(mol, dm, target_s=15.0, opt=None, repeats=1):
    """Oracle J/K on all host cores over a uniform subsample of ij rows
    (rows ij = stride/2 mod stride of every class pair), scaled to one full
    build by exact quartet counts: a count-only pass gives the quartets of
    the full build and the build's fixed cost (density transforms, final
    contraction), the sample its time per quartet.  Returns (builds/s, info)."""
    from oracle import hf_oracle
    if opt is None:
        opt = hf_oracle.VHFOpt(mol).build()
    st = {}
    hf_oracle.get_jk(mol, dm, vhfopt=opt, count_only=True, stats=st)  # warm-up
    t = time.perf_counter()
    hf_oracle.get_jk(mol, dm, vhfopt=opt, count_only=True, stats=st)
    fixed = time.perf_counter() - t
    total = st['quartets']

    def sample(stride):
        s2 = {}
        t = time.perf_counter()
        hf_oracle.get_jk(mol, dm, vhfopt=opt, ij_stride=stride,
                         ij_offset=stride // 2, stats=s2)
        return time.perf_counter() - t, s2['quartets']
    # calibration: quadruple the sample until its work beyond the fixed cost
    # reaches a quarter of the target (the samples grow geometrically, so the
    # calibration costs about a third of the final sample)
    stride = 1 << 14
    while True:
        dt, q = sample(stride)
        if stride == 1 or dt - fixed >= 0.25 * target_s:
            break
        stride = max(1, stride // 4)
    vals = []
    for _ in range(repeats):
        dt, q = sample(stride)
        # per-quartet time from the sample beyond the fixed cost; when the
        # sample is too small to separate them, its whole time per quartet
        work = dt - fixed if dt > 2 * fixed else dt
        est = (fixed if dt > 2 * fixed else 0.) + work * total / max(q, 1)
        vals.append(1.0 / est)
    cores = int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1))
    info = {'cores': cores, 'stride': stride, 'sample_s': dt,
            'sample_quartets': q, 'total_quartets': total,
            'fixed_s': fixed, 'est_build_s': est}
    return (vals if repeats > 1 else vals[0]), info


def run_reference(args):
    """The reference arm, rank 0 only.  ``value``: the oracle (a port of the
    reference's algorithm for this path; the reference has no CPU J/K of its
    own) on all host cores, every step one bounded sample of the build
    scaled by quartet count.  ``reference_gpu``: the reference's own kernels
    (cuobc gint/gvhf compiled unmodified for sm_100a into oracle/_ref)
    through its GINTbuild_jk task loop on the same workload and GPU, in a
    child process.  No engine library is loaded on this arm."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    mol, dm = make_workload(args.workload, oracle_overlap=True)
    vals, info = cpu_baseline(mol, dm, target_s=args.ref_sample_s,
                              repeats=args.warmup + args.steps)
    vals = vals if isinstance(vals, list) else [vals]
    value = float(np.median(vals[args.warmup:] or vals))
    line = {
        'impl': 'reference', 'metric': 'jk_builds_per_s', 'value': value,
        'unit': 'builds/s', 'n_gpus': args.gpus, 'steps': args.steps,
        'warmup': args.warmup, 'higher_is_better': True, 'dtype': 'f64',
        'data': 'synthetic', 'scaling': 'weak',
        'config': {'workload': args.workload},
        'cpu_baseline': {
            'value': value, 'unit': 'builds/s', 'cores': info['cores'],
            'kind': 'port',
            'sample': ('oracle J/K on every %d-th shell-pair row of each class pair (%d of %d quartets, %.1f s of CPU work), scaled to one build by quartet count'
                       % (info['stride'], info['sample_quartets'],
                          info['total_quartets'], info['sample_s']))},
        'e2e': {'value': value, 'unit': 'builds/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    if not args.no_reference_gpu:
        line['reference_gpu'] = reference_gpu(args, mol, dm)
        if not args.no_int4c:
            line['reference_gpu_int4c'] = reference_gpu_int4c()
    print(json.dumps(line))


def reference_gpu_int4c():
    """The reference's get_int4c flow with its own GINTfill_int2e kernels
    on this GPU, on the workload of the int4c section ((H2O)2 / cc-pVDZ
    stand-in, working basis), in a child process; the set-up (groups, pair
    lists, Schwarz values) is the oracle's restatement of _VHFOpt.build."""
    from oracle import hf_oracle, ref_jk
    from byteqc_b200.gto import Mole, geom
    if not ref_jk.available():
        return {'unavailable': 'oracle/_ref not built'}
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
               basis='standin-cc-pvdz').build()
    ropt = hf_oracle.VHFOpt(mol).build(diag_block_with_triu=True)
    try:
        info = ref_jk.run('get_int4c_timing', ropt)
    except Exception as e:
        return {'unavailable': str(e)[-300:]}
    n = info['nao']
    info.update(workload='(H2O)2 standin-cc-pvdz, working basis',
                tensor_write_gbs=8. * n ** 4 / (info['ms'] * 1e-3) / 1e9,
                what='cuobc/lib/int4c.py get_int4c flow over GINTfill_int2e '
                     '(compiled unmodified for sm_100a)')
    return info


def reference_gpu(args, mol, dm):
    """The reference's own J/K kernels on this GPU (same workload, FP64):
    CUDA events around its whole GINTbuild_jk task loop, density already on
    the device, task bins precomputed; no L2 flush between builds."""
    from oracle import ref_jk
    if not ref_jk.available():
        return {'unavailable': 'oracle/_ref not built (the reference sources '
                               'were absent at build time)'}
    reps = max(1, min(args.steps, 5))
    try:
        _, _, info = ref_jk.run('get_jk', mol, dm, timing=(2, reps))
    except Exception as e:  # reported, not fatal: the CPU arm stands
        return {'unavailable': str(e)[-300:]}
    ms = info['ms_per_build']
    return {'ms_per_build': ms, 'builds_per_s': 1e3 / ms, 'builds_timed': reps,
            'class_pair_calls': info['launch_calls'], 'nbins': info['nbins'],
            'what': 'ByteQC cuobc gint/gvhf kernels compiled unmodified for '
                    'sm_100a (oracle/ref/Makefile), GINTbuild_jk per class '
                    'pair as cuobc/scf/hf.py:get_jk calls it; AO transforms '
                    'not included'}


def profile_builds(args, torch, lib):
    """jk_build of the workload density in the working basis, repeated (for
    ncu launch lists and captures); prints nothing but a line count."""
    import ctypes
    from byteqc_b200.cuobc import lib as jklib
    from byteqc_b200.cuobc.scf import hf
    mol, dm = make_workload(args.workload)
    opt = hf._VHFOpt(mol).build()
    nao = opt.coeff.shape[0]
    C = opt.coeff_dev
    w = (C @ torch.as_tensor(dm, device='cuda') @ C.T).contiguous()
    vj = torch.zeros(nao, nao, dtype=torch.float64, device='cuda')
    vk = torch.zeros_like(vj)
    o = jklib.JKOpts()
    o.direct_scf_tol = opt.direct_scf_tol
    o.nbins = opt.default_nbins()
    o.prescreen = 1
    o.fp32_cutoff = args.fp32_cutoff if '--fp32-cutoff' in sys.argv else 0.
    for _ in range(args.profile_builds):
        jklib.check(lib.jk_build(opt.handle, w.data_ptr(), 1, vj.data_ptr(),
                                 vk.data_ptr(), ctypes.byref(o), None), 'jk_build')
    torch.cuda.synchronize()
    print('profile builds done: %d x %s' % (args.profile_builds, args.workload))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='h2o32-tzvp', choices=sorted(WORKLOADS))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-int4c', action='store_true',
                    help='skip the ERI-tensor fill and density-fitting measurements')
    ap.add_argument('--profile-fill', type=int, default=0,
                    help='only run this many get_int4c calls of the (H2O)2 / '
                         'cc-pVDZ ERI-tensor workload and exit (ncu target)')
    ap.add_argument('--profile-builds', type=int, default=0,
                    help='only run this many jk_build calls of the workload '
                         '(FP64, or mixed with --fp32-cutoff > 0 given '
                         'explicitly) and exit: the command profiled by ncu')
    ap.add_argument('--ref-sample-s', type=float, default=4.0)
    ap.add_argument('--no-reference-gpu', action='store_true',
                    help='reference arm: skip timing the reference kernels')
    ap.add_argument('--batch-mols', type=int, default=256,
                    help='molecules of the batched workload (0: skip)')
    ap.add_argument('--batch-steps', type=int, default=1,
                    help='timed repetitions of each batched variant')
    ap.add_argument('--batch-scf', type=int, default=0,
                    help='molecules of the batched workload run to SCF '
                         'convergence in FP64 and mixed (0: skip; the '
                         'random-walk geometries converge poorly)')
    ap.add_argument('--batch-scf-iters', type=int, default=50,
                    help='iteration cap of those SCF runs')
    ap.add_argument('--no-rhf', action='store_true',
                    help='skip the full RHF of the headline workload')
    ap.add_argument('--no-sweep', action='store_true',
                    help='skip the mixed-precision cutoff sweep with SCF energies')
    ap.add_argument('--sweep-cutoffs', type=float, nargs='*',
                    default=[1e-8, 1e-7, 1e-6, 1e-5, 1e-4])
    ap.add_argument('--serve-requests', type=int, default=8,
                    help='requests of the serving stream (0: skip)')
    ap.add_argument('--serve-iters', type=int, default=15)
    ap.add_argument('--serve-max-nbf', type=int, default=2000,
                    help='largest request in basis functions (2000 for the '
                         'full 50-2000 range)')
    ap.add_argument('--fp32-cutoff', type=float, default=1e-6,
                    help='also time the mixed-precision build at this cutoff '
                         '(0: skip)')
    args = ap.parse_args()
    if args.impl == 'reference':
        return run_reference(args)

    import torch
    from byteqc_b200.cuobc import lib as jklib
    from byteqc_b200.cuobc.scf import hf

    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))

    lib = jklib.load_library()
    if args.profile_builds > 0:
        return profile_builds(args, torch, lib)
    if args.profile_fill > 0:
        from byteqc_b200.cuobc.lib import int4c
        from byteqc_b200.gto import Mole, geom
        fmol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
                    basis='standin-cc-pvdz').build()
        fopt = hf._VHFOpt(fmol).build(diag_block_with_triu=True)
        for _ in range(args.profile_fill):
            int4c.get_int4c(fmol, vhfopt=fopt)
        torch.cuda.synchronize()
        print('profile fill done: %d x (H2O)2 / cc-pVDZ' % args.profile_fill)
        return
    mol, dm = make_workload(args.workload)
    t = time.perf_counter()
    opt = hf._VHFOpt(mol).build()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t
    nao, nao0 = opt.coeff.shape
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    d_dm = torch.as_tensor(dm, device='cuda').reshape(1, nao0, nao0).contiguous()
    d_vj = torch.empty_like(d_dm)
    d_vk = torch.empty_like(d_dm)
    opts = jklib.JKOpts()
    opts.direct_scf_tol = opt.direct_scf_tol
    opts.nbins = opt.default_nbins()
    opts.prescreen = 1
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device='cuda')

    def step_device():
        jklib.check(lib.jk_get_jk(opt.handle, opt.coeff_dev.data_ptr(), nao0,
                                  d_dm.data_ptr(), 1, d_vj.data_ptr(),
                                  d_vk.data_ptr(), ctypes.byref(opts), sptr),
                    'jk_get_jk')

    # working-basis density for the kernel-only timing
    C = opt.coeff_dev
    d_w = (C @ d_dm[0] @ C.T).contiguous()
    w_vj = torch.zeros(nao, nao, dtype=torch.float64, device='cuda')
    w_vk = torch.zeros_like(w_vj)

    def step_kernels():
        jklib.check(lib.jk_build(opt.handle, d_w.data_ptr(), 1,
                                 w_vj.data_ptr(), w_vk.data_ptr(),
                                 ctypes.byref(opts), sptr), 'jk_build')

    def timed(fn, n):
        tot = 0.
        for _ in range(n):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / n

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_step = timed(step_device, args.steps)
        ms_kern = timed(step_kernels, args.steps)
    torch.cuda.synchronize()
    # end-to-end through the public call: host numpy in, host numpy out
    for _ in range(1):
        hf.get_jk(mol, dm, vhfopt=opt)

    def step_e2e():
        hf.get_jk(mol, dm, vhfopt=opt)
    ms_e2e = timed(step_e2e, max(2, args.steps // 2))
    # mixed precision: same build with FP32 recursion below fp32_cutoff
    ms_mixed = None
    mixed_err = None
    if args.fp32_cutoff > 0:
        ref_j, ref_k = d_vj.clone(), d_vk.clone()
        opts.fp32_cutoff = args.fp32_cutoff
        for _ in range(2):
            step_device()
        ms_mixed = timed(step_device, args.steps)
        mixed_err = max((d_vj - ref_j).abs().max().item(),
                        (d_vk - ref_k).abs().max().item())
        opts.fp32_cutoff = 0.
    if dist:
        t = torch.tensor([ms_step, ms_kern, ms_e2e, ms_mixed or 0.], device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step, ms_kern, ms_e2e, mm = t.tolist()
        ms_mixed = mm if ms_mixed is not None else None

    # quartet counts and the FLOP model
    info = np.zeros(7, dtype=np.int32)
    lib.jk_basis_info(opt.handle, info.ctypes.data)
    ncq = int(info[6])
    cq = np.zeros((max(ncq, 1), 8), dtype=np.int32)
    lib.jk_basis_cq_info(opt.handle, cq.ctypes.data)
    counts2 = np.zeros(2 * max(ncq, 1), dtype=np.int64)
    lib.jk_last_counts(opt.handle, counts2.ctypes.data, sptr)
    counts = counts2[:ncq] + counts2[ncq:2 * ncq]
    quartets = int(counts[:ncq].sum())
    flops = sum(int(c) * class_flops(*(int(v) for v in cq[i, 2:8]))
                for i, c in enumerate(counts[:ncq]) if c)
    # one FP64 atomic per element of the six J/K blocks of every quartet
    atomics = 0
    for i, c in enumerate(counts[:ncq]):
        fi, fj, fk, fl = (ncart(int(v)) for v in cq[i, 2:6])
        atomics += int(c) * (fi * fj + fk * fl + fi * fk + fi * fl + fj * fk
                             + fj * fl)
    peak = ctypes.c_double()
    lib.jk_fma_peak(0, ctypes.byref(peak))
    peak32 = ctypes.c_double()
    lib.jk_fma_peak(1, ctypes.byref(peak32))
    achieved = flops / (ms_kern * 1e-3) / 1e12
    # the last build was the mixed one when it ran: its FP32 share of quartets
    f32_share = float(counts2[ncq:2 * ncq].sum()) / max(1, quartets)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    line = {
        'metric': 'jk_builds_per_s',
        'value': world * 1e3 / ms_step,
        'unit': 'builds/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': args.workload,
                   'molecule': ('random walk, %d atoms' % WORKLOADS[args.workload][1]
                                if WORKLOADS[args.workload][0] == 'walk'
                                else '(H2O)%d' % WORKLOADS[args.workload][0]),
                   'basis': WORKLOADS[args.workload][3],
                   'nao': int(nao0), 'nao_working': int(nao),
                   'parallelism': 'replicas' if world > 1 else 'single',
                   'l2': 'flushed (512 MiB write) before every timed step',
                   'direct_scf_tol': opt.direct_scf_tol,
                   'nbins': int(opts.nbins)},
        'quartets_per_build': quartets,
        'quartets_per_s': world * quartets / (ms_step * 1e-3),
        'kernel_ms_per_build': ms_kern,
        'atomics_per_build': atomics,
        'setup_s': setup_s,
        # dm_cond + screen + one launch per class quartet + 2 symmetrize
        'gpu_launches': 4 + ncq,
        'roofline': {'bound': 'fp64', 'achieved': achieved,
                     'peak': peak.value, 'unit': 'TFLOP/s',
                     'frac': achieved / peak.value if peak.value else None,
                     'peak_source': 'measured FP64 FMA-chain kernel '
                                    '(jk_fma_peak) in this process',
                     'flops_per_build': flops,
                     'traffic': PROFILED_TRAFFIC.get(args.workload),
                     'traffic_unit': 'DRAM bytes per build (class launches)',
                     'traffic_source': 'ncu dram__bytes_read.sum + dram__bytes_write.sum '
                                       'of `bench.py --profile-builds 2` '
                                       '(profiles/jk_build_launches_h2o32-tzvp.txt)',
                     'algorithmic_bytes_per_build': 3 * 8 * int(nao) ** 2},
        'e2e': {'value': world * 1e3 / ms_e2e, 'unit': 'builds/s',
                'h2d_bytes_per_step': int(dm.nbytes),
                'd2h_bytes_per_step': int(2 * dm.nbytes)},
        'clocks': clk.summary(),
    }
    if not args.no_rhf and world == 1:
        line['rhf'] = bench_rhf(args, mol, opt)
    if args.batch_mols > 0 and world == 1:
        line['batch'] = bench_batch(args, torch, timed)
    if not args.no_sweep and world == 1:
        line['sweep'] = bench_sweep(args, torch, timed)
    if args.serve_requests > 0 and world == 1:
        line['serve'] = bench_serve(args, torch)
    if not args.no_int4c and world == 1:
        line['int4c'] = bench_int4c(args, torch, timed)
        line['df'] = bench_df(args, torch, timed)
    if ms_mixed is not None:
        line['mixed'] = {'fp32_cutoff': args.fp32_cutoff,
                         'value': world * 1e3 / ms_mixed, 'unit': 'builds/s',
                         'ms_per_step': ms_mixed,
                         'speedup_vs_fp64': ms_step / ms_mixed,
                         'max_abs_err_jk': mixed_err,
                         'fp32_quartet_share': f32_share,
                         'achieved_tflops': flops / (ms_mixed * 1e-3) / 1e12,
                         'peak_fp32_tflops': peak32.value}
    if world == 1 and not args.no_cpu_baseline:
        v, inf = cpu_baseline(mol, dm)
        line['cpu_baseline'] = {
            'value': v, 'unit': 'builds/s', 'cores': inf['cores'],
            'kind': 'port',
            'sample': ('oracle J/K on every %d-th shell-pair row of each class pair (%d of %d quartets, %.1f s of CPU work), scaled to one build by quartet count'
                       % (inf['stride'], inf['sample_quartets'],
                          inf['total_quartets'], inf['sample_s']))}
    print(json.dumps(line, default=float))
    if dist:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
