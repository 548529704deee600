"""Continuous batching: a request's SCF energies are the same when it runs
alone and when it shares the GPU with requests that arrive while it runs;
admission respects the device-memory budget."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu


def _mol(n, seed, basis):
    return Mole(atom=geom.random_walk_molecule(n, seed=seed), basis=basis).build()


def test_result_same_alone_and_in_the_mix():
    from byteqc_b200.cuobc.scf.serve import JKServer
    a = _mol(6, 11, 'standin-6-31g*')
    others = [_mol(4, 12, 'standin-cc-pvdz'), _mol(8, 13, 'standin-6-31g*'),
              _mol(3, 14, 'standin-def2-tzvp')]
    alone = JKServer(n_iter=6)
    alone.submit(a)
    alone.run_until_empty()
    e_alone = alone.finished[0].energies

    mix = JKServer(n_iter=6)
    mix.submit(others[0])
    mix.step()
    ra = mix.submit(a)          # arrives while others[0] is running
    mix.step()
    mix.submit(others[1])
    mix.step()
    mix.submit(others[2])
    mix.run_until_empty()
    req = [r for r in mix.finished if r.rid == ra][0]
    assert len(req.energies) == len(e_alone)
    assert max(abs(x - y) for x, y in zip(req.energies, e_alone)) < 1e-9
    st = mix.stats()
    assert st['requests'] == 4 and st['builds'] == 24


def test_admission_by_memory_budget():
    """Admission bounds each request's footprint from its basis before
    anything is allocated (a request is admitted when the exact footprint of
    the active ones plus its own bound fits): with room for little more than
    one bound, one request runs at a time, the device budget is never
    exceeded, and no basis handle is built for a request that waits."""
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.serve import JKServer, footprint_bound_bytes
    mols = [_mol(5, 20 + i, 'standin-cc-pvdz') for i in range(4)]
    need = max(footprint_bound_bytes(m) for m in mols)
    built = []
    orig = hf._VHFOpt.build

    def counting_build(self, *a, **k):
        built.append(self)
        return orig(self, *a, **k)
    hf._VHFOpt.build = counting_build
    try:
        srv = JKServer(hbm_budget_bytes=int(1.2 * need), n_iter=3)
        for m in mols:
            srv.submit(m)
        while srv.waiting or srv.active:
            srv.step()
            assert len(srv.active) <= 1
            assert len(built) == len(srv.active) + len(srv.finished)
            assert srv.used <= srv.budget
    finally:
        hf._VHFOpt.build = orig
    assert len(srv.finished) == 4


def test_scf_to_convergence_and_batch_reuse():
    """conv_tol ends a request once its energy change is below it; the final
    energy equals the RHF driver's; the engine batch is rebuilt only when
    the set of active requests changes."""
    from byteqc_b200.cuobc.scf import RHF
    from byteqc_b200.cuobc.scf.serve import JKServer
    mols = [Mole(atom=geom.water_cluster(n, box=5.0, seed=30 + n),
                 basis='standin-6-31g*').build() for n in (1, 2)]
    srv = JKServer(n_iter=60, conv_tol=1e-10)
    for m in mols:
        srv.submit(m)
    srv.run_until_empty()
    assert all(r.converged for r in srv.finished)
    assert srv.batch_builds < srv.steps
    for r in srv.finished:
        mf = RHF(r.mol)
        e = mf.kernel()
        assert abs(r.energies[-1] - e) < 1e-8, (r.energies[-1], e)
    st = srv.stats()
    assert st['iteration_p50_ms'] >= st['build_p50_ms'] * 0.5
