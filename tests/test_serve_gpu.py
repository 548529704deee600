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
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.cuobc.scf.serve import JKServer, footprint_bytes
    mols = [_mol(5, 20 + i, 'standin-cc-pvdz') for i in range(4)]
    need = max(footprint_bytes(hf._VHFOpt(m).build()) for m in mols)
    srv = JKServer(hbm_budget_bytes=int(2.5 * need), n_iter=3)
    for m in mols:
        srv.submit(m)
    peak = 0
    while srv.waiting or srv.active:
        srv.step()
        peak = max(peak, len(srv.active) + (1 if srv.finished else 0))
        assert srv.used <= srv.budget
    assert len(srv.finished) == 4
