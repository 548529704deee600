"""Generates golden_jk.npz: J and K of seeded small inputs computed by the
oracle (the CPU restatement of the reference's get_jk).  The reference has no
J/K golden vectors of its own (its tests print sums only) and cannot run in
this container, so these fixtures pin the oracle against regressions and give
the GPU tests a fixed target.

    python -m tests.golden.make_golden
"""
import os

import numpy as np

from byteqc_b200.gto import Mole, geom

CASES = ('h2o-dz', 'h2o2-tzvp', 'walk6-631gs')


def case_inputs(case):
    """(mol, dm) of a fixture case: seeded geometry, seeded symmetric dm."""
    if case == 'h2o-dz':
        mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=0),
                   basis='standin-cc-pvdz').build()
    elif case == 'h2o2-tzvp':
        mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=1),
                   basis='standin-def2-tzvp').build()
    elif case == 'walk6-631gs':
        mol = Mole(atom=geom.random_walk_molecule(6, seed=2),
                   basis='standin-6-31g*').build()
    else:
        raise KeyError(case)
    s = mol.intor('int1e_ovlp')
    dm = geom.scf_like_density(s, nocc=mol.nelectron // 2, seed=3)
    return mol, dm


def main():
    from oracle import hf_oracle
    out = {}
    for case in CASES:
        mol, dm = case_inputs(case)
        vj, vk = hf_oracle.get_jk(mol, dm)
        out[case + '/vj'] = vj
        out[case + '/vk'] = vk
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden_jk.npz')
    np.savez_compressed(path, **out)
    print('wrote', path, {k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main()
