"""Worker of the sharded get_jk test (launched by torch.distributed.run,
two ranks on one GPU with the gloo backend): each rank builds its share of
the class quartets, the partial J/K are all-reduced, and every rank checks
the result against the unsharded build at 1e-10."""
import datetime
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    import torch.distributed as dist
    from byteqc_b200.cuobc.scf import hf
    from byteqc_b200.gto import Mole, geom
    torch.cuda.set_device(0)
    dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=120))
    rank = dist.get_rank()
    mol = Mole(atom=geom.water_cluster(4, box=6.5, seed=7),
               basis='standin-def2-tzvp').build()
    s = mol.intor('int1e_ovlp')
    dm = geom.scf_like_density(s, nocc=mol.nelectron // 2, seed=2)
    dm2 = np.stack([dm, 0.3 * dm])
    opt = hf._VHFOpt(mol).build()
    for d, kw in ((dm, {}), (dm2, {}), (dm, {'fp32_cutoff': 1e-6}),
                  (dm, {'with_k': False})):
        vj, vk = hf.get_jk(mol, d, vhfopt=opt, group=dist.group.WORLD, **kw)
        rj, rk = hf.get_jk(mol, d, vhfopt=opt, **kw)
        for a, b in ((vj, rj), (vk, rk)):
            if b is None:
                assert a is None
                continue
            err = abs(a - b).max()
            assert err <= 1e-10, (rank, kw, err)
    dist.barrier()
    dist.destroy_process_group()
    print('rank %d ok' % rank)


if __name__ == '__main__':
    main()
