"""ERI tensor fill (jk_fill_int2e through byteqc_b200.cuobc.lib.int4c, the
counterpart of the reference's int4c.get_int4c) against the oracle's shell
quartets.  Tolerance: 1e-10 max-abs (relative to max(1, max|block|)); the
fill screens quartets below the Schwarz cutoff (1e-13), which the oracle's
direct blocks keep, so the bar is set above that."""
import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _blocks(pm):
    ao = pm.ao_loc_nr(cart=True)
    return [slice(ao[i], ao[i + 1]) for i in range(pm.nbas)]


def test_int4c_full_tensor_vs_oracle():
    """Every shell quartet of one water in the cc-pVDZ stand-in."""
    import oracle
    from oracle import hf_oracle
    from byteqc_b200.cuobc.lib import int4c
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=2),
               basis='standin-cc-pvdz').build()
    eri = int4c.get_int4c(mol).cpu().numpy()
    pm = hf_oracle.VHFOpt(mol).build().mol
    sl = _blocks(pm)
    n = pm.nbas
    assert eri.shape == (pm.ao_loc_nr(cart=True)[-1],) * 4
    # the eight permutations agree, so the canonical quartets i >= j,
    # k >= l, (ij) >= (kl) cover the tensor
    assert abs(eri - eri.transpose(1, 0, 2, 3)).max() <= 1e-14
    assert abs(eri - eri.transpose(0, 1, 3, 2)).max() <= 1e-14
    assert abs(eri - eri.transpose(2, 3, 0, 1)).max() <= 1e-14
    worst = 0.
    for i in range(n):
        for j in range(i + 1):
            for k in range(i + 1):
                for l in range((j if k == i else k) + 1):
                    ref = oracle.eri_shells(pm, i, j, k, l)
                    got = eri[sl[i], sl[j], sl[k], sl[l]]
                    worst = max(worst, abs(got - ref).max() / max(1., abs(ref).max()))
    assert worst <= TOL, worst


def test_int4c_g_h_shells_vs_oracle():
    """A water with added g and h shells: random shell quartets of the
    tensor (all classes up to (hh|hh) go through the fill kernel)."""
    import oracle
    from oracle import hf_oracle
    from byteqc_b200.cuobc.lib import int4c
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]]], 'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
           for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=2), basis=bas).build()
    eri = int4c.get_int4c(mol).cpu().numpy()
    pm = hf_oracle.VHFOpt(mol).build().mol
    sl = _blocks(pm)
    ls = pm._bas[:, 1]
    rng = np.random.default_rng(11)
    hi = np.flatnonzero(ls >= 4)
    quartets = [tuple(int(x) for x in rng.integers(0, pm.nbas, 4)) for _ in range(150)]
    quartets += [(int(hi[-1]), int(hi[-1]), int(hi[-1]), int(hi[-1])),
                 (int(hi[0]), int(hi[-1]), 0, int(hi[-1]))]
    for q in quartets:
        ref = oracle.eri_shells(pm, *q)
        got = eri[sl[q[0]], sl[q[1]], sl[q[2]], sl[q[3]]]
        err = abs(got - ref).max() / max(1., abs(ref).max())
        assert err <= TOL, (q, err)
