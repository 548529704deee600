"""The oracle itself (CPU, no GPU): pinned against an independent integral
algorithm (Obara-Saika / Head-Gordon-Pople on scipy's Boys function,
oracle/eri_os.py), a closed form, a brute-force contraction of the full ERI
tensor, and the committed golden J/K fixtures (tests/golden)."""
import math
import os

import numpy as np
import pytest

from byteqc_b200.gto import Mole, geom

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'golden_jk.npz')


def _pmol(nw, basis, box, seed):
    from oracle import hf_oracle
    mol = Mole(atom=geom.water_cluster(nw, box=box, seed=seed),
               basis=basis).build()
    return hf_oracle.VHFOpt(mol).build().mol


def test_ss_closed_form():
    """(s_A s_A | s_B s_B) of single s primitives: with p = q = 2a,
    (c f)^4 2 pi^2.5 / (p q sqrt(p+q)) F0(T), T = a |AB|^2 and
    F0(T) = sqrt(pi/T) erf(sqrt T) / 2 (c the stored coefficient, f the
    libcint s-factor)."""
    import oracle
    from oracle import eri_os
    mol = Mole(atom=[('H', (0., 0., 0.)), ('H', (0., 0., 0.9))],
               basis={'H': [[0, [1.3, 1.0]]]}, cart=True).build()
    a = 1.3
    A, B = mol.atom_coords()
    c = mol.bas_ctr_coeff(0)[0, 0]
    p = q = 2 * a
    T = p * q / (p + q) * float(np.dot(A - B, A - B))
    f0 = math.sqrt(math.pi / T) * math.erf(math.sqrt(T)) / 2
    ref = (c * eri_os.FAC_SP[0]) ** 4 * 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * f0
    got = oracle.eri_shells(mol, 0, 0, 1, 1)[0, 0, 0, 0]
    assert abs(got - ref) <= 1e-14 * abs(ref)


def test_rys_quadrature_exact_on_moments():
    """sum_r w_r t_r^(2k) = F_k(x) for k < 2n (the Rys rule integrates the
    Boys moments exactly), n = 1..13 on x in [0, 120]."""
    import oracle
    from oracle.eri_os import boys
    for n in range(1, 14):
        for x in (0.0, 0.3, 1.7, 6.0, 25.0, 60.0, 119.0):
            s, w = oracle.rys_roots(n, x)
            for k in range(2 * n):
                lhs = float(np.sum(w * s ** k))
                rhs = boys(k, x)
                assert abs(lhs - rhs) <= 1e-12 * max(abs(rhs), 1e-30) + 1e-300, (n, x, k)


def test_eri_vs_obara_saika():
    """Contracted Cartesian shell quartets up to (ff|ff) from the oracle's Rys
    engine against Obara-Saika."""
    import oracle
    from oracle import eri_os
    pm = _pmol(1, 'standin-def2-tzvp', 4.0, 1)
    rng = np.random.default_rng(0)
    ls = pm._bas[:, 1]
    by_l = {l: np.flatnonzero(ls == l) for l in range(4)}
    picks = [(3, 3, 3, 3), (3, 2, 1, 0), (2, 2, 2, 1), (1, 1, 1, 1), (3, 0, 2, 0)]
    for lq in picks:
        sh = [int(rng.choice(by_l[l])) for l in lq]
        a = oracle.eri_shells(pm, *sh)
        b = eri_os.eri_shells(pm, *sh)
        assert a.shape == b.shape
        # relative to the block's largest element, with an absolute floor for
        # blocks that vanish by symmetry (one-centre, odd total parity)
        assert abs(a - b).max() <= 1e-12 * abs(b).max() + 1e-14, lq


def test_eri_vs_obara_saika_g_h():
    """Quartets with g and h shells (the classes of the generic GPU kernel):
    the oracle's Rys engine against Obara-Saika."""
    import oracle
    from oracle import eri_os
    from oracle import hf_oracle
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]],
                   [4, [3.0, 0.6], [0.7, 0.5]]],
             'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
           for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=2), basis=bas).build()
    pm = hf_oracle.VHFOpt(mol).build().mol
    rng = np.random.default_rng(0)
    ls = pm._bas[:, 1]
    by_l = {l: np.flatnonzero(ls == l) for l in (0, 1, 2, 4, 5)}
    picks = [(4, 0, 0, 0), (5, 1, 2, 0), (4, 4, 1, 0), (5, 4, 2, 2),
             (5, 5, 1, 1)]
    for lq in picks:
        sh = [int(rng.choice(by_l[l])) for l in lq]
        a = oracle.eri_shells(pm, *sh)
        b = eri_os.eri_shells(pm, *sh)
        assert a.shape == b.shape
        assert abs(a - b).max() <= 1e-12 * abs(b).max() + 1e-14, lq


def test_eri_vs_obara_saika_every_class():
    """The oracle against Obara-Saika on every class up to (ff|ff) (one
    random quartet each) and on a seeded sample of the g/h classes including
    (hh|hh).  Blocks that vanish by symmetry agree to an absolute 1e-13."""
    import oracle
    from oracle import eri_os
    from oracle import hf_oracle
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]]], 'H': [[4, [0.8, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-def2-tzvp', s)) + extra[s]
           for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=2), basis=bas).build()
    pm = hf_oracle.VHFOpt(mol).build().mol
    ls = pm._bas[:, 1]
    by_l = {l: np.flatnonzero(ls == l) for l in range(6)}
    rng = np.random.default_rng(3)
    pairs = [(a, b) for a in range(6) for b in range(a + 1)]
    classes = [(a, b, c, d) for i, (a, b) in enumerate(pairs)
               for (c, d) in pairs[:i + 1]]
    low = [q for q in classes if max(q) <= 3]
    high = [q for q in classes if max(q) >= 4 and sum(q) <= 12]
    picks = low + [high[i] for i in rng.choice(len(high), 16, replace=False)]
    picks.append((5, 5, 5, 5))
    assert len(low) == 55
    for lq in picks:
        sh = [int(rng.choice(by_l[l])) for l in lq]
        a = oracle.eri_shells(pm, *sh)
        b = eri_os.eri_shells(pm, *sh)
        assert abs(a - b).max() <= 1e-12 * abs(b).max() + 1e-13, lq


def _boys_series(m, x, digits=130):
    """F_m(x) = e^-x sum_k (2x)^k / ((2m+1)(2m+3)...(2m+2k+1)), summed in
    decimal arithmetic with enough digits for the cancellation at x = 200."""
    from decimal import Decimal, getcontext
    getcontext().prec = digits
    X = Decimal(repr(float(x)))
    term = Decimal(1) / Decimal(2 * m + 1)
    tot = term
    k = 0
    while True:
        k += 1
        term = term * 2 * X / Decimal(2 * m + 2 * k + 1)
        tot += term
        if term < tot * Decimal(10) ** (-40):
            break
    return float(tot * (-X).exp())


def test_boys_vs_high_precision_series():
    """The Boys function used as the reference of the Rys moment test
    against a high-precision series, m = 0..12, x in [0, 200]."""
    from oracle.eri_os import boys
    for m in range(13):
        for x in (0.0, 1e-3, 0.3, 1.0, 4.7, 12.0, 33.0, 60.0, 119.0, 200.0):
            ref = _boys_series(m, x)
            got = boys(m, x)
            assert abs(got - ref) <= 1e-13 * ref, (m, x, got, ref)


def _shifted(atoms, shift=(0., 0., 0.), rot=None):
    out = []
    for sym, xyz in atoms:
        v = np.asarray(xyz, dtype=float)
        if rot is not None:
            v = rot @ v
        out.append((sym, tuple(v + np.asarray(shift))))
    return out


def test_eri_symmetry_and_invariance():
    """Contracted shell quartets of the oracle: the 8-fold permutation
    symmetry, invariance under a translation of the molecule, and the
    transformation of a (pp|pp) block under a rotation."""
    import oracle
    from oracle import hf_oracle
    atoms = geom.water_cluster(2, box=4.0, seed=2)

    def pmol(at):
        mol = Mole(atom=at, basis='standin-def2-tzvp').build()
        return hf_oracle.VHFOpt(mol).build().mol
    pm = pmol(atoms)
    pt = pmol(_shifted(atoms, shift=(1.3, -0.7, 2.1)))
    ls = pm._bas[:, 1]
    rng = np.random.default_rng(5)
    by_l = {l: np.flatnonzero(ls == l) for l in range(4)}
    for lq in [(3, 2, 1, 0), (2, 1, 2, 1), (1, 1, 0, 0), (3, 3, 1, 1)]:
        i, j, k, l = [int(rng.choice(by_l[x])) for x in lq]
        a = oracle.eri_shells(pm, i, j, k, l)
        tol = 1e-13 * abs(a).max() + 1e-15
        assert abs(a - oracle.eri_shells(pm, j, i, k, l).transpose(1, 0, 2, 3)).max() <= tol
        assert abs(a - oracle.eri_shells(pm, i, j, l, k).transpose(0, 1, 3, 2)).max() <= tol
        assert abs(a - oracle.eri_shells(pm, k, l, i, j).transpose(2, 3, 0, 1)).max() <= tol
        assert abs(a - oracle.eri_shells(pt, i, j, k, l)).max() <= 1e-12 * abs(a).max() + 1e-15
    # rotation: Cartesian p components transform as vectors
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0.], [np.sin(th), np.cos(th), 0.], [0., 0., 1.]])
    ax = np.array([1., 2., 2.]) / 3.
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = R @ (np.eye(3) + np.sin(0.4) * K + (1 - np.cos(0.4)) * K @ K)
    pr = pmol(_shifted(atoms, rot=R))
    p_sh = by_l[1]
    i, j, k, l = (int(p_sh[0]), int(p_sh[-1]), int(p_sh[1]), int(p_sh[-2]))
    a = oracle.eri_shells(pm, i, j, k, l)
    b = oracle.eri_shells(pr, i, j, k, l)
    ra = np.einsum('ai,bj,ck,dl,ijkl->abcd', R, R, R, R, a)
    assert abs(ra - b).max() <= 1e-12 * abs(a).max()


def test_jk_linearity_and_symmetry():
    """Oracle J/K as operators: J(D) and K(D) symmetric for symmetric D,
    linear in D, and tr(D1 J(D2)) = tr(D2 J(D1)) (likewise K)."""
    from oracle import hf_oracle
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=3),
               basis='standin-cc-pvdz').build()
    opt = hf_oracle.VHFOpt(mol).build()
    rng = np.random.default_rng(9)
    d = rng.random((2, mol.nao, mol.nao))
    d = d + d.transpose(0, 2, 1)
    dm = np.stack([d[0], d[1], 0.3 * d[0] - 1.7 * d[1]])
    vj, vk = hf_oracle.get_jk(mol, dm, vhfopt=opt)
    sc = max(abs(vj).max(), abs(vk).max())
    for v in (vj, vk):
        assert abs(v - v.transpose(0, 2, 1)).max() <= 1e-12 * sc
        assert abs(v[2] - (0.3 * v[0] - 1.7 * v[1])).max() <= 1e-11 * sc
        t12 = np.sum(d[0] * v[1])
        t21 = np.sum(d[1] * v[0])
        assert abs(t12 - t21) <= 1e-11 * abs(t12)


def test_jk_vs_full_eri_tensor():
    """Oracle get_jk (screened, binned, 8-fold symmetric loop) against J and K
    contracted from the full ERI tensor of the working basis."""
    import oracle
    from oracle import hf_oracle
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=2),
               basis='standin-cc-pvdz').build()
    opt = hf_oracle.VHFOpt(mol).build()
    pm, C = opt.mol, opt.coeff
    ao = pm.ao_loc_nr(cart=True)
    n = ao[-1]
    eri = np.zeros((n, n, n, n))
    for i in range(pm.nbas):
        for j in range(pm.nbas):
            for k in range(pm.nbas):
                for l in range(pm.nbas):
                    eri[ao[i]:ao[i + 1], ao[j]:ao[j + 1], ao[k]:ao[k + 1],
                        ao[l]:ao[l + 1]] = oracle.eri_shells(pm, i, j, k, l)
    rng = np.random.default_rng(4)
    d = rng.random((mol.nao, mol.nao))
    d = d + d.T
    w = C @ d @ C.T
    rj = C.T @ np.einsum('ijkl,kl->ij', eri, w) @ C
    rk = C.T @ np.einsum('ikjl,kl->ij', eri, w) @ C
    vj, vk = hf_oracle.get_jk(mol, d, vhfopt=opt)
    assert abs(vj - rj).max() <= 1e-11 * abs(rj).max()
    assert abs(vk - rk).max() <= 1e-11 * abs(rk).max()


@pytest.mark.parametrize('case', ['h2o-dz', 'h2o2-tzvp', 'walk6-631gs'])
def test_oracle_reproduces_golden(case):
    """The oracle against the committed fixtures (regression pin; the
    fixtures and their generator are in tests/golden)."""
    from oracle import hf_oracle
    from tests.golden.make_golden import case_inputs
    g = np.load(GOLDEN)
    mol, dm = case_inputs(case)
    vj, vk = hf_oracle.get_jk(mol, dm)
    np.testing.assert_allclose(vj, g[case + '/vj'], rtol=0, atol=1e-12)
    np.testing.assert_allclose(vk, g[case + '/vk'], rtol=0, atol=1e-12)


def test_basis_conventions_independent_of_product():
    """The oracle's radial normalisation and Cartesian-to-spherical matrix
    (oracle/gto_oracle.py: scipy's gamma function and spherical harmonics)
    against the product's (byteqc_b200.gto.mole: closed-form solid
    harmonics) for l = 0..6; the two are derived independently, so a wrong
    matrix or norm cannot cancel between the engine and the oracle."""
    from byteqc_b200.gto import mole
    from oracle import gto_oracle
    for l in range(7):
        np.testing.assert_allclose(gto_oracle.cart2sph(l), mole.cart2sph(l),
                                   rtol=0, atol=5e-14)
        e = np.array([0.07, 0.9, 13.0, 4000.0])
        np.testing.assert_allclose(gto_oracle.gto_norm(l, e),
                                   mole.gto_norm(l, e), rtol=1e-14)


@pytest.mark.parametrize('basis', ['standin-cc-pvdz', 'standin-def2-tzvp',
                                   'standin-6-31g*', 'i-shells'])
def test_contracted_spherical_overlap_is_normalised(basis):
    """Every contracted spherical function has unit norm under the oracle's
    own overlap integrals (Obara-Saika, jk_oracle.c) and transforms, and the
    overlap matrix equals the product's one-electron code; also for a basis
    with g, h and i shells."""
    from oracle import gto_oracle
    if basis == 'i-shells':
        from byteqc_b200.gto import basis as basis_mod
        extra = {'O': [[4, [1.1, 1.0]], [5, [0.9, 1.0]],
                       [6, [2.5, 0.7], [0.6, 0.5]]],
                 'H': [[6, [0.9, 1.0]]]}
        basis = {s: list(basis_mod.load('standin-cc-pvdz', s)) + extra[s]
                 for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(2, box=5.0, seed=0),
               basis=basis).build()
    s = gto_oracle.overlap(mol)
    assert abs(np.diag(s) - 1).max() < 1e-13
    # (i shells: the two recursions round differently at about 1e-13)
    np.testing.assert_allclose(s, mol.intor('int1e_ovlp'), rtol=0, atol=5e-13)


@pytest.mark.parametrize('basis', ['standin-cc-pvdz', 'standin-def2-tzvp',
                                   'standin-6-31g*'])
def test_pair_data_matches_reference_cache(basis):
    """The oracle's primitive-pair table (a12, e12, product centres, the
    0.5 diagonal factor) is identical, bit for bit, to the one the
    reference's own GINTinit_basis_prod_cpu (cuobc/lib/gint/pair_data.c,
    compiled unmodified into oracle/_ref/) builds from the same pair lists;
    host code only, no GPU."""
    import ctypes
    import oracle
    from oracle import hf_oracle, ref_jk
    if not ref_jk.available():
        pytest.skip('oracle/_ref not built (needs the reference sources)')
    gint, _ = ref_jk.libs()
    mol = Mole(atom=geom.water_cluster(3, box=6.0, seed=2),
               basis=basis).build()
    for triu in (False, True):
        opt = hf_oracle.VHFOpt(mol).build(diag_block_with_triu=triu)
        pmol = opt.mol
        atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
        bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
        env = np.ascontiguousarray(pmol._env)
        p2s = np.ascontiguousarray(opt.bas_pair2shls, dtype=np.int32)
        locs = np.ascontiguousarray(opt.bas_pairs_locs, dtype=np.int32)
        ncp = len(opt.log_qs)
        coords = np.empty(pmol.nbas * 3)
        cache = ctypes.POINTER(ref_jk.BasisProdCache)()
        P = ref_jk._ptr
        gint.GINTinit_basis_prod_cpu(
            ctypes.byref(cache), ctypes.c_double(opt.diag_fac), P(coords),
            P(p2s), P(locs), ctypes.c_int(ncp), P(atm),
            ctypes.c_int(pmol.natm), P(bas), ctypes.c_int(pmol.nbas), P(env))
        c = cache.contents
        n = c.primitive_pairs_locs[ncp]
        ref = np.ctypeslib.as_array(c.aexyz, (n * 5,)).copy()
        for k in range(ncp):
            t = c.cptype[k]
            i, j = p2s[0, locs[k]], p2s[1, locs[k]]
            assert (t.l_bra, t.l_ket) == (pmol._bas[i, 1], pmol._bas[j, 1])
            assert t.npairs == locs[k + 1] - locs[k]
        mine = np.zeros(n * 5)
        lib = oracle.lib()
        lib.oracle_pair_data.restype = ctypes.c_long
        got = lib.oracle_pair_data(
            P(atm), P(bas), P(env), ctypes.c_int(pmol.nbas),
            P(np.ascontiguousarray(p2s[0])), P(np.ascontiguousarray(p2s[1])),
            ctypes.c_int(p2s.shape[1]), ctypes.c_double(opt.diag_fac),
            P(mine), ctypes.c_long(n * 5))
        assert got == n
        np.testing.assert_array_equal(mine, ref)
        gint.GINTdel_basis_prod(ctypes.byref(cache))


def test_eri_vs_obara_saika_i_shells():
    """Quartets with i shells (l = 6; the reference hands these to PySCF on
    the CPU, the engine runs them in its generic GPU kernel with up to 13
    Rys roots): the oracle's Rys engine against Obara-Saika."""
    import oracle
    from oracle import eri_os
    from oracle import hf_oracle
    from byteqc_b200.gto import basis as basis_mod
    extra = {'O': [[6, [1.3, 1.0]], [6, [2.5, 0.7], [0.6, 0.5]]],
             'H': [[6, [0.9, 1.0]]]}
    bas = {s: list(basis_mod.load('standin-6-31g*', s)) + extra[s]
           for s in ('O', 'H')}
    mol = Mole(atom=geom.water_cluster(1, box=4.0, seed=3), basis=bas).build()
    pm = hf_oracle.VHFOpt(mol).build().mol
    rng = np.random.default_rng(1)
    ls = pm._bas[:, 1]
    by_l = {l: np.flatnonzero(ls == l) for l in (0, 1, 2, 6)}
    for lq in [(6, 0, 0, 0), (6, 1, 1, 0), (6, 2, 0, 0), (6, 6, 0, 0),
               (6, 0, 6, 0)]:
        sh = [int(rng.choice(by_l[l])) for l in lq]
        a = oracle.eri_shells(pm, *sh)
        b = eri_os.eri_shells(pm, *sh)
        assert a.shape == b.shape
        assert abs(a - b).max() <= 1e-12 * abs(b).max() + 1e-14, lq
