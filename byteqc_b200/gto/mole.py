"""Minimal molecule object in the libcint ``atm/bas/env`` layout.

The J/K path of the reference takes a PySCF ``Mole`` (``cuobc/scf/hf.py:53``)
and reads ``_atm``, ``_bas``, ``_env``, ``ao_loc``, ``cart`` and
``cart2sph_coeff()`` from it (``hf.py:71,114,481-564``).  PySCF is not a
dependency of this package, so this module provides the subset of that object
the path needs, with the same slot layout (``cuobc/lib/gint/gint.h:29-46``)
and the same normalisation conventions:

* primitive radial normalisation ``gto_norm(l, a) = 1/sqrt(int r^(2l+2)
  exp(-2 a r^2) dr)`` folded into the stored contraction coefficients, and
  each contracted radial function normalised to one;
* Cartesian components ``x^a y^b z^c`` carry no per-component factor; the
  s/p common factors 1/sqrt(4 pi) and sqrt(3/(4 pi)) are applied by the
  integral code (``cuobc/lib/gint/pair_data.c:27-28``);
* spherical functions are real solid harmonics ``r^l Y_lm`` ordered
  m = -l..l (p functions stay x, y, z), built from the closed formula for
  real solid harmonics and normalised on the unit sphere.
"""
import math

import numpy as np

# atm slots
CHARGE_OF = 0
PTR_COORD = 1
NUC_MOD_OF = 2
PTR_ZETA = 3
ATM_SLOTS = 6
# bas slots
ATOM_OF = 0
ANG_OF = 1
NPRIM_OF = 2
NCTR_OF = 3
KAPPA_OF = 4
PTR_EXP = 5
PTR_COEFF = 6
BAS_SLOTS = 8
PTR_ENV_START = 20

BOHR = 0.52917721092  # Angstrom per Bohr

ELEMENTS = ['X', 'H', 'He', 'Li', 'Be', 'B', 'C', 'N', 'O', 'F', 'Ne',
            'Na', 'Mg', 'Al', 'Si', 'P', 'S', 'Cl', 'Ar']
CHARGE = {s: i for i, s in enumerate(ELEMENTS)}
ANGULAR = 'spdfghik'


def charge(symb):
    return CHARGE[symb[0].upper() + symb[1:].lower()]


def gaussian_int(n, alpha):
    """int_0^inf x^n exp(-alpha x^2) dx."""
    n1 = (n + 1) * .5
    return math.gamma(n1) / (2. * alpha ** n1)


def gto_norm(l, expnt):
    """Radial normalisation of r^l exp(-a r^2)."""
    expnt = np.asarray(expnt, dtype=np.float64)
    n1 = (2 * l + 3) * .5
    return 1. / np.sqrt(math.gamma(n1) / (2. * (2. * expnt) ** n1))


def normalize_contracted(l, es, cs):
    """Fold primitive norms into ``cs`` (nprim, nctr) and normalise every
    contracted radial function to one."""
    es = np.asarray(es, dtype=np.float64)
    cs = np.asarray(cs, dtype=np.float64).reshape(len(es), -1)
    cs = cs * gto_norm(l, es)[:, None]
    ee = es[:, None] + es[None, :]
    n1 = (2 * l + 3) * .5
    ovlp = np.array([[math.gamma(n1) / (2. * e ** n1) for e in row]
                     for row in ee])
    s1 = 1. / np.sqrt(np.einsum('pi,pq,qi->i', cs, ovlp, cs))
    return cs * s1[None, :]


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nsph(l):
    return 2 * l + 1


def cart_powers(l):
    """libcint Cartesian order: lx descending, then ly descending."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def _solid_harmonic(l, m):
    """Coefficients {(a, b, c): coef} of the real solid harmonic S_lm
    (normalised as r^l sqrt(4 pi/(2l+1)) Y_lm) over monomials x^a y^b z^c.

    Closed formula for real solid harmonics: a triple sum over t, u, v with
    coefficients (-1)^(t+v-vm) 4^-t C(l,t) C(l-t,|m|+t) C(t,u) C(|m|,2v).
    """
    am = abs(m)
    vm = 0. if m >= 0 else .5
    nrm = (1. / (2 ** am * math.factorial(l))) * math.sqrt(
        2. * math.factorial(l + am) * math.factorial(l - am)
        / (2. if m == 0 else 1.))
    terms = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            v = vm
            vmax = math.floor(am / 2. - vm) + vm
            while v <= vmax + 1e-9:
                two_v = int(round(2 * v))
                sgn = (-1) ** int(round(t + v - vm))
                coef = (sgn * .25 ** t * math.comb(l, t)
                        * math.comb(l - t, am + t) * math.comb(t, u)
                        * math.comb(am, two_v))
                a = 2 * t + am - 2 * u - two_v
                b = 2 * u + two_v
                c = l - 2 * t - am
                if coef != 0:
                    key = (a, b, c)
                    terms[key] = terms.get(key, 0.) + nrm * coef
                v += 1.
    return terms


_C2S_CACHE = {}


def cart2sph(l):
    """(ncart(l), nsph(l)) transform; columns are spherical functions."""
    if l in _C2S_CACHE:
        return _C2S_CACHE[l]
    if l == 0:
        c = np.ones((1, 1))
    elif l == 1:
        c = np.eye(3)
    else:
        pows = cart_powers(l)
        index = {p: i for i, p in enumerate(pows)}
        c = np.zeros((ncart(l), nsph(l)))
        fac = math.sqrt((2 * l + 1) / (4 * math.pi))
        for im, m in enumerate(range(-l, l + 1)):
            for key, v in _solid_harmonic(l, m).items():
                c[index[key], im] += v * fac
    _C2S_CACHE[l] = c
    return c


class Mole:
    """Molecule with a Gaussian basis.

    ``atom``: list of (symbol, (x, y, z)) in ``unit`` (Angstrom default).
    ``basis``: dict symbol -> list of shells ``[l, [exp, c1, c2, ...], ...]``
    (the PySCF internal format), or a name accepted by
    :func:`byteqc_b200.gto.basis.load`.
    """

    def __init__(self, atom=None, basis=None, cart=False, unit='Angstrom',
                 charge=0, spin=0, verbose=0):
        self.atom = atom or []
        self.basis = basis
        self.cart = cart
        self.unit = unit
        self.charge = charge
        self.spin = spin
        self.verbose = verbose
        self._atm = np.zeros((0, ATM_SLOTS), dtype=np.int32)
        self._bas = np.zeros((0, BAS_SLOTS), dtype=np.int32)
        self._env = np.zeros(PTR_ENV_START)
        self._built = False

    # -- construction -----------------------------------------------------
    def build(self):
        from byteqc_b200.gto import basis as basis_mod
        atoms = self.atom
        if isinstance(atoms, str):
            atoms = _parse_atom_string(atoms)
        scale = 1. / BOHR if self.unit.lower().startswith('a') else 1.
        env = [0.] * PTR_ENV_START
        atm = []
        for symb, xyz in atoms:
            ptr = len(env)
            env.extend([float(v) * scale for v in xyz])
            env.append(0.)  # zeta slot for a point nucleus
            atm.append([charge(symb), ptr, 1, ptr + 3, 0, 0])
        basis = self.basis
        if isinstance(basis, str):
            basis = {s: basis for s, _ in atoms}
        shells_by_symb = {}
        bas = []
        for ia, (symb, _) in enumerate(atoms):
            key = symb
            if key not in shells_by_symb:
                spec = basis.get(symb, basis.get(
                    symb[0].upper() + symb[1:].lower()))
                if spec is None:
                    raise KeyError('no basis for element %s' % symb)
                if isinstance(spec, str):
                    spec = basis_mod.load(spec, symb)
                rows = []
                for shell in spec:
                    l = int(shell[0])
                    prim = np.asarray(shell[1:], dtype=np.float64)
                    es = prim[:, 0]
                    cs = normalize_contracted(l, es, prim[:, 1:])
                    pexp = len(env)
                    env.extend(es.tolist())
                    pcoeff = len(env)
                    env.extend(cs.T.ravel().tolist())
                    rows.append([0, l, len(es), cs.shape[1], 0, pexp,
                                 pcoeff, 0])
                shells_by_symb[key] = rows
            for row in shells_by_symb[key]:
                r = list(row)
                r[ATOM_OF] = ia
                bas.append(r)
        self._atm = np.asarray(atm, dtype=np.int32).reshape(-1, ATM_SLOTS)
        self._bas = np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS)
        self._env = np.asarray(env, dtype=np.float64)
        self._atom_symbols = [s for s, _ in atoms]
        self._built = True
        return self

    # -- geometry / size --------------------------------------------------
    @property
    def natm(self):
        return len(self._atm)

    @property
    def nbas(self):
        return len(self._bas)

    def atom_coords(self):
        ptr = self._atm[:, PTR_COORD]
        return np.stack([self._env[ptr], self._env[ptr + 1],
                         self._env[ptr + 2]], axis=1)

    def atom_charges(self):
        return self._atm[:, CHARGE_OF].astype(np.int64)

    def atom_symbol(self, ia):
        return self._atom_symbols[ia]

    @property
    def nelectron(self):
        return int(self.atom_charges().sum()) - self.charge

    def ao_loc_nr(self, cart=None):
        if cart is None:
            cart = self.cart
        l = self._bas[:, ANG_OF]
        nf = (l + 1) * (l + 2) // 2 if cart else 2 * l + 1
        return np.append(0, np.cumsum(nf * self._bas[:, NCTR_OF])).astype(
            np.int32)

    @property
    def ao_loc(self):
        return self.ao_loc_nr()

    @property
    def nao(self):
        return int(self.ao_loc_nr()[-1])

    def nao_nr(self, cart=None):
        return int(self.ao_loc_nr(cart)[-1])

    def aoslice_by_atom(self):
        ao_loc = self.ao_loc_nr()
        out = np.zeros((self.natm, 4), dtype=np.int64)
        atom_of = self._bas[:, ATOM_OF]
        for ia in range(self.natm):
            idx = np.where(atom_of == ia)[0]
            if idx.size:
                b0, b1 = idx[0], idx[-1] + 1
            else:
                b0 = b1 = out[ia - 1, 1] if ia else 0
            out[ia] = (b0, b1, ao_loc[b0], ao_loc[b1])
        return out

    def bas_angular(self, ib):
        return int(self._bas[ib, ANG_OF])

    def bas_exp(self, ib):
        p = self._bas[ib, PTR_EXP]
        return self._env[p:p + self._bas[ib, NPRIM_OF]]

    def bas_ctr_coeff(self, ib):
        """(nprim, nctr) stored coefficients (primitive norms included)."""
        p = self._bas[ib, PTR_COEFF]
        npr, nct = self._bas[ib, NPRIM_OF], self._bas[ib, NCTR_OF]
        return self._env[p:p + npr * nct].reshape(nct, npr).T

    def cart2sph_coeff(self):
        """Block-diagonal (nao_cart, nao_sph) transform over all shells."""
        ao_c = self.ao_loc_nr(cart=True)
        ao_s = self.ao_loc_nr(cart=False)
        c = np.zeros((ao_c[-1], ao_s[-1]))
        for ib in range(self.nbas):
            l = self._bas[ib, ANG_OF]
            blk = cart2sph(l)
            i0, j0 = ao_c[ib], ao_s[ib]
            for ic in range(self._bas[ib, NCTR_OF]):
                c[i0 + ic * ncart(l):i0 + (ic + 1) * ncart(l),
                  j0 + ic * nsph(l):j0 + (ic + 1) * nsph(l)] = blk
        return c

    def intor(self, name):
        """One-electron integrals 'int1e_ovlp', 'int1e_kin', 'int1e_nuc'
        in this molecule's basis (host code in libjk.so)."""
        import ctypes
        from byteqc_b200.cuobc import lib as jklib
        which = {'int1e_ovlp': 0, 'int1e_kin': 1, 'int1e_nuc': 2}[name]
        n = self.nao_nr(cart=True)
        out = np.zeros((n, n))
        atm = np.ascontiguousarray(self._atm, dtype=np.int32)
        bas = np.ascontiguousarray(self._bas, dtype=np.int32)
        env = np.ascontiguousarray(self._env)
        rc = jklib.load_library().jk_int1e_cart(
            which, atm.ctypes.data, self.natm, bas.ctypes.data, self.nbas,
            env.ctypes.data, out.ctypes.data)
        if rc:
            raise RuntimeError('jk_int1e_cart failed with status %d' % rc)
        if not self.cart:
            c = self.cart2sph_coeff()
            out = c.T @ out @ c
        return out

    def energy_nuc(self):
        z = self.atom_charges().astype(np.float64)
        r = self.atom_coords()
        e = 0.
        for i in range(self.natm):
            for j in range(i):
                e += z[i] * z[j] / np.linalg.norm(r[i] - r[j])
        return e

    def copy(self):
        m = Mole.__new__(Mole)
        m.__dict__.update(self.__dict__)
        m._atm = self._atm.copy()
        m._bas = self._bas.copy()
        m._env = self._env.copy()
        return m


def conc_mol(m1, m2):
    """One molecule holding the atoms and shells of ``m1`` followed by those
    of ``m2`` (PySCF's gto.conc_mol): ``m2``'s atom indices and environment
    pointers are shifted past ``m1``'s."""
    m = m1.copy()
    off = len(m1._env)
    atm2 = m2._atm.copy()
    atm2[:, PTR_COORD] += off
    atm2[:, PTR_ZETA] += off
    bas2 = m2._bas.copy()
    bas2[:, ATOM_OF] += m1.natm
    bas2[:, PTR_EXP] += off
    bas2[:, PTR_COEFF] += off
    m._atm = np.vstack([m1._atm, atm2]).astype(np.int32)
    m._bas = np.vstack([m1._bas, bas2]).astype(np.int32)
    m._env = np.concatenate([m1._env, m2._env])
    m.cart = m1.cart
    return m


def _parse_atom_string(s):
    out = []
    for line in s.replace(';', '\n').splitlines():
        tok = line.split()
        if len(tok) >= 4:
            out.append((tok[0], tuple(float(v) for v in tok[1:4])))
    return out


def M(atom, basis, **kw):
    return Mole(atom=atom, basis=basis, **kw).build()
