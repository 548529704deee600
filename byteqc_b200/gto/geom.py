"""Seeded synthetic geometries and densities for the J/K workloads.

* :func:`water_cluster` -- rigid waters (r_OH 0.957 A, HOH 104.5 deg) with
  random orientations, oxygens placed by seeded rejection sampling in a cube
  with O-O >= 2.6 A.  The reference benchmarks J/K on water clusters
  (``cuobc/test/jk.py:27-7807``, ``cuobc/test/scf.py:22-120``); these are
  seeded stand-ins of the same kind.
* :func:`random_walk_molecule` -- atoms grown by a seeded random walk, each
  bonded to a random earlier atom at 0.95-1.55 A and at least 1.2 A from
  all others, elements drawn C:N:O:H = 3:1:1:5.
* :func:`scf_like_density` -- D = 2 C C^T with C (nao, nocc) from a seeded
  normal matrix orthonormalised in the overlap metric (C^T S C = 1).
"""
import numpy as np

R_OH = 0.957
THETA_HOH = np.deg2rad(104.5)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster(nwater, box=9.0, seed=0, min_oo=2.6, max_tries=200000):
    """List of (symbol, xyz in Angstrom) for ``nwater`` waters."""
    rng = np.random.default_rng(seed)
    h1 = np.array([R_OH, 0., 0.])
    h2 = R_OH * np.array([np.cos(THETA_HOH), np.sin(THETA_HOH), 0.])
    oxy = []
    tries = 0
    while len(oxy) < nwater:
        tries += 1
        if tries > max_tries:
            raise RuntimeError('cannot pack %d waters in a %.1f A cube'
                               % (nwater, box))
        p = rng.uniform(0., box, size=3)
        if all(np.linalg.norm(p - o) >= min_oo for o in oxy):
            oxy.append(p)
    atoms = []
    for o in oxy:
        rot = _random_rotation(rng)
        atoms.append(('O', tuple(o)))
        atoms.append(('H', tuple(o + rot @ h1)))
        atoms.append(('H', tuple(o + rot @ h2)))
    return atoms


ELEMENT_WEIGHTS = (('C', 3), ('N', 1), ('O', 1), ('H', 5))


def random_walk_molecule(natm, seed=0, bond=(0.95, 1.55), min_dist=1.2,
                         max_tries=100000):
    rng = np.random.default_rng(seed)
    symbs = [s for s, w in ELEMENT_WEIGHTS for _ in range(w)]
    heavy = [s for s in symbs if s != 'H']
    pos = [np.zeros(3)]
    elems = [heavy[rng.integers(len(heavy))]]
    tries = 0
    while len(pos) < natm:
        tries += 1
        if tries > max_tries:
            raise RuntimeError('random walk stuck at %d atoms' % len(pos))
        anchor = pos[rng.integers(len(pos))]
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        p = anchor + v * rng.uniform(*bond)
        if all(np.linalg.norm(p - q) >= min_dist for q in pos):
            pos.append(p)
            elems.append(symbs[rng.integers(len(symbs))])
    # closed shell: the electron count must be even
    z = {'H': 1, 'C': 6, 'N': 7, 'O': 8}
    if sum(z[e] for e in elems) % 2:
        for i in range(len(elems) - 1, -1, -1):
            if elems[i] == 'H':
                elems[i] = 'C' if len(elems) > 1 else 'N'
                break
        else:
            elems[-1] = 'N' if elems[-1] != 'N' else 'O'
        if sum(z[e] for e in elems) % 2:
            elems[-1] = {'C': 'N', 'N': 'C', 'O': 'N', 'H': 'C'}[elems[-1]]
    return [(e, tuple(p)) for e, p in zip(elems, pos)]


def scf_like_density(s, nocc, seed=1):
    """D = 2 C C^T with C^T S C = 1 for a seeded normal C (nao, nocc)."""
    rng = np.random.default_rng(seed)
    nao = s.shape[0]
    c = rng.normal(size=(nao, nocc))
    m = c.T @ s @ c
    lo = np.linalg.cholesky(m)
    c = np.linalg.solve(lo, c.T).T
    return 2. * c @ c.T
