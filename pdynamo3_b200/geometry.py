"""Seeded synthetic geometries for the benchmark and test workloads (coordinates in angstroms).

* Water clusters: rigid waters (O-H 0.9572 A, H-O-H 104.52 deg); oxygen positions uniform in a
  cube by seeded rejection sampling with a minimum O-O distance of 2.6 A; orientations from
  uniformly random unit quaternions.
* Organic molecules: seed-grown random saturated trees of C/N/O heavy atoms (70/15/15), valences
  filled with hydrogen, tetrahedral angles, uniform torsions, bond lengths C-C 1.53, C-N 1.47,
  C-O 1.43, C-H 1.09, N-H 1.01, O-H 0.96 A; nonbonded pairs closer than 1.0 A are rejected (a new
  torsion is drawn for a clashing atom, then the whole molecule is regrown).
"""
import numpy as np

SYMBOLS = {1: "H", 6: "C", 7: "N", 8: "O"}
NUMBERS = {v: k for k, v in SYMBOLS.items()}


def _rotation(q):
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster(n_waters, box, seed):
    """Return (atomic_numbers, coordinates[A]) for a rigid-water cluster (O, H, H per water)."""
    rng = np.random.default_rng(seed)
    oxygens = []
    while len(oxygens) < n_waters:
        p = rng.uniform(0.0, box, 3)
        if all(np.linalg.norm(p - q) >= 2.6 for q in oxygens):
            oxygens.append(p)
    r, th = 0.9572, np.deg2rad(104.52)
    local = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0], [r * np.cos(th), r * np.sin(th), 0.0]])
    z, xyz = [], []
    for p in oxygens:
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        xyz.extend(local @ _rotation(q).T + p)
        z.extend([8, 1, 1])
    return np.array(z, dtype=np.int32), np.array(xyz)


_VALENCE = {6: 4, 7: 3, 8: 2}
_BOND = {(6, 6): 1.53, (6, 7): 1.47, (6, 8): 1.43, (7, 7): 1.45, (7, 8): 1.40, (8, 8): 1.48,
         (1, 6): 1.09, (1, 7): 1.01, (1, 8): 0.96}
_TETRA = np.deg2rad(109.4712206)


def _bond(a, b):
    return _BOND[(min(a, b), max(a, b))]


def _place(rng, xyz, i, j, k, length):
    """New atom bonded to i, with angle j-i-new tetrahedral and a uniform torsion about (k, j, i)."""
    bc = xyz[i] - xyz[j]
    bc /= np.linalg.norm(bc)
    ref = xyz[k] - xyz[j] if k is not None else rng.normal(size=3)
    n = np.cross(ref, bc)
    if np.linalg.norm(n) < 1e-8:
        n = np.cross(bc, [1.0, 0.0, 0.0]) if abs(bc[0]) < 0.9 else np.cross(bc, [0.0, 1.0, 0.0])
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    tor = rng.uniform(-np.pi, np.pi)
    d = np.array([-length * np.cos(_TETRA), length * np.sin(_TETRA) * np.cos(tor), length * np.sin(_TETRA) * np.sin(tor)])
    return xyz[i] + d[0] * bc + d[1] * m + d[2] * n


def organic_molecule(n_heavy, seed, max_tries=200):
    """Return (atomic_numbers, coordinates[A]) of a random saturated tree molecule."""
    rng = np.random.default_rng(seed)
    for _ in range(max_tries):
        kinds = rng.choice([6, 7, 8], size=n_heavy, p=[0.70, 0.15, 0.15])
        z = [int(kinds[0])]
        xyz = [np.zeros(3)]
        parent = [-1]
        free = [_VALENCE[z[0]]]
        ok = True
        for a in range(1, n_heavy):
            cands = [i for i in range(len(z)) if free[i] > 0 and z[i] != 1]
            # an atom with one bond left can only be a leaf: keep at least one open site overall
            if not cands:
                ok = False
                break
            elem = int(kinds[a])
            if elem == 8 and len(cands) == 1 and free[cands[0]] == 1 and a < n_heavy - 1:
                elem = 6
            i = int(rng.choice(cands))
            j = parent[i] if parent[i] >= 0 else None
            for _t in range(_PLACE_TRIES):
                if j is None:
                    pos = xyz[i] + _bond(z[i], elem) * _unit(rng)
                else:
                    k = parent[j] if parent[j] >= 0 else None
                    pos = _place(rng, np.array(xyz), i, j, k, _bond(z[i], elem))
                if _fits(xyz, pos, i):
                    break
            z.append(elem)
            xyz.append(pos)
            parent.append(i)
            free[i] -= 1
            free.append(_VALENCE[elem] - 1)
        if not ok:
            continue
        heavy = len(z)
        for i in range(heavy):
            for _h in range(free[i]):
                j = parent[i] if parent[i] >= 0 else None
                if j is None:
                    # first heavy atom with no parent: use any bonded child as reference
                    kids = [c for c in range(heavy) if parent[c] == i]
                    j = kids[0] if kids else None
                for _t in range(_PLACE_TRIES):
                    if j is None:
                        pos = xyz[i] + _bond(z[i], 1) * _unit(rng)
                    else:
                        pos = _place(rng, np.array(xyz), i, j, None, _bond(z[i], 1))
                    if _fits(xyz, pos, i):
                        break
                z.append(1)
                xyz.append(pos)
                parent.append(i)
        xyz = np.array(xyz)
        if _clash_free(z, xyz, parent):
            return np.array(z, dtype=np.int32), xyz
    raise RuntimeError("could not grow a clash-free molecule")


_PLACE_TRIES = 30


def _fits(xyz, pos, bonded_to):
    """True when pos is at least 1.0 A from every placed atom except the one it is bonded to (a new
    random torsion is drawn otherwise, so molecules that grow without clashes are unchanged)."""
    for a, q in enumerate(xyz):
        if a != bonded_to and np.linalg.norm(np.asarray(q) - pos) < 1.0:
            return False
    return True


def _unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def _clash_free(z, xyz, parent):
    n = len(z)
    bonded = set()
    for i, p in enumerate(parent):
        if p >= 0:
            bonded.add((min(i, p), max(i, p)))
    d = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=-1)
    for i in range(n):
        for j in range(i):
            if (j, i) not in bonded and d[i, j] < 1.0:
                return False
    return True


def write_xyz(path, z, xyz, title="generated"):
    with open(path, "w") as f:
        f.write("%d\n%s\n" % (len(z), title))
        for a, r in zip(z, xyz):
            f.write("%s %.10f %.10f %.10f\n" % (SYMBOLS[int(a)], r[0], r[1], r[2]))
