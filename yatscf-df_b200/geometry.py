"""Synthetic molecular geometries used by the benchmarks and tests.

* water: O at the origin, H at (0, +/-0.757, 0.587) Angstrom.
* alkane(n): all-trans linear C_nH_(2n+2), C-C 1.54 A, C-H 1.09 A (or as given),
  exact tetrahedral angles, zig-zag in the xz-plane, centred at the origin.
* water_cluster(seed): 2..32 molecules (count from the seed), random rigid
  rotations (unit quaternions) and translations in a cube of 30 A^3 per
  molecule, rejection until every O-O distance is >= 2.6 A.
Coordinates are in Angstrom; write_xyz() writes the reference's .xyz format
(atom count, net charge on the comment line, then "El x y z").
"""
import math

import numpy as np

TET = math.acos(-1.0 / 3.0)                 # 109.4712 degrees


def water():
    return [("O", 0.0, 0.0, 0.0), ("H", 0.0, 0.757, 0.587), ("H", 0.0, -0.757, 0.587)]


def alkane(n, cc=1.54, ch=1.09):
    half = TET / 2.0
    dx = cc * math.sin(half)                 # C-C projection on the chain axis
    dz = cc * math.cos(half)                 # zig-zag amplitude
    x0 = -0.5 * dx * (n - 1)
    cs = [(x0 + k * dx, 0.0, (dz / 2.0) * (1 if k % 2 == 0 else -1)) for k in range(n)]
    atoms = []
    for k, (x, y, z) in enumerate(cs):
        atoms.append(("C", x, y, z))
        up = 1.0 if z > 0 else -1.0          # hydrogens point away from the chain's other side
        hy, hz = ch * math.sin(half), ch * math.cos(half)
        atoms.append(("H", x, hy, z + up * hz))
        atoms.append(("H", x, -hy, z + up * hz))
        if k == 0 or k == n - 1:
            # terminal H continues the zig-zag where the next carbon would be
            sgn = -1.0 if k == 0 else 1.0
            nz = -z                           # the missing neighbour's z
            vx, vz = sgn * dx, nz - z
            norm = math.hypot(vx, vz)
            atoms.append(("H", x + ch * vx / norm, 0.0, z + ch * vz / norm))
    return atoms


def _rotation(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(seed, nmin=2, nmax=32, vol_per_mol=30.0, min_oo=2.6, max_tries=100000):
    rng = np.random.default_rng(seed)
    nmol = int(rng.integers(nmin, nmax + 1))
    box = (vol_per_mol * nmol) ** (1.0 / 3.0)
    mono = np.array([a[1:] for a in water()])
    placed, atoms = [], []
    tries = 0
    while len(placed) < nmol:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place %d waters" % nmol)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        t = rng.uniform(0.0, box, size=3)
        xyz = mono @ _rotation(q).T + t
        if all(np.linalg.norm(xyz[0] - p) >= min_oo for p in placed):
            placed.append(xyz[0])
            for (el, _, _, _), r in zip(water(), xyz):
                atoms.append((el, float(r[0]), float(r[1]), float(r[2])))
    return atoms


def write_xyz(path, atoms, charge=0):
    with open(path, "w") as f:
        f.write("%d\n%d\n" % (len(atoms), charge))
        for el, x, y, z in atoms:
            f.write("%-2s %22.16f %22.16f %22.16f\n" % (el, x, y, z))
