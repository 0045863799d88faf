"""Seeded synthetic geometries for the benchmark and parity workloads.

No public dataset is involved: every system is generated here from a seed.
  * ``water()``            H2O, O (0,0,0.1173) A, H (0,+-0.7572,-0.4692) A
  * ``water_cluster(k, box, seed)``  k rigid monomers, uniform random rotation
    (unit quaternion) and uniform O position inside a box of side ``box`` A,
    rejecting placements with any O-O distance below 2.7 A
  * ``alkane(nc, seed)``   all-trans CnH(2n+2) zig-zag, C-C 1.54 A, C-H 1.09 A,
    tetrahedral angles, uniform +-0.02 A jitter on every coordinate
"""
import numpy as np

from .basis import Molecule

WATER_O = np.array([0.0, 0.0, 0.1173])
WATER_H1 = np.array([0.0, 0.7572, -0.4692])
WATER_H2 = np.array([0.0, -0.7572, -0.4692])


def water():
    return Molecule(["o", "h", "h"], [WATER_O, WATER_H1, WATER_H2], angstrom=True)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_cluster(k, box, seed, min_oo=2.7, max_tries=200000):
    rng = np.random.default_rng(seed)
    mono = np.stack([WATER_O, WATER_H1, WATER_H2]) - WATER_O
    oxygens, syms, coords = [], [], []
    tries = 0
    while len(oxygens) < k:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could not place {k} waters in a {box} A box")
        o = rng.uniform(0.0, box, size=3)
        if any(np.linalg.norm(o - p) < min_oo for p in oxygens):
            continue
        R = _random_rotation(rng)
        pos = mono @ R.T + o
        oxygens.append(o)
        syms += ["o", "h", "h"]
        coords += list(pos)
    return Molecule(syms, coords, angstrom=True)


def alkane(nc, seed, jitter=0.02):
    rng = np.random.default_rng(seed)
    theta = np.deg2rad(109.47)
    cc, ch = 1.54, 1.09
    # zig-zag backbone in the xy plane along x
    dx = cc * np.sin(theta / 2)
    dy = cc * np.cos(theta / 2)
    carbons = np.array([[i * dx, (i % 2) * dy, 0.0] for i in range(nc)])
    syms = ["c"] * nc
    coords = list(carbons)
    # hydrogens: two per carbon out of plane (+-z), plus the end caps
    for i in range(nc):
        c = carbons[i]
        out_y = -1.0 if i % 2 else 1.0  # away from the backbone kink
        # bisector direction in-plane opposite to neighbours, tilted out of plane
        half = theta / 2
        for sz in (1.0, -1.0):
            v = np.array([0.0, -out_y * np.cos(half), sz * np.sin(half)])
            coords.append(c + ch * v / np.linalg.norm(v))
            syms.append("h")
    # methyl caps: the third H sits where the zig-zag's next carbon would be
    for end, virt in ((0, -1), (nc - 1, nc)):
        c = carbons[end]
        v = np.array([virt * dx, (virt % 2) * dy, 0.0]) - c
        v /= np.linalg.norm(v)
        coords.append(c + ch * v)
        syms.append("h")
    coords = np.array(coords) + rng.uniform(-jitter, jitter, size=(len(coords), 3))
    return Molecule(syms, coords, angstrom=True)


# The five workloads, by what they are.
def h2o():
    """H2O / cc-pVDZ (24 functions), direct FP64 SCF."""
    return water()


def water16(seed=16):
    """(H2O)16 in a 9 A cube: cc-pVDZ (384) + VDZ-JKFIT (1856)."""
    return water_cluster(16, 9.0, seed)


def c20h42(seed=20):
    """C20H42 / 6-311G** (612 functions), direct J/K."""
    return alkane(20, seed)


def water8(seed=8):
    """(H2O)8 in a 7 A cube: cc-pVDZ (192) + VDZ-JKFIT (928), gradient."""
    return water_cluster(8, 7.0, seed)


def water64(seed=64):
    """(H2O)64 in a 14 A cube: aug-cc-pVDZ (2624) + AVDZ-JKFIT (9600)."""
    return water_cluster(64, 14.0, seed)
