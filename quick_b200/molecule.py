"""Seeded synthetic molecules for the Fock-build workloads.

QUICK reads Cartesian coordinates in Angstrom and converts them to bohr with
``A_TO_BOHRS`` (src/modules/quick_molspec_module_.f90:355); every generator
here returns Angstrom coordinates plus the same conversion.

Workloads (all seeded, no external data):
  * water clusters (H2O)_n: O-H 0.9572 A, H-O-H 104.52 deg, a uniformly random
    orientation per water (random unit quaternion), oxygens on an
    nx x ny x nz grid of 2.9 A spacing, each jittered uniformly by +-0.2 A;
  * linear alkanes C_nH_{2n+2}: C-C 1.54 A, C-H 1.09 A, tetrahedral angles,
    backbone torsions drawn from {180, +60, -60} deg with p = 0.6/0.2/0.2.
"""
from dataclasses import dataclass

import numpy as np

from .basis import A_TO_BOHRS, ATOMIC_NUMBER


@dataclass
class Molecule:
    symbols: list            # element symbols, upper case
    xyz_angstrom: np.ndarray  # (natom, 3)
    charge: int = 0
    mult: int = 1

    @property
    def natom(self):
        return len(self.symbols)

    @property
    def xyz_bohr(self):
        """(3, natom) column-major bohr coordinates, QUICK's ``xyz`` layout."""
        return np.asfortranarray((self.xyz_angstrom * A_TO_BOHRS).T)

    @property
    def atomic_numbers(self):
        return np.array([ATOMIC_NUMBER[s] for s in self.symbols], dtype=np.int32)

    @property
    def n_electrons(self):
        return int(self.atomic_numbers.sum()) - self.charge

    def nuclear_repulsion(self):
        """sum_{i<j} Z_i Z_j / |R_i - R_j|."""
        z = self.atomic_numbers.astype(np.float64)
        x = self.xyz_bohr.T
        i, j = np.tril_indices(self.natom, -1)
        return float(np.sum(z[i] * z[j] / np.linalg.norm(x[i] - x[j], axis=1)))


def _random_rotation(rng):
    """Uniform random rotation from a uniform unit quaternion (Shoemake)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
                  np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3),
                  np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(grid, seed=0, spacing=2.9, jitter=0.2):
    """(H2O)_n with oxygens on a jittered ``grid`` = (nx, ny, nz)."""
    rng = np.random.default_rng(seed)
    roh, theta = 0.9572, np.deg2rad(104.52)
    local = np.array([[0.0, 0.0, 0.0],
                      [roh * np.sin(theta / 2), 0.0, roh * np.cos(theta / 2)],
                      [-roh * np.sin(theta / 2), 0.0, roh * np.cos(theta / 2)]])
    symbols, xyz = [], []
    nx, ny, nz = grid
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                centre = np.array([ix, iy, iz], dtype=float) * spacing
                centre += rng.uniform(-jitter, jitter, 3)
                rot = _random_rotation(rng)
                for s, p in zip("OHH", local):
                    symbols.append(s)
                    xyz.append(centre + rot @ p)
    return Molecule(symbols, np.array(xyz))


def water_cluster_n(n, seed=0):
    """(H2O)_n for arbitrary n: the first n sites of a cubic-ish grid."""
    side = int(np.ceil(n ** (1.0 / 3.0)))
    full = water_cluster((side, side, side), seed=seed)
    return Molecule(full.symbols[:3 * n], full.xyz_angstrom[:3 * n].copy())


def _place(a, b, c, bond, angle, torsion):
    """Position of atom d bonded to c with angle b-c-d and torsion a-b-c-d."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * np.cos(angle),
                   bond * np.sin(angle) * np.cos(torsion),
                   bond * np.sin(angle) * np.sin(torsion)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def linear_alkane(n_carbon, seed=0):
    """C_nH_{2n+2} built from internal coordinates (z-matrix style)."""
    rng = np.random.default_rng(seed)
    rcc, rch = 1.54, 1.09
    tet = np.arccos(-1.0 / 3.0)
    carbons = [np.array([0.0, 0.0, 0.0]), np.array([rcc, 0.0, 0.0])]
    carbons.append(carbons[1] + rcc * np.array([-np.cos(tet), np.sin(tet), 0.0]))
    choices = [np.pi, np.pi / 3, -np.pi / 3]
    for k in range(3, n_carbon):
        # redraw a torsion that would put the new carbon within 3.0 A of a
        # carbon four or more bonds back (syn-pentane clashes, ring closure)
        for attempt in range(32):
            t = choices[rng.choice(3, p=[0.6, 0.2, 0.2])] if attempt < 31 else np.pi
            c = _place(carbons[k - 3], carbons[k - 2], carbons[k - 1], rcc, tet, t)
            if all(np.linalg.norm(c - carbons[j]) >= 3.0 for j in range(k - 3)):
                break
        carbons.append(c)
    carbons = carbons[:n_carbon]
    symbols = ["C"] * n_carbon
    xyz = list(carbons)
    for k in range(n_carbon):
        c = carbons[k]
        if 0 < k < n_carbon - 1:
            a, b = carbons[k - 1], carbons[k + 1]
            bis = (c - a) / np.linalg.norm(c - a) + (c - b) / np.linalg.norm(c - b)
            bis /= np.linalg.norm(bis)
            perp = np.cross(c - a, c - b)
            perp /= np.linalg.norm(perp)
            half = tet / 2.0
            for sgn in (1, -1):
                d = np.cos(half) * bis + sgn * np.sin(half) * perp
                xyz.append(c + rch * d)
                symbols.append("H")
        else:
            nb = carbons[1] if k == 0 else carbons[k - 1]
            nb2 = carbons[2] if k == 0 else carbons[k - 2]
            for t in (np.pi, np.pi / 3, -np.pi / 3):
                xyz.append(_place(nb2, nb, c, rch, tet, t))
                symbols.append("H")
    return Molecule(symbols, np.array(xyz))


def parse_quick_input(text):
    """Atoms of a QUICK ``.in`` file: the block after the keyword line."""
    lines = text.splitlines()
    symbols, xyz = [], []
    started = False
    for ln in lines[1:]:
        tok = ln.split()
        if not tok:
            if started:
                break
            continue
        if tok[0].upper() in ATOMIC_NUMBER and len(tok) >= 4:
            started = True
            symbols.append(tok[0].upper())
            xyz.append([float(t) for t in tok[1:4]])
        elif started:
            break
    return Molecule(symbols, np.array(xyz))


def model_density(mol, basis, seed=0):
    """A symmetric density with the magnitude structure of a real one:
    |D_ij| ~ 0.5 exp(-R_ij / 1.5 bohr) between the centres of functions i and
    j, random signs, unit diagonal.  Seeded; used where no SCF density exists."""
    rng = np.random.default_rng(seed)
    xyz = mol.xyz_bohr.T
    c = xyz[basis.ncenter - 1]
    R = np.linalg.norm(c[:, None, :] - c[None, :, :], axis=-1)
    u = rng.uniform(-1.0, 1.0, R.shape)
    u = 0.5 * (u + u.T)
    D = 0.5 * np.exp(-R / 1.5) * u
    np.fill_diagonal(D, 1.0)
    return np.asfortranarray(D)
