"""Shared test inputs: seeded molecules, their QUICK arrays and densities."""
import numpy as np

from quick_b200.basis import build_basis
from quick_b200.molecule import linear_alkane, water_cluster

CASES = {
    "water2_631gs": (lambda: water_cluster((2, 1, 1), seed=0), "6-31G*"),
    "water4_631gs": (lambda: water_cluster((2, 2, 1), seed=0), "6-31G*"),
    "water3_631gss": (lambda: water_cluster((3, 1, 1), seed=2), "6-31G**"),
    "propane_631gss": (lambda: linear_alkane(3, seed=1), "6-31G**"),
    "hexane_631gs": (lambda: linear_alkane(6, seed=4), "6-31G*"),
}


def case(name):
    mk, bas = CASES[name]
    m = mk()
    return m, build_basis(m.symbols, bas)


def random_density(n, seed=0, scale=0.1):
    """A symmetric test density with entries spread like a real one."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, n)) * scale
    d = d + d.T
    d[np.diag_indices(n)] += 1.0
    return np.asfortranarray(d)


def psd_density(n, nocc, seed=0, scale=0.3):
    """A positive semi-definite closed-shell density 2 C C^T (so rho(r) >= 0
    everywhere, as for a real density), C random (n x nocc)."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((n, nocc)) * scale
    return np.asfortranarray(2.0 * c @ c.T)
