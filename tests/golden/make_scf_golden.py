"""Writes scf_golden.json: RHF total energies from the CPU oracle (its
one-electron integrals, Fock build and this package's SCF driver) for the
GPU SCF tests to compare with.  About two minutes on one host.

    python tests/golden/make_scf_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, ".."))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from helpers import OracleEngine, ace_ala  # noqa: E402
from quick_b200 import scf  # noqa: E402
from quick_b200.basis import build_basis  # noqa: E402

CUTOFF, PRIM = 1e-9, 1e-20     # QUICK's keywords of these inputs: cutoff=1.0e-9 (primLimit 1e-20)


def main():
    out = dict(integral_cutoff=CUTOFF, prim_limit=PRIM, conv=1e-8, energies={})
    for name, bs in (("ala2", "6-31G"), ("ala2", "6-31G*")):
        m = ace_ala(name)
        b = build_basis(m.symbols, bs)
        r = scf.rhf(OracleEngine(m, b, CUTOFF, PRIM), m.n_electrons // 2, conv=1e-8)
        assert r.converged
        out["energies"]["%s/%s" % (name, bs)] = r.energy
        print(name, bs, "%.9f" % r.energy)
    # Kohn-Sham: water (O-H 0.96 A, 104.5 deg) in 6-31G*, B3LYP (method 1) and
    # BLYP (method 2), functional and SG1 quadrature from QUICK's own getxc
    # compiled for the host (oracle/_ref), integral cutoff 1e-11
    import math
    import numpy as np
    from quick_b200.molecule import Molecule
    t = math.radians(104.5)
    w = Molecule(["O", "H", "H"], np.array([[0, 0, 0], [0.96, 0, 0], [0.96 * math.cos(t), 0.96 * math.sin(t), 0]]))
    wb = build_basis(w.symbols, "6-31G*")
    for method, name in ((1, "B3LYP"), (2, "BLYP")):
        r = scf.rhf(OracleEngine(w, wb, 1e-11, 1e-20, method=method), w.n_electrons // 2, conv=1e-8)
        assert r.converged
        out["energies"]["water/6-31G*/%s" % name] = r.energy
        print("water", name, "%.10f" % r.energy)
    with open(os.path.join(HERE, "scf_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
