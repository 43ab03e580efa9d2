"""Generate the golden fixtures in this directory from QUICK itself.

Runs QUICK's own CUDA bridge and two-electron kernels, compiled as host code
(oracle/build_ref.py, needs the QUICK source tree), on small seeded
molecules and stores what they return: the shell-pair list of
gpu_upload_cutoff_matrix_ and the operator of gpu_get2e_ for a fixed
density.  Inputs that QUICK's Fortran host would compute (Schwarz bounds,
density screen) come from the oracle's restatement and are stored too, so the
fixtures replay without either.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.helpers import case, random_density  # noqa: E402

CASES = ["water2_631gs", "water3_631gss", "propane_631gss"]


def main():
    if not oracle.ref_available():
        subprocess = __import__("subprocess")
        subprocess.run([sys.executable, os.path.join(oracle.HERE, "build_ref.py")], check=True)
    for name in CASES:
        m, b = case(name)
        Y, cp = oracle.schwarz(b, m.xyz_bohr)
        D = random_density(b.nbasis, seed=7)
        cm = oracle.cutmatrix(b, D)
        H = random_density(b.nbasis, seed=8, scale=0.3)
        oracle.ref_upload_molecule(m, b, Y, cp, threads=8)
        pl = oracle.ref_pairlist()
        out = {}
        for method in (0, 1):
            out["fock_m%d" % method] = oracle.ref_get2e(H, D, cm, 1e-10, 1e-20, method=method)
        # QUICK's two-electron gradient (its gradient path runs with the HF method)
        oracle.ref_lib().gpu_upload_method_(oracle._i(0))
        Dg = random_density(b.nbasis, seed=5, scale=0.05)
        cmg = oracle.cutmatrix(b, Dg)
        out["grad_dense"] = Dg
        out["grad_cutMatrix"] = cmg
        out["grad2e"] = oracle.ref_grad(np.zeros(3 * m.natom), Dg, cmg, 1e-10, 1e-20)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), YCutoff=Y, cutPrim=cp, dense=D, cutMatrix=cm,
                            O_in=H, pairs=pl["pairs"], fStart=pl["fStart"], ffStart=pl["ffStart"],
                            sorted_Q=pl["sorted_Q"], sorted_Qnumber=pl["sorted_Qnumber"], **out)
        print(name, b.nbasis, len(pl["pairs"]))


if __name__ == "__main__":
    main()
