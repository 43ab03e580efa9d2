"""Generate the golden fixtures in this directory from QUICK itself.

Runs QUICK's own CUDA bridge, two-electron and XC kernels, compiled as host
code (oracle/build_ref.py, needs the QUICK source tree), on small seeded
molecules and stores what they return: the shell-pair list of
gpu_upload_cutoff_matrix_, the operator of gpu_get2e_ for a fixed density,
the two-electron gradient of gpu_grad_, the operator and scalars of
gpu_getxc_ (B3LYP and BLYP), and QUICK's functional routines at sample
points.  Inputs that QUICK's Fortran host would compute (Schwarz bounds,
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
from quick_b200.basis import sigrad2  # noqa: E402
from tests.helpers import case, psd_density, random_density  # noqa: E402

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
        # QUICK's XC quadrature (gpu_getxc_) for B3LYP and BLYP at a PSD density
        sg = sigrad2(b)
        Dx = psd_density(b.nbasis, m.n_electrons // 2, seed=3)
        Hx = random_density(b.nbasis, seed=9, scale=0.3)
        out["xc_sigrad2"], out["xc_dense"], out["xc_O_in"] = sg, Dx, Hx
        for method in (1, 2):
            o, e, a, bb = oracle.ref_getxc(Hx, Dx, sg, method=method)
            out["xc_O_m%d" % method] = o
            out["xc_scalars_m%d" % method] = np.array([e, a, bb])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), YCutoff=Y, cutPrim=cp, dense=D, cutMatrix=cm,
                            O_in=H, pairs=pl["pairs"], fStart=pl["fStart"], ffStart=pl["ffStart"],
                            sorted_Q=pl["sorted_Q"], sorted_Qnumber=pl["sorted_Qnumber"], **out)
        print(name, b.nbasis, len(pl["pairs"]))


def functional_fixture():
    """QUICK's b3lyp_e/b3lypf and becke/lyp at seeded (rho, sigma) samples."""
    rng = np.random.default_rng(11)
    rho = 10.0 ** rng.uniform(-8.5, 2.5, 400)
    sigma = rho ** 2 * 10.0 ** rng.uniform(-6.0, 2.0, 400)
    out = dict(rho=rho, sigma=sigma)
    for method in (1, 2):
        f, fr, fs = oracle.ref_functional(method, rho, sigma)
        out["m%d" % method] = np.stack([f, fr, fs], axis=1)
    np.savez_compressed(os.path.join(HERE, "xc_functional.npz"), **out)


if __name__ == "__main__":
    main()
    functional_fixture()
