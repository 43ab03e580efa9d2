"""Fixtures pinning the timed workloads to QUICK's own kernels.

QUICK's two-electron Fock build and gradient (src/cuda/gpu_get2e.cu and
gpu_get2e_subs*.h, driven through its gpu.cu bridge) compiled for the host
(oracle/_ref/libquickref.so, oracle/build_ref.py) are run on the seeded
workloads of the bench and written to tests/golden/:

* config0_water4_631gs.npz -- (H2O)4 in 6-31G* (76 functions), 2x2x1 cluster,
  seed 0: QUICK's full G(D), its gradient, its shell-quartet counts;
* config1_water32_631gss.npz -- (H2O)32 in 6-31G** (800 functions), 4x4x2
  cluster, seed 0: QUICK's shell-quartet counts, its gradient, and G(D) as
  projections G R (R seeded standard normal, 800 x 8), the diagonal and
  20000 seeded sampled elements (the full matrix would be 5 MB);
* config4s_water8_ccpvtz.npz -- (H2O)8 in cc-pVTZ (520 functions), 2x2x2
  cluster, seed 0: G(D) from this project's C oracle (oracle/oracle.c), as
  projections, diagonal and samples.

Density: the bench's model density (quick_b200.molecule.model_density,
seed 0), cutMatrix from QUICK's density screen, integral cutoff 1e-10,
primitive limit 1e-20, HF exchange.  Shell-quartet counts are QUICK's iclass
calls (raw) and the same walk counted once per unordered pair of shell pairs
(unique; see oracle.ref_quartet_counts).

    python tests/golden/make_config_golden.py [--threads N] [--only 0|1|4]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import oracle  # noqa: E402
from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecule import model_density, water_cluster  # noqa: E402
from quick_b200.scf import shell_cut_matrix  # noqa: E402

CONFIGS = {
    0: dict(file="config0_water4_631gs.npz", grid=(2, 2, 1), basis="6-31G*", full=True),
    1: dict(file="config1_water32_631gss.npz", grid=(4, 4, 2), basis="6-31G**", full=False),
    # the f-shell workload's basis on the largest cluster the C oracle builds
    # in about a minute: its Fock matrix only (QUICK's own f-shell kernels are
    # not rotationally covariant in their fd/ff zones, so the oracle, pinned
    # to QUICK on the spd classes and to finite differences on f, is the
    # reference here)
    4: dict(file="config4s_water8_ccpvtz.npz", grid=(2, 2, 2), basis="cc-pVTZ", full=False, source="oracle"),
}
CUTOFF, PRIM_LIMIT = 1e-10, 1e-20
NPROJ, NSAMPLE = 8, 20000


def probes(n, seed=123):
    """The projection vectors and sampled (row, column) positions of a
    fixture, regenerated from the seed by the tests."""
    rng = np.random.default_rng(seed)
    R = rng.standard_normal((n, NPROJ))
    idx = rng.integers(0, n, size=(NSAMPLE, 2))
    return R, idx


def make(k, threads):
    c = CONFIGS[k]
    m = water_cluster(c["grid"], seed=0)
    b = build_basis(m.symbols, c["basis"])
    n = b.nbasis
    Y, cp = oracle.schwarz(b, m.xyz_bohr)
    D = model_density(m, b, seed=0)
    cm = shell_cut_matrix(b, D)
    if c.get("source") == "oracle":
        t0 = time.time()
        G, cnt = oracle.fock(b, m.xyz_bohr, Y, cp, cm, D, CUTOFF, PRIM_LIMIT)
        R, idx = probes(n)
        np.savez_compressed(os.path.join(HERE, c["file"]), nbasis=n, GR=G @ R, diag=np.diag(G).copy(),
                            sample=G[idx[:, 0], idx[:, 1]])
        print("config %d (oracle): %d functions, Fock %.1f s" % (k, n, time.time() - t0))
        return
    keep = oracle.ref_upload_molecule(m, b, Y, cp, threads=threads)   # noqa: F841
    t0 = time.time()
    G = oracle.ref_get2e(np.zeros((n, n), order="F"), D, cm, CUTOFF, PRIM_LIMIT)
    raw, uniq = oracle.ref_quartet_counts()
    t1 = time.time()
    g = oracle.ref_grad(np.zeros(3 * m.natom), D, cm, CUTOFF, PRIM_LIMIT)
    t2 = time.time()
    out = dict(nbasis=n, raw_quartets=raw, unique_quartets=uniq, grad=g)
    if c["full"]:
        out["G"] = G
    else:
        R, idx = probes(n)
        out.update(GR=G @ R, diag=np.diag(G).copy(), sample=G[idx[:, 0], idx[:, 1]])
    np.savez_compressed(os.path.join(HERE, c["file"]), **out)
    print("config %d: %d functions, %d unique / %d raw quartets, Fock %.1f s, gradient %.1f s"
          % (k, n, uniq, raw, t1 - t0, t2 - t1))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--only", type=int, choices=sorted(CONFIGS), default=None)
    a = ap.parse_args()
    for k in sorted(CONFIGS):
        if a.only is None or a.only == k:
            make(k, a.threads)
