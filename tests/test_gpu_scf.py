"""GPU one-electron integrals, one-electron gradient and the SCF built on the
GPU Fock build and gradients, against the CPU oracle, QUICK's published HF
energies and central finite differences.

Tolerances: S and H 1e-11 absolute; the one-electron gradient 1e-10
relative to its largest element; SCF energies 1e-8 Eh against the oracle's
SCF (tests/golden/scf_golden.json) and 1e-4 Eh against QUICK's 2011
published energies (the present code differs from them by 1.0e-5 to
5.3e-5 Eh; QUICK's present two-electron kernels agree with this code);
the full gradient 1e-6 Eh/bohr against central differences (h = 1e-3 bohr);
mixed precision |dE| <= 1e-6 Eh and gradient 1e-5 Eh/bohr against FP64."""
import json
import os

import numpy as np
import pytest

from conftest import gpu_available
from helpers import PUBLISHED_HF, ace_ala
from quick_b200 import capi, scf
from quick_b200.basis import A_TO_BOHRS, build_basis
from quick_b200.molecule import Molecule, water_cluster

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no GPU")]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scf_golden.json")


def _session(m, b):
    s = capi.Session(0)
    s.upload_molecule(m, b)
    return s


def _sym(n, rng):
    a = rng.uniform(-1.0, 1.0, (n, n))
    return np.asfortranarray(0.5 * (a + a.T))


@pytest.mark.parametrize("mk,bs", [
    (lambda: water_cluster((3, 1, 1), seed=1), "6-31G**"),
    (lambda: water_cluster((2, 1, 1), seed=1), "cc-pVTZ"),
    (lambda: ace_ala("ala2"), "6-31G*"),
])
def test_oneint_and_grad1e_vs_oracle(oracle_lib, mk, bs):
    m = mk()
    b = build_basis(m.symbols, bs)
    s = _session(m, b)
    try:
        S, H = s.oneint()
        So, Ho = oracle_lib.oneint(b, m)
        assert np.abs(S - So).max() < 1e-11
        assert np.abs(H - Ho).max() < 1e-11
        rng = np.random.default_rng(0)
        D, W = _sym(b.nbasis, rng), _sym(b.nbasis, rng)
        g = s.grad1e(D, W)
        go = oracle_lib.grad1e(b, m, D, W)
        assert np.abs(g - go).max() < 1e-10 * np.abs(go).max()
    finally:
        s.close()


@pytest.mark.parametrize("name,bs", [("ala2", "6-31G"), ("ala2", "6-31G*")])
def test_scf_energy_vs_oracle_and_published(name, bs):
    with open(GOLDEN) as fh:
        gold = json.load(fh)
    m = ace_ala(name)
    b = build_basis(m.symbols, bs)
    s = _session(m, b)
    try:
        r = scf.rhf(scf.GpuEngine(s, m, b, gold["integral_cutoff"], gold["prim_limit"]), m.n_electrons // 2,
                    conv=gold["conv"])
    finally:
        s.close()
    assert r.converged
    assert abs(r.energy - gold["energies"]["%s/%s" % (name, bs)]) < 1e-8
    assert abs(r.energy - PUBLISHED_HF[(name, bs)]) < 1e-4


@pytest.mark.parametrize("name,bs", [("ala3", "6-31G"), ("ala3", "6-31G*")])
def test_scf_energy_vs_published(name, bs):
    m = ace_ala(name)
    b = build_basis(m.symbols, bs)
    s = _session(m, b)
    try:
        r = scf.rhf(scf.GpuEngine(s, m, b, 1e-9, 1e-20), m.n_electrons // 2, conv=1e-8)
    finally:
        s.close()
    assert r.converged
    assert abs(r.energy - PUBLISHED_HF[(name, bs)]) < 1e-4


def _energy(m, b, cut=1e-12):
    s = _session(m, b)
    try:
        eng = scf.GpuEngine(s, m, b, cut, 1e-25)
        r = scf.rhf(eng, m.n_electrons // 2, conv=1e-10)
        return r, eng.gradient(r.D, r.W)
    finally:
        s.close()


def test_full_gradient_vs_finite_differences():
    """Six seeded coordinates of a water dimer (6-31G*), central differences
    of the SCF energy with h = 1e-3 bohr."""
    m = water_cluster((2, 1, 1), seed=3)
    b = build_basis(m.symbols, "6-31G*")
    r, g = _energy(m, b)
    h = 1e-3
    rng = np.random.default_rng(7)
    coords = [(int(a), int(k)) for a, k in zip(rng.integers(0, m.natom, 6), rng.integers(0, 3, 6))]
    for atom, k in coords:
        e = []
        for sgn in (1, -1):
            x = m.xyz_angstrom.copy()
            x[atom, k] += sgn * h / A_TO_BOHRS
            e.append(_energy(Molecule(m.symbols, x), b)[0].energy)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(g[3 * atom + k] - fd) < 1e-6, (atom, k, g[3 * atom + k], fd)
    assert np.abs(g.reshape(-1, 3).sum(axis=0)).max() < 1e-8


def test_mixed_precision_scf():
    """(H2O)8 in 6-31G**: the SCF energy and gradient with quartets below the
    Schwarz x |D| bound 1e-3 in FP32 against all-FP64."""
    m = water_cluster((2, 2, 2), seed=0)
    b = build_basis(m.symbols, "6-31G**")
    s = _session(m, b)
    try:
        eng = scf.GpuEngine(s, m, b, 1e-10, 1e-20)
        r64 = scf.rhf(eng, m.n_electrons // 2, conv=1e-8)
        g64 = eng.gradient(r64.D, r64.W)
        s.set_mixed_precision(1e-3)
        r32 = scf.rhf(eng, m.n_electrons // 2, conv=1e-8)
        split = s.fock_split()
        g32 = eng.gradient(r32.D, r32.W)
        s.set_mixed_precision(0.0)
    finally:
        s.close()
    assert r64.converged and r32.converged
    assert split["fp32"] > 0
    assert abs(r32.energy - r64.energy) < 1e-6
    assert np.abs(g32 - g64).max() < 1e-5


def test_incremental_fock_builds():
    """Delta-D Fock builds (G(D_n) = G(D_n-1) + G(D_n - D_n-1), full rebuild
    every 8 iterations) converge to the same energy."""
    m = water_cluster((2, 2, 1), seed=2)
    b = build_basis(m.symbols, "6-31G*")
    s = _session(m, b)
    try:
        eng = scf.GpuEngine(s, m, b, 1e-11, 1e-20)
        full = scf.rhf(eng, m.n_electrons // 2, conv=1e-8)
        inc = scf.rhf(eng, m.n_electrons // 2, conv=1e-8, incremental=True)
    finally:
        s.close()
    assert full.converged and inc.converged
    assert abs(full.energy - inc.energy) < 1e-8


def test_device_scf_matches_host_scf():
    """The device-resident SCF (DeviceRHF: density screen, Fock build,
    gradients and the SCF algebra on the GPU) against the host-driven SCF
    through the gpu_* host entry points: energy 1e-9 Eh, gradient 1e-8."""
    m = water_cluster((2, 2, 1), seed=5)
    r_h, g_h = scf.run_rhf_gpu(m, "6-31G*", 1e-10, 1e-20, conv=1e-9, gradient=True)
    r_d, g_d = scf.run_rhf_device(m, "6-31G*", 1e-10, 1e-20, conv=1e-9)
    assert r_h.converged and r_d.converged
    assert abs(r_h.energy - r_d.energy) < 1e-9
    assert np.abs(g_h - g_d).max() < 1e-8
    # delta-D builds and the mixed split on the device path
    r_i, g_i = scf.run_rhf_device(m, "6-31G*", 1e-10, 1e-20, conv=1e-9, incremental=True, mixed_cut=1e-3)
    assert r_i.converged
    assert abs(r_i.energy - r_d.energy) < 1e-6
    assert np.abs(g_i - g_d).max() < 1e-5


@pytest.mark.parametrize("incremental,mixed", [(False, 0.0), (True, 1e-3)])
def test_graph_captured_scf(incremental, mixed):
    """Each SCF iteration as one CUDA-graph replay (device DIIS solve, SP2
    purification instead of diagonalisation) against the eager device SCF:
    energy 5e-8 Eh (the two converge along different DIIS paths to density
    RMS 1e-9; 1e-6 with the mixed split), gradient 1e-7 Eh/bohr (1e-5
    mixed); the converged density is idempotent (D S D = 2 D to 1e-7; its
    elements reach 2)."""
    m = water_cluster((2, 2, 1), seed=5)
    r_d, g_d = scf.run_rhf_device(m, "6-31G*", 1e-10, 1e-20, conv=1e-9)
    r_g, g_g = scf.run_rhf_device(m, "6-31G*", 1e-10, 1e-20, conv=1e-9, graph=True, incremental=incremental,
                                  mixed_cut=mixed)
    assert r_d.converged and r_g.converged
    tol_e, tol_g = (1e-6, 1e-5) if mixed else (5e-8, 1e-7)
    assert abs(r_g.energy - r_d.energy) < tol_e
    assert np.abs(g_g - g_d).max() < tol_g
    b = build_basis(m.symbols, "6-31G*")
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b)
        S, _ = s.oneint()
    finally:
        s.close()
    D = r_g.D
    assert np.abs(D @ S @ D - 2.0 * D).max() < 1e-7


@pytest.mark.parametrize("method,name", [(1, "B3LYP"), (2, "BLYP")])
def test_kohn_sham_scf(method, name):
    """Kohn-Sham SCF (hybrid-exchange Fock build + SG1 XC quadrature on the
    GPU), host-driven and device-resident, against the oracle's SCF with
    QUICK's own getxc (tests/golden/scf_golden.json): 1e-7 Eh."""
    import math
    with open(GOLDEN) as fh:
        gold = json.load(fh)["energies"]["water/6-31G*/%s" % name]
    t = math.radians(104.5)
    m = Molecule(["O", "H", "H"], np.array([[0, 0, 0], [0.96, 0, 0], [0.96 * math.cos(t), 0.96 * math.sin(t), 0]]))
    r_h, _ = scf.run_rhf_gpu(m, "6-31G*", 1e-11, 1e-20, conv=1e-8, method=method)
    r_d, g_d = scf.run_rhf_device(m, "6-31G*", 1e-11, 1e-20, conv=1e-8, method=method)
    assert r_h.converged and r_d.converged
    assert g_d is not None and np.abs(g_d.reshape(-1, 3).sum(axis=0)).max() < 1e-6   # translational invariance
    assert abs(r_h.energy - gold) < 1e-7
    assert abs(r_d.energy - gold) < 1e-7


@pytest.mark.parametrize("xc_grid", [1, 2])
def test_kohn_sham_gradient_vs_finite_differences(xc_grid):
    """The B3LYP nuclear gradient (one-electron, two-electron with the 0.2
    exchange fraction, and the XC term with the grid moving with the atoms:
    basis-centre, point-movement and partition-weight derivatives) against
    central differences (h = 1e-3 bohr) of the converged Kohn-Sham energy, on
    QUICK's SG1 grid (xc_grid 1) and the 75 x 302 Becke grid (2): 1e-5
    Eh/bohr on six seeded coordinates of a water dimer in 6-31G*."""
    m = water_cluster((2, 1, 1), seed=3)
    kw = dict(conv=1e-10, method=1, xc_grid=xc_grid, max_iter=200)
    r, g = scf.run_rhf_device(m, "6-31G*", 1e-12, 1e-25, **kw)
    assert r.converged
    h = 1e-3
    rng = np.random.default_rng(11)
    for atom, k in [(int(a), int(c)) for a, c in zip(rng.integers(0, m.natom, 6), rng.integers(0, 3, 6))]:
        e = []
        for sgn in (1, -1):
            x = m.xyz_angstrom.copy()
            x[atom, k] += sgn * h / A_TO_BOHRS
            rr, _ = scf.run_rhf_device(Molecule(m.symbols, x), "6-31G*", 1e-12, 1e-25, gradient=False, **kw)
            e.append(rr.energy)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(g[3 * atom + k] - fd) < 1e-5, (xc_grid, atom, k, g[3 * atom + k], fd)
    assert np.abs(g.reshape(-1, 3).sum(axis=0)).max() < 1e-6


def test_becke_grid_integrates_the_density():
    """The 75 x 302 Becke grid: its weights integrate a sum of atom-centred
    Gaussians exp(-|r - R_A|^2) to 1e-7 relative (SG1: 1e-4); the electron
    count of a converged B3LYP density of a water trimer is 30 to 5e-4 on
    both grids (QUICK's density cutoffs drop the far tails); the B3LYP energy
    on the two grids agrees to 1e-3 Eh."""
    m = water_cluster((3, 1, 1), seed=2)
    rs, _ = scf.run_rhf_device(m, "6-31G*", 1e-11, 1e-20, conv=1e-8, method=1, xc_grid=1, gradient=False)
    rb, _ = scf.run_rhf_device(m, "6-31G*", 1e-11, 1e-20, conv=1e-8, method=1, xc_grid=2, gradient=False)
    assert rs.converged and rb.converged
    assert abs(rs.energy - rb.energy) < 1e-3
    b = build_basis(m.symbols, "6-31G*")
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b)
        from quick_b200.basis import sigrad2
        sg = np.ascontiguousarray(sigrad2(b))
        for grid, tol_q in ((2, 1e-7), (1, 1e-4)):
            _, _, na, nb_ = s.getxc(np.zeros((b.nbasis, b.nbasis), order="F"), rb.D, sg, method=1, isg=grid)
            assert abs(na + nb_ - m.n_electrons) < 5e-4, (grid, na + nb_)
            p = s.xc_grid()
            d2 = ((p[:, None, :3] - m.xyz_bohr.T[None, :, :]) ** 2).sum(axis=2)
            got = float((p[:, 3] * np.exp(-d2).sum(axis=1)).sum())
            ref = m.natom * np.pi ** 1.5
            assert abs(got - ref) < tol_q * ref, (grid, got, ref)
    finally:
        s.close()


def test_fshell_full_gradient_vs_finite_differences():
    """cc-pVTZ water (f on O): the full analytic RHF gradient through the
    f-class gradient kernel against central differences (h = 1e-3 bohr) of
    the SCF energy."""
    import math
    t = math.radians(103.0)
    m = Molecule(["O", "H", "H"], np.array([[0, 0, 0], [0.97, 0, 0], [0.97 * math.cos(t), 0.97 * math.sin(t), 0]]))
    b = build_basis(m.symbols, "cc-pVTZ")
    r, g = _energy(m, b)
    h = 1e-3
    for atom, k in ((0, 0), (1, 1), (2, 0)):
        e = []
        for sgn in (1, -1):
            x = m.xyz_angstrom.copy()
            x[atom, k] += sgn * h / A_TO_BOHRS
            e.append(_energy(Molecule(m.symbols, x), b)[0].energy)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(g[3 * atom + k] - fd) < 1e-6, (atom, k, g[3 * atom + k], fd)


def test_batched_scf_matches_single_molecules():
    """Eight water clusters of 1..6 molecules advanced together (one batched
    Fock build per iteration, batched DIIS and SP2, one batched two-electron
    gradient) against the single-molecule device SCF: energies 1e-7 Eh,
    gradients 1e-6 Eh/bohr; and with the mixed split: 1e-6 / 1e-5."""
    from quick_b200.molecule import water_cluster_n
    mols = [water_cluster_n(k, seed=40 + k) for k in (1, 3, 2, 6, 4, 1, 5, 2)]
    ref = [scf.run_rhf_device(m, "6-31G*", 1e-10, 1e-20, conv=1e-9) for m in mols]
    for mixed, tol_e, tol_g in ((0.0, 1e-7, 1e-6), (1e-3, 1e-6, 1e-5)):
        res, grads, _ = scf.run_batch_rhf(mols, "6-31G*", 1e-10, 1e-20, conv=1e-9, mixed_cut=mixed)
        for (r0, g0), r, g in zip(ref, res, grads):
            assert r0.converged and r.converged
            assert abs(r.energy - r0.energy) < tol_e, (mixed, r.energy, r0.energy)
            assert np.abs(g - g0).max() < tol_g, (mixed, np.abs(g - g0).max())
