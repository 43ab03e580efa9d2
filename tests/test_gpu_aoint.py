"""QUICK's stored-integral (conventional SCF) path: gpu_aoint_ writes every
unique integral of the Schwarz-screened quartets to a file in QUICK's block
format, gpu_addint_ digests them with the uploaded density.  Checked: the
Fock matrix from the stored integrals against the direct gpu_get2e_ (1e-9,
both with tight cutoffs), for HF and B3LYP exchange and for a cc-pVTZ basis
(f shells: the classes up to total angular momentum 8 store from their
straight-line kernels, the larger ones from the block-per-quartet kernel);
the file holds each canonical index tuple once (i <= j, k <= l,
(i, j) <= (k, l)), in blocks of 150000 records."""
import os

import numpy as np
import pytest

from tests.helpers import case, random_density

pytestmark = pytest.mark.gpu


def _read(path, nint, block=150000):
    raw = open(path, "rb").read()
    ij, kl, val, pos = [], [], [], 0
    left = nint
    while left > 0:
        m = min(block, left)
        ij.append(np.frombuffer(raw, dtype=np.int32, count=m, offset=pos)); pos += 4 * m
        kl.append(np.frombuffer(raw, dtype=np.int32, count=m, offset=pos)); pos += 4 * m
        val.append(np.frombuffer(raw, dtype=np.float64, count=m, offset=pos)); pos += 8 * m
        left -= m
    assert pos == len(raw)
    return np.concatenate(ij), np.concatenate(kl), np.concatenate(val)


@pytest.mark.parametrize("name,method", [("water4_631gs", 0), ("propane_631gss", 1)])
def test_stored_integrals_match_direct_fock(tmp_path, oracle_lib, name, method):
    from quick_b200 import capi
    m, b = case(name)
    n = b.nbasis
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b)
        D = random_density(n, seed=3)
        cm = oracle_lib.cutmatrix(b, D)
        direct = s.get2e(np.zeros((n, n), order="F"), D, cm, 1e-14, 1e-30, method=method)
        path = str(tmp_path / "ints.bin")
        nint = s.aoint(path, 1e-14, 1e-16)
        stored = s.addint(np.zeros((n, n), order="F"), D, path, nint, method=method)
    finally:
        s.close()
    assert nint > 0
    assert np.abs(stored - direct).max() < 1e-9
    ij, kl, val = _read(path, nint)
    i, j, k, l = ij // n, ij % n, kl // n, kl % n
    assert np.all(i <= j) and np.all(k <= l) and np.all((i < k) | ((i == k) & (j <= l)))
    assert len(np.unique(ij.astype(np.int64) * n * n + kl)) == nint
    assert np.all(np.abs(val) > 1e-16)


def test_stored_integrals_with_f_shells(tmp_path, oracle_lib):
    from quick_b200 import capi
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster
    m = water_cluster((2, 1, 1), seed=0)
    b = build_basis(m.symbols, "cc-pVTZ")
    n = b.nbasis
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b)
        D = random_density(n, seed=3, scale=0.05)
        cm = oracle_lib.cutmatrix(b, D)
        direct = s.get2e(np.zeros((n, n), order="F"), D, cm, 1e-14, 1e-30, method=0)
        path = str(tmp_path / "f.bin")
        nint = s.aoint(path, 1e-14, 1e-16)
        stored = s.addint(np.zeros((n, n), order="F"), D, path, nint, method=0)
    finally:
        s.close()
    assert nint > 0
    assert np.abs(stored - direct).max() < 1e-9
    ij, kl, val = _read(path, nint)
    assert len(np.unique(ij.astype(np.int64) * n * n + kl)) == nint
