"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "quick_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:gpu|qb)_\w+)\s*\(", txt)))


def test_header_declares_quick_bridge():
    syms = declared_symbols()
    for s in ["gpu_startup_", "gpu_init_", "gpu_setup_", "gpu_upload_basis_", "gpu_upload_cutoff_matrix_",
              "gpu_upload_calculated_", "gpu_upload_cutoff_", "gpu_get2e_", "gpu_grad_", "gpu_getxc_"]:
        assert s in syms


def test_library_exports_all_declared_symbols():
    from quick_b200 import capi
    lib = capi.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_init_without_gpu_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from quick_b200 import capi
    with pytest.raises(capi.QuickB200Error):
        capi.Session(0)
