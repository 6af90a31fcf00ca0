"""The C-ABI library loads, exports every symbol include/pdfxc.h declares, and
fails cleanly (status codes, no crash) where no GPU is present."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
import proteindf_b200.xc as xc


def header_symbols():
    text = open(os.path.join(ROOT, "include", "pdfxc.h")).read()
    decl = r"^\s*(?:pdfxc_status|void|const char\s*\*)\s*(pdfxc_[a-z_]+)\s*\("
    return sorted(set(re.findall(decl, text, flags=re.M)))


def test_library_exports_header_symbols():
    L = xc.load_library()
    syms = header_symbols()
    assert len(syms) >= 13
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(xc.EXPORTS)


def test_default_options():
    L = xc.load_library()
    o = xc.Options()
    L.pdfxc_default_options(ctypes.byref(o))
    assert o.precision == 0 and o.block_points == 128 and o.rho_cutoff == 1e-16


def test_null_and_state_errors_without_gpu():
    L = xc.load_library()
    assert L.pdfxc_create(None, 0, None) == 1  # PDFXC_ERR_ARG
    assert L.pdfxc_set_grid(None, 10, None, None) == 1
    assert L.pdfxc_build_vxc(None, 0, None, 0, None, None, None) == 1
    assert L.pdfxc_last_error(None) == b"null context"


def test_create_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = xc.load_library()
    h = ctypes.c_void_p()
    assert L.pdfxc_create(ctypes.byref(h), 0, None) == 2  # PDFXC_ERR_CUDA
