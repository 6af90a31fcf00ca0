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


def test_plan_grid_matches_between_precisions_on_host():
    """The host planner (no device): blocks of 128 points on the FP64 path, groups of up to
    four blocks on the INT8 path, the same screened-basis statistics the contexts report."""
    from conftest import golden, shell_table
    fx = golden("ref_water2.npz")
    sh = shell_table(fx)
    g = fx["grid"][:, :4]
    f = xc.plan_grid(sh, g, precision="fp64")
    m = xc.plan_grid(sh, g, precision="mixed", split_terms=10)
    assert f["nblocks"] == f["ngroups"] and f["npts_padded"] == 128 * f["nblocks"]
    assert m["ngroups"] <= m["nblocks"] and m["nblocks"] >= len(g) // 128
    assert 0 < f["max_nb"] <= sh.nao and 0 < m["max_nb"] <= sh.nao
    assert f["contraction_flops"] > 0 and f["workspace_bytes"] > 0


def test_plan_grid_refuses_int8_group_beyond_exact_bound():
    """A group that screens in more AOs than the INT8 contraction accumulates exactly
    (32,512: four digit products of 128^2 per K index within int32, their FP64 combination
    below 2^53) is refused with
    PDFXC_ERR_UNSUPPORTED on the mixed path and accepted on the FP64 path."""
    import numpy as np

    class Synthetic:  # 6,600 d shells on one atom: 33,000 AOs, every one of them screened in
        natom, nshell = 1, 6600
        atom_xyz = np.zeros((1, 3))
        shell_atom = np.zeros(6600, np.int32)
        shell_l = np.full(6600, 2, np.int32)
        shell_nprim = np.ones(6600, np.int32)
        prim_exp = np.full(6600, 0.5)
        prim_coef = np.ones(6600)
    xyzw = np.zeros((16, 4))
    xyzw[:, 0] = np.linspace(0.1, 0.5, 16)
    xyzw[:, 3] = 1.0
    f = xc.plan_grid(Synthetic, xyzw, precision="fp64")
    assert f["max_nb"] == 33000
    with pytest.raises(RuntimeError, match="status 6"):
        xc.plan_grid(Synthetic, xyzw, precision="mixed", split_terms=10)
    # just inside the bound: 6,502 d shells and two s shells = 32,512 AOs
    Synthetic.nshell = 6504
    for k in ("shell_atom", "shell_l", "shell_nprim", "prim_exp", "prim_coef"):
        setattr(Synthetic, k, getattr(Synthetic, k)[:6504].copy())
    Synthetic.shell_l[:2] = 0
    assert xc.plan_grid(Synthetic, xyzw, precision="mixed", split_terms=10)["max_nb"] == 32512
