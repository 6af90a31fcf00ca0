"""pdfxc_build_vxc_noalloc, called through the C ABI, against pdfxc_build_vxc.

pdfxc_build_vxc_noalloc serves callers that cannot allocate device memory
(their memory belongs to a pool or arena they do not control, or they run
where allocation is forbidden): every operand is a device pointer they own and
the intermediates live in a fixed array inside the library. This test gives it
torch-owned device buffers, calls it twice in a row (the second call must not
see anything the first left in the shared array), and checks both results
against the regular entry point at the FP64 parity tolerances.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden, shell_table

pytestmark = pytest.mark.gpu

EXC_TOL = 1e-8
VXC_TOL = 1e-7


def device_inputs(torch, sh, xyzw, PA):
    t = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    return {
        "atom_xyz": t(sh.atom_xyz, torch.float64), "shell_atom": t(sh.shell_atom, torch.int32),
        "shell_l": t(sh.shell_l, torch.int32), "shell_nprim": t(sh.shell_nprim, torch.int32),
        "prim_exp": t(sh.prim_exp, torch.float64), "prim_coef": t(sh.prim_coef, torch.float64),
        "xyzw": t(xyzw, torch.float64), "PA": t(PA, torch.float64),
        "V": torch.full((sh.nao, sh.nao), float("nan"), dtype=torch.float64, device="cuda"),
        "en": torch.zeros(2, dtype=torch.float64, device="cuda"),
    }


def call_noalloc(L, fn_id, sh, d, npts):
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    return L.pdfxc_build_vxc_noalloc(0, fn_id, sh.natom, p(d["atom_xyz"]), sh.nshell, p(d["shell_atom"]),
                                     p(d["shell_l"]), p(d["shell_nprim"]), p(d["prim_exp"]), p(d["prim_coef"]),
                                     sh.nao, npts, p(d["xyzw"]), p(d["PA"]), p(d["V"]), p(d["en"]), None)


@pytest.mark.parametrize("name,fn,tile", [("ref_water2.npz", "SVWN", 1), ("ref_chain12.npz", "B3LYP", 4)])
def test_noalloc_matches_build_vxc_twice(name, fn, tile):
    import torch
    from proteindf_b200.xc import FUNCTIONALS, XcEngine, load_library
    fx = golden(name)
    sh = shell_table(fx)
    xyzw = np.tile(fx["grid"][:, :4], (tile, 1))  # tile > 1: several scratch chunks
    eng = XcEngine()
    eng.set_system(sh)
    eng.set_grid(xyzw)
    exc_ref, nel_ref, V_ref = eng.build_vxc(fn, fx["PA"])
    L = load_library()
    d = device_inputs(torch, sh, xyzw, fx["PA"])
    for call in range(2):
        d["V"].fill_(float("nan"))
        torch.cuda.synchronize()
        st = call_noalloc(L, FUNCTIONALS[fn], sh, d, len(xyzw))
        assert st == 0, f"call {call}: status {st}"
        exc, nel = d["en"].cpu().numpy()
        V = d["V"].cpu().numpy()
        assert abs(exc - exc_ref) <= EXC_TOL, (call, exc, exc_ref)
        assert abs(nel - nel_ref) <= 1e-9, (call, nel, nel_ref)
        assert np.abs(V - V_ref).max() <= VXC_TOL, call


def test_noalloc_rejects_oversized_basis():
    from proteindf_b200.xc import load_library
    L = load_library()
    one = ctypes.c_void_p(1)
    # 300 AOs exceeds the fixed scratch limit of 256 AOs
    assert L.pdfxc_build_vxc_noalloc(0, 0, 1, one, 1, one, one, one, one, one, 300, 10, one, one, one, one,
                                     None) == 1
