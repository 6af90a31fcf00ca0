"""Open-shell build (pdfxc_build_vxc_uks) on the GPU against the reference's own
P_A, P_B overloads (tests/golden/ref_uks_water2.npz) and against the closed-shell
build. Tolerances: FP64 with atomic accumulation order, 1e-12 relative for Exc,
1e-12 absolute for Vxc elements (magnitudes ~1). The INT8 path: the mixed tolerances of
the closed-shell tests, |dExc|/|Exc| <= 2e-10 and max|dVxc|/max|Vxc| <= 5e-9."""
import numpy as np
import pytest

from conftest import golden, shell_table

pytestmark = pytest.mark.gpu

FUNCS = ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"]


@pytest.fixture(scope="module")
def uks():
    return golden("ref_uks_water2.npz")


def _engine(water2, precision="fp64"):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(device=0, precision=precision, split_terms=10 if precision == "mixed" else 6)
    eng.set_system(shell_table(water2))
    eng.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
    return eng


@pytest.mark.parametrize("fn", FUNCS)
def test_uks_vs_reference(water2, uks, fn):
    eng = _engine(water2)
    exc, na, nb, FA, FB = eng.build_vxc_uks(fn, uks["PA"], uks["PB"])
    assert abs(exc - uks[f"{fn}_exc"][0]) < 1e-12 * abs(uks[f"{fn}_exc"][0])
    assert np.abs(FA - uks[f"{fn}_vxc_a"]).max() < 1e-12
    assert np.abs(FB - uks[f"{fn}_vxc_b"]).max() < 1e-12
    assert abs(na - uks[f"{fn}_nelec_alpha"][0]) < 1e-12
    assert abs(nb - uks[f"{fn}_nelec_beta"][0]) < 1e-12
    if f"{fn}_rho" in uks:
        gga = fn != "SVWN"
        rho = eng.get_rho_uks(gga)
        ref = uks[f"{fn}_rho"]
        assert np.all(np.abs(rho - ref) <= 1e-12 * np.maximum(1.0, np.abs(ref)))
    eng.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_uks_with_equal_spins_is_the_closed_shell_build(water2, fn):
    eng = _engine(water2)
    PA = water2["PA"]
    e_r, n_r, V = eng.build_vxc(fn, PA)
    e_u, na, nb, FA, FB = eng.build_vxc_uks(fn, PA, PA)
    assert abs(e_u - e_r) < 1e-12 * abs(e_r)
    assert abs(na - n_r) < 1e-12 and abs(nb - n_r) < 1e-12
    assert np.abs(FA - V).max() < 1e-12 and np.abs(FB - V).max() < 1e-12
    eng.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_uks_incremental_and_restart(water2, uks, fn):
    """xc-update for both spins: rho(P/2) stored, then rho(P/2) added; and the same
    second step after reseeding the stored densities with set_rho_uks."""
    gga = fn != "SVWN"
    eng = _engine(water2)
    eng.build_vxc_uks(fn, 0.5 * uks["PA"], 0.5 * uks["PB"])
    saved = eng.get_rho_uks(gga)
    exc, na, nb, FA, FB = eng.build_vxc_uks(fn, 0.5 * uks["PA"], 0.5 * uks["PB"], incremental=True)
    assert abs(exc - uks[f"{fn}_exc"][0]) < 1e-11 * abs(uks[f"{fn}_exc"][0])
    assert np.abs(FA - uks[f"{fn}_vxc_a"]).max() < 1e-11
    assert np.abs(FB - uks[f"{fn}_vxc_b"]).max() < 1e-11
    eng.close()
    eng = _engine(water2)
    eng.set_rho_uks(saved, gga)
    exc2, _, _, FA2, FB2 = eng.build_vxc_uks(fn, 0.5 * uks["PA"], 0.5 * uks["PB"], incremental=True)
    assert abs(exc2 - exc) < 1e-12 * abs(exc)
    assert np.abs(FA2 - FA).max() < 1e-12 and np.abs(FB2 - FB).max() < 1e-12
    eng.close()


def test_uks_state_errors(water2, uks):
    eng = _engine(water2)
    with pytest.raises(RuntimeError, match="incremental"):
        eng.build_vxc_uks("SVWN", uks["PA"], uks["PB"], incremental=True)
    eng.build_vxc("SVWN", uks["PA"])  # a closed-shell build does not seed the open-shell update
    with pytest.raises(RuntimeError, match="incremental"):
        eng.build_vxc_uks("SVWN", uks["PA"], uks["PB"], incremental=True)
    eng.close()
    from proteindf_b200.xc import XcEngine
    bf = XcEngine(device=0, precision="mixed", split_terms=6)
    bf.set_system(shell_table(water2))
    bf.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
    with pytest.raises(RuntimeError, match="BF16"):
        bf.build_vxc_uks("SVWN", uks["PA"], uks["PB"])
    bf.close()


OZ_TOL = (2e-10, 5e-9)


@pytest.mark.parametrize("fn", ["SVWN", "BLYP", "B3LYP"])
def test_uks_int8_vs_reference(water2, uks, fn):
    eng = _engine(water2, precision="mixed")
    exc, na, nb, FA, FB = eng.build_vxc_uks(fn, uks["PA"], uks["PB"])
    rE = abs(exc - uks[f"{fn}_exc"][0]) / abs(uks[f"{fn}_exc"][0])
    rA = np.abs(FA - uks[f"{fn}_vxc_a"]).max() / np.abs(uks[f"{fn}_vxc_a"]).max()
    rB = np.abs(FB - uks[f"{fn}_vxc_b"]).max() / np.abs(uks[f"{fn}_vxc_b"]).max()
    print(f"(H2O)2 open shell {fn} INT8: |dExc|/|Exc|={rE:.3e} Vxc_A {rA:.3e} Vxc_B {rB:.3e}")
    assert rE <= OZ_TOL[0] and rA <= OZ_TOL[1] and rB <= OZ_TOL[1]
    assert abs(na - uks[f"{fn}_nelec_alpha"][0]) < 1e-8 and abs(nb - uks[f"{fn}_nelec_beta"][0]) < 1e-8
    eng.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_uks_int8_equal_spins_is_the_closed_shell_int8_build(water2, fn):
    eng = _engine(water2, precision="mixed")
    PA = water2["PA"]
    e_r, n_r, V = eng.build_vxc(fn, PA)
    e_u, na, nb, FA, FB = eng.build_vxc_uks(fn, PA, PA)
    assert abs(e_u - e_r) < 1e-12 * abs(e_r)
    assert abs(na - n_r) < 1e-12 and abs(nb - n_r) < 1e-12
    assert np.abs(FA - V).max() < 1e-12 and np.abs(FB - V).max() < 1e-12
    eng.close()


def test_uks_int8_chunks_incremental_and_fp64(water2):
    """A 30-atom chain in several workspace chunks (a 64 MiB workspace), B3LYP with
    different alpha and beta densities: the INT8 open-shell build against the FP64 one on
    the same grid, then an xc-update step (half the densities stored, half added) on the
    INT8 path against the one-step build."""
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(30, seed=41)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["USER-75x302"])
    PA = 0.5 * systems.density_matrix(sh.nao, 60, seed=42)
    PB = 0.5 * systems.density_matrix(sh.nao, 52, seed=43)
    from proteindf_b200 import xc
    wb = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    assert xc.plan_grid(sh, np.c_[P, W], precision="mixed", workspace_bytes=64 << 20)["nchunks"] > 1
    out = {}
    for prec in ("fp64", "mixed"):
        eng = XcEngine(device=0, precision=prec, split_terms=10, workspace_bytes=64 << 20)
        eng.set_system(sh)
        eng.set_grid(np.c_[P, eng.becke_weights(P, A, W, wb)], A)
        out[prec] = eng.build_vxc_uks("B3LYP", PA, PB)
        if prec == "mixed":
            eng.build_vxc_uks("B3LYP", 0.5 * PA, 0.5 * PB)
            out["step"] = eng.build_vxc_uks("B3LYP", 0.5 * PA, 0.5 * PB, incremental=True)
        eng.close()
    f, m, st = out["fp64"], out["mixed"], out["step"]
    rE = abs(m[0] - f[0]) / abs(f[0])
    rV = max(np.abs(m[3] - f[3]).max() / np.abs(f[3]).max(), np.abs(m[4] - f[4]).max() / np.abs(f[4]).max())
    print(f"chain30 open shell B3LYP INT8 vs FP64: |dExc|/|Exc|={rE:.3e} max|dVxc|/max|Vxc|={rV:.3e}")
    assert rE <= OZ_TOL[0] and rV <= OZ_TOL[1]
    assert abs(m[1] - f[1]) < 1e-8 and abs(m[2] - f[2]) < 1e-8
    assert abs(st[0] - m[0]) <= 1e-11 * abs(m[0])
    assert np.abs(st[3] - m[3]).max() <= 1e-9 * np.abs(m[3]).max() and np.abs(st[4] - m[4]).max() <= 1e-9 * np.abs(m[4]).max()
