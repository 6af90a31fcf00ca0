"""Open-shell build (pdfxc_build_vxc_uks) on the GPU against the reference's own
P_A, P_B overloads (tests/golden/ref_uks_water2.npz) and against the closed-shell
build. Tolerances: FP64 with atomic accumulation order, 1e-12 relative for Exc,
1e-12 absolute for Vxc elements (magnitudes ~1)."""
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
    mix = _engine(water2, precision="mixed")
    with pytest.raises(RuntimeError, match="FP64"):
        mix.build_vxc_uks("SVWN", uks["PA"], uks["PB"])
    mix.close()
