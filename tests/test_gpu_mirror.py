"""proteindf_b200.dfcalcgridx.DfCalcGridX: the reference class's interface
(accumulate into F_A, return Exc, xc-update across iterations, grid-matrix rho
columns) on top of libpdfxc, against the reference fixtures."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def param(fx):
    return {"coordinates": [(str(s), tuple(r)) for s, r in zip(fx["symbols"], fx["xyz"])],
            "basis_set": "cc-pVDZ", "xc-update": "yes"}


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_mirror_two_iterations_with_xc_update(water2, fn):
    from proteindf_b200.dfcalcgridx import DfCalcGridX
    calc = DfCalcGridX(param(water2), grid_matrix=water2["grid"])
    PA = water2["PA"]
    F = np.zeros_like(PA)
    calc.calcXCIntegForFockAndEnergy(0.5 * PA, fn, F)
    F2 = np.zeros_like(PA)
    exc = calc.calcXCIntegForFockAndEnergy(0.5 * PA, fn, F2)   # xc-update: rho(P/2) + rho(P/2)
    assert abs(exc - water2[f"{fn}_exc"][0]) <= 1e-8
    assert np.abs(F2 - water2[f"{fn}_vxc"]).max() <= 1e-7
    g = calc.getGridMatrix()
    assert np.abs(g[:, 5:] - water2[f"{fn}_rho"]).max() <= 1e-9
    nel, _ = calc.getWholeDensity()
    assert abs(nel - water2[f"{fn}_nelec_alpha"][0]) <= 1e-9
    calc.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_mirror_energy_gradient_on_reference_grid(fn):
    """energyGradient on the reference's SG-1 gradient grid reproduces the reference's
    result (its AO-centre term; its grid-weight term is zero)."""
    from conftest import golden
    from proteindf_b200.dfcalcgridx import DfCalcGridX
    fx = golden("ref_grad_water.npz")
    grid = np.c_[fx["points"], fx["w_single"] * fx["w_partition"], fx["atom"].astype(np.float64)]
    calc = DfCalcGridX(param(fx), grid_matrix=grid)
    g = calc.energyGradient(fx["PA"], fn)
    ref = fx[f"{fn}_grad_orbital"] + fx[f"{fn}_grad_weight"]
    assert np.abs(g - ref).max() < 1e-11 * np.abs(ref).max()
    calc.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_mirror_open_shell(water2, fn):
    from conftest import golden
    from proteindf_b200.dfcalcgridx import DfCalcGridX
    uks = golden("ref_uks_water2.npz")
    calc = DfCalcGridX(param(water2), grid_matrix=water2["grid"])
    FA, FB = np.zeros_like(uks["PA"]), np.zeros_like(uks["PA"])
    exc = calc.calcXCIntegForFockAndEnergy(uks["PA"], fn, FA, P_B=uks["PB"], F_B=FB)
    assert abs(exc - uks[f"{fn}_exc"][0]) < 1e-11 * abs(uks[f"{fn}_exc"][0])
    assert np.abs(FA - uks[f"{fn}_vxc_a"]).max() < 1e-11
    assert np.abs(FB - uks[f"{fn}_vxc_b"]).max() < 1e-11
    na, nb = calc.getWholeDensity()
    assert abs(na - uks[f"{fn}_nelec_alpha"][0]) < 1e-11 and abs(nb - uks[f"{fn}_nelec_beta"][0]) < 1e-11
    g = calc.getGridMatrix()
    assert g.shape[1] == (13 if fn == "B3LYP" else 7)
    calc.close()
