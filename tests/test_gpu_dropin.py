"""The drop-in at the C++ class level: DfCalcGridX_B200 (proteindf_b200/host)
beside the reference DfCalcGridX, both driven through the reference's own
matrix classes, parameter set and grid-matrix files for two SCF iterations
(the second with xc-update, so the rho columns written by the first are read
back). Built as oracle/_ref/pdfxc_dropin from the reference sources."""
import numpy as np
import pytest

from conftest import shell_table
from oracle import refio

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not refio.dropin_available(), reason="oracle/_ref/pdfxc_dropin not built")
@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_dfcalcgridx_b200_matches_reference_class(tmp_path, water2, fn):
    from proteindf_b200 import basis, systems
    syms = [str(s) for s in water2["symbols"]]
    g = water2["grid"][:3000]
    r = refio.run_dropin(str(tmp_path), syms, systems.nuclear_charges(syms), water2["xyz"],
                         basis.load_basis("cc-pVDZ"), fn, g, water2["PA"])
    n = shell_table(water2).nao
    for it in (1, 2):
        e_ref, e_b = r[f"ref_exc{it}"][0], r[f"b200_exc{it}"][0]
        v_ref, v_b = r[f"ref_vxc{it}"].reshape(n, n), r[f"b200_vxc{it}"].reshape(n, n)
        assert abs(e_ref - e_b) <= 1e-8, (it, e_ref, e_b)
        assert np.abs(v_ref - v_b).max() <= 1e-7, it


@pytest.mark.skipif(not refio.dropin_available(), reason="oracle/_ref/pdfxc_dropin not built")
@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_energy_gradient_matches_reference_class(tmp_path, fn):
    """DfCalcGridX_B200::energyGradient against DfCalcGridX::energyGradient on one
    H2O (each class builds the SG-1 gradient grid itself)."""
    from proteindf_b200 import basis, systems
    syms, xyz = systems.water_cluster(1, seed=0)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    PA = 0.5 * systems.density_matrix(sh.nao, 5, seed=0)
    r = refio.run_dropin_grad(str(tmp_path), syms, systems.nuclear_charges(syms), xyz,
                              basis.load_basis("cc-pVDZ"), fn, PA)
    ref, b200, won = r["ref_grad"], r["b200_grad"], r["b200_grad_weight_on"]
    assert np.abs(ref - b200).max() < 1e-11 * np.abs(ref).max()
    # the weight term moves the result, and the total stays translation invariant
    assert np.abs(won - b200).max() > 1e-8
    assert np.abs(won.reshape(-1, 3).sum(axis=0)).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.skipif(not refio.dropin_available(), reason="oracle/_ref/pdfxc_dropin not built")
@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_open_shell_overloads_match_reference_class(tmp_path, water2, fn):
    """The P_A, P_B overloads of DfCalcGridX_B200 against the reference class, two SCF
    iterations through the grid-matrix files (the second with xc-update)."""
    from conftest import golden
    from proteindf_b200 import basis, systems
    uks = golden("ref_uks_water2.npz")
    syms = [str(s) for s in water2["symbols"]]
    g = water2["grid"][:3000]
    r = refio.run_dropin_uks(str(tmp_path), syms, systems.nuclear_charges(syms), water2["xyz"],
                             basis.load_basis("cc-pVDZ"), fn, g, uks["PA"], uks["PB"])
    n = shell_table(water2).nao
    for it in (1, 2):
        e_ref, e_b = r[f"ref_exc{it}"][0], r[f"b200_exc{it}"][0]
        assert abs(e_ref - e_b) <= 1e-10 * abs(e_ref), (it, e_ref, e_b)
        for spin in ("a", "b"):
            v_ref, v_b = r[f"ref_vxc{spin}{it}"].reshape(n, n), r[f"b200_vxc{spin}{it}"].reshape(n, n)
            assert np.abs(v_ref - v_b).max() <= 1e-10, (it, spin)
