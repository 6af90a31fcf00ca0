"""Density at arbitrary points (pdfxc_density, DfCalcGridX::gridDensity) on the GPU against
the reference's gridDensity (tests/golden/ref_density_water2.npz), the CPU oracle, and the
drop-in class. The FP64 path screens AOs below 1e-14, so values agree to ~1e-13."""
import numpy as np
import pytest

from conftest import golden, shell_table
from oracle import refio

pytestmark = pytest.mark.gpu


def _engine(fx, **kw):
    from proteindf_b200.xc import XcEngine
    e = XcEngine(device=0, **kw)
    e.set_system(shell_table(fx))
    return e


def test_density_vs_reference():
    fx = golden("ref_density_water2.npz")
    e = _engine(fx)
    rho = e.density(fx["P"], fx["points"])
    assert np.all(np.abs(rho - fx["rho"]) <= 1e-12 * np.maximum(1.0, np.abs(fx["rho"])))
    assert np.all(rho[-20:] == 0.0)  # far points: no shell reaches them
    assert e.density(fx["P"], np.zeros((0, 3))).shape == (0,)
    e.close()


def test_density_leaves_the_build_grid_alone(water2):
    """A density call between two builds changes neither build (private grid), and the
    mixed-precision context answers in FP64 too."""
    fx = golden("ref_density_water2.npz")
    for precision in ("fp64", "mixed"):
        e = _engine(water2, precision=precision)
        e.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
        exc0, _, V0 = e.build_vxc("B3LYP", water2["PA"])
        rho = e.density(fx["P"], fx["points"])
        exc1, _, V1 = e.build_vxc("B3LYP", water2["PA"])
        # equal up to the summation order of the FP64 atomics
        assert abs(exc1 - exc0) <= 1e-12 and np.abs(V1 - V0).max() <= 1e-13
        assert np.all(np.abs(rho - fx["rho"]) <= 1e-12 * np.maximum(1.0, np.abs(fx["rho"])))
        # xc-update still finds the build's own densities
        exc2, _, _ = e.build_vxc("B3LYP", np.zeros_like(water2["PA"]), incremental=True)
        assert abs(exc2 - exc0) <= 1e-12
        e.close()


def test_density_chain_vs_oracle():
    """A 30-atom chain, 20,000 points spread over and around it (several blocks, ragged
    last block) against the oracle's AO values."""
    from oracle import oracle
    from proteindf_b200 import basis, systems
    syms, xyz = systems.peptide_chain(30, seed=7)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P = 0.5 * systems.density_matrix(sh.nao, 40, seed=7)
    rng = np.random.default_rng(7)
    pts = xyz[rng.integers(0, len(xyz), 20000)] + rng.normal(scale=1.5, size=(20000, 3))
    from proteindf_b200.xc import XcEngine
    e = XcEngine(device=0)
    e.set_system(sh)
    rho = e.density(P, pts)
    phi, _ = oracle.aos(sh, pts)
    ref = np.einsum("pi,ij,pj->p", phi, P, phi)
    assert np.all(np.abs(rho - ref) <= 1e-12 * np.maximum(1.0, np.abs(ref)))
    e.close()


def test_python_class_grid_density():
    from proteindf_b200.dfcalcgridx import DfCalcGridX
    fx = golden("ref_density_water2.npz")
    syms = [str(s) for s in fx["symbols"]]
    c = DfCalcGridX({"coordinates": list(zip(syms, fx["xyz"])), "basis_set": "cc-pVDZ"})
    one = c.gridDensity(fx["P"], fx["points"][3])
    many = c.gridDensities(fx["P"], fx["points"])
    assert one == many[3]
    assert np.all(np.abs(many - fx["rho"]) <= 1e-12 * np.maximum(1.0, np.abs(fx["rho"])))
    c.close()


def test_density_needs_a_system():
    from proteindf_b200.xc import XcEngine
    e = XcEngine(device=0)
    with pytest.raises(RuntimeError, match="set_system"):
        e.density(np.eye(2), np.zeros((1, 3)))
    e.close()


@pytest.mark.skipif(not refio.dropin_available(), reason="oracle/_ref/pdfxc_dropin not built")
def test_dfcalcgridx_b200_grid_density_matches_reference_class(tmp_path):
    """DfCalcGridX_B200::gridDensity (per point) and gridDensities (batched) beside the
    reference class's gridDensity on the same parameter set."""
    from proteindf_b200 import basis, systems
    fx = golden("ref_density_water2.npz")
    syms = [str(s) for s in fx["symbols"]]
    r = refio.run_dropin_density(str(tmp_path), syms, systems.nuclear_charges(syms), fx["xyz"],
                                 basis.load_basis("cc-pVDZ"), fx["P"], fx["points"])
    ref = r["ref_rho"]
    assert np.all(np.abs(r["b200_rho"] - ref) <= 1e-12 * np.maximum(1.0, np.abs(ref)))
    assert np.array_equal(r["b200_rho_single"], r["b200_rho"][:8])
