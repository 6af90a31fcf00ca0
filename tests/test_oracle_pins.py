"""The CPU oracle pinned against the reference: its own known-answer tests and
outputs of the reference engine itself (tests/golden/*, made by
tests/golden/make_ref_fixtures.py from oracle/_ref/pdfxc_ref)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, shell_table
from oracle import oracle, refio

KEYS = ["f", "vA", "vB", "vgAA", "vgAB", "vgBB"]


def kat_cases():
    return json.load(open(os.path.join(GOLDEN, "functional_kats.json")))


@pytest.mark.parametrize("case", kat_cases(), ids=lambda c: f"{c['component']}-{c['test']}")
def test_functional_known_answers(case):
    """src/unit_test/DfFunctional_*Test.cpp, at each test's own tolerance."""
    if case["component"] == "B3LYP":
        o = oracle.functional("B3LYP", *case["inputs"])[0]
    else:
        o = oracle.component(case["component"], *case["inputs"])
    for k, v in case["expected"].items():
        assert abs(o[KEYS.index(k)] - v) <= case["tol"], (k, v, o[KEYS.index(k)])


@pytest.mark.parametrize("fn", ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"])
def test_functionals_vs_reference_engine(fn):
    fx = golden("ref_functionals.npz")
    inp = fx["inputs"]
    ref = fx[fn]
    got = oracle.functional(fn, *inp.T)
    # open-shell overload: f, vA, vB, vgAA, vgAB, vgBB
    scale = np.maximum(np.abs(ref[:, :6]), 1e-300)
    assert np.all(np.abs(got - ref[:, :6]) <= 1e-12 * scale + 1e-300)
    # closed-shell overloads (rhoB = rhoA, gammas equal) used by the grid path
    ra, gaa = inp[:, 0], inp[:, 2]
    rks = oracle.functional(fn, ra, ra, gaa, gaa, gaa)
    for col, ref_col in ((0, 6), (1, 7), (3, 8), (4, 9)):
        r = ref[:, ref_col]
        assert np.all(np.abs(rks[:, col] - r) <= 1e-12 * np.abs(r) + 1e-300), (fn, col)


@pytest.mark.parametrize("name,fns", [("ref_water2.npz", ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"]),
                                      ("ref_chain12.npz", ["SVWN", "B3LYP"])])
def test_quadrature_vs_reference_engine(name, fns):
    fx = golden(name)
    sh = shell_table(fx)
    grid = fx["grid"]
    for fn in fns:
        r = oracle.xc(fn, sh, grid[:, :4], fx["PA"])
        assert abs(r["exc"] - fx[f"{fn}_exc"][0]) < 1e-12, fn
        assert np.abs(r["vxc"] - fx[f"{fn}_vxc"]).max() < 1e-12, fn
        assert np.abs(r["rho"] - fx[f"{fn}_rho"]).max() < 1e-10, fn
        assert abs(r["nelec_alpha"] - fx[f"{fn}_nelec_alpha"][0]) < 1e-10


def test_basis_normalisation_and_order(water2):
    """Normalised contraction coefficients and AO order of TlOrbitalInfo."""
    sh = shell_table(water2)
    assert np.array_equal(sh.ao_atom(), water2["ao_atom"].astype(np.int32))
    assert np.array_equal(sh.ao_type(), water2["ao_type"].astype(np.int32))
    exps, coefs = [], []
    for s in range(sh.nshell):
        p0, n = sh.shell_p0[s], sh.shell_nprim[s]
        for _ in range(2 * sh.shell_l[s] + 1):
            exps.extend(sh.prim_exp[p0:p0 + n])
            coefs.extend(sh.prim_coef[p0:p0 + n])
    assert np.allclose(exps, water2["ao_exp"], rtol=0, atol=0)
    assert np.allclose(coefs, water2["ao_coef"], rtol=1e-14, atol=0)


def test_ao_values(water2):
    sh = shell_table(water2)
    phi, dphi = oracle.aos(sh, water2["grid"][:5, :3])
    assert np.abs(phi.ravel() - water2["phi"]).max() < 1e-14
    assert np.abs(dphi.ravel() - water2["dphi"]).max() < 1e-13


def test_becke_weights(water2):
    fx = water2
    brad = fx["radii"][:, 1]
    fac = oracle.becke(fx["xyz"], brad, fx["becke_points"], fx["becke_atom"])
    w = fx["becke_w_single"] * fac
    assert np.abs(w - fx["becke_w_final"]).max() <= 1e-15 * np.abs(fx["becke_w_single"]).max()


def test_grid_generator_matches_reference(water2):
    """Host grid helper + oracle Becke + weight screening reproduce the reference's grid."""
    from proteindf_b200 import grids
    fx = water2
    z = [1 if s == "H" else 8 for s in fx["symbols"]]
    P, W, A = grids.molecular_grid(fx["xyz"], z, **grids.PRESETS["USER-75x302"])
    fac = oracle.becke(fx["xyz"], fx["radii"][:, 1], P, A)
    P2, W2, A2 = grids.screen_by_weight(P, W * fac, A)
    assert len(W2) == int(fx["grid_npts_full"])
    assert abs(W2.sum() - float(fx["grid_wsum_full"])) < 1e-9 * abs(W2.sum())


@pytest.mark.skipif(not refio.ref_available(), reason="reference harness not built here")
def test_oracle_vs_live_reference_random_system(tmp_path):
    """A fresh random case through the reference engine (when its harness is present)."""
    from proteindf_b200 import basis, systems
    syms, xyz = systems.water_cluster(3, seed=11)
    b = basis.load_basis("cc-pVDZ")
    sh = basis.ShellTable(syms, xyz, b)
    rng = np.random.default_rng(5)
    g = np.concatenate([xyz[rng.integers(len(xyz), size=800)] + rng.normal(scale=1.2, size=(800, 3)),
                        rng.uniform(1e-3, 1.0, size=(800, 1)), np.zeros((800, 1))], axis=1)
    PA = 0.5 * systems.density_matrix(sh.nao, 15, seed=5)
    r = refio.run_xc(str(tmp_path), syms, systems.nuclear_charges(syms), xyz, b, "B3LYP", g, PA)
    o = oracle.xc("B3LYP", sh, g[:, :4], PA)
    assert abs(r["exc"][0] - o["exc"]) < 1e-12
    assert np.abs(r["vxc"].reshape(sh.nao, -1) - o["vxc"]).max() < 1e-12


@pytest.mark.parametrize("fn", ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"])
def test_oracle_open_shell_vs_reference(water2, fn):
    """The P_A, P_B overloads (src/libpdf/DfCalcGridX.cpp:2292-2328) on the water-dimer
    grid sample: Exc, Vxc_A, Vxc_B, electron counts and rho columns."""
    fx = golden("ref_uks_water2.npz")
    o = oracle.xc_uks(fn, shell_table(water2), water2["grid"][:, :4], fx["PA"], fx["PB"])
    assert abs(o["exc"] - fx[f"{fn}_exc"][0]) < 1e-13 * abs(fx[f"{fn}_exc"][0])
    assert np.abs(o["vxc_a"] - fx[f"{fn}_vxc_a"]).max() < 1e-14
    assert np.abs(o["vxc_b"] - fx[f"{fn}_vxc_b"]).max() < 1e-14
    assert abs(o["nelec_alpha"] - fx[f"{fn}_nelec_alpha"][0]) < 1e-13
    assert abs(o["nelec_beta"] - fx[f"{fn}_nelec_beta"][0]) < 1e-13
    if f"{fn}_rho" in fx:
        ref = fx[f"{fn}_rho"]
        assert np.all(np.abs(o["rho"] - ref) <= 1e-13 * np.maximum(1.0, np.abs(ref)))


def test_oracle_ss_weights_vs_reference(water2):
    """Stratmann-Scuseria partition (src/libpdf/DfGenerateGrid.cpp:1878-1956) on the
    reference's own SSWeight grid of the water dimer."""
    fx = golden("ref_ss_water2.npz")
    fac = oracle.ss(water2["xyz"], fx["points"], fx["atom"])
    assert np.abs(fx["w_single"] * fac - fx["w_final"]).max() <= 1e-15 * np.abs(fx["w_single"]).max()


def test_oracle_density_at_points_vs_reference():
    """rho = phi^T P phi at arbitrary points (DfCalcGridX::gridDensity) from the oracle's AO
    values against the reference's gridDensity on the committed point set."""
    fx = golden("ref_density_water2.npz")
    phi, _ = oracle.aos(shell_table(fx), fx["points"])
    rho = np.einsum("pi,ij,pj->p", phi, fx["P"], phi)
    assert np.all(np.abs(rho - fx["rho"]) <= 1e-12 * np.maximum(1.0, np.abs(fx["rho"])))
    assert np.all(fx["rho"][-20:] == 0.0)  # far points: every primitive beyond the a r^2 > 30 cut


def test_oracle_becke_leaves_dummy_atoms_out():
    """The reference's Becke product skips partner atoms of atomic number <= 0 (dummy atoms X,
    src/libpdf/DfGenerateGrid.cpp:2056); a dummy atom between two waters changes the weights
    by up to 0.47 if it is counted."""
    fx = golden("ref_becke_ghost_water2.npz")
    syms = [str(s) for s in fx["symbols"]]
    ghost = np.array([s == "X" for s in syms])
    brad = fx["radii"][:, 1]
    ref = fx["w_final"] / fx["w_single"]
    f = oracle.becke(fx["xyz"], brad, fx["points"], fx["atom"], ghost=ghost)
    assert np.all(np.abs(f - ref) <= 1e-14 * np.maximum(np.abs(ref), 1e-300) + 1e-300)
    f_all = oracle.becke(fx["xyz"], brad, fx["points"], fx["atom"])
    assert np.abs(f_all - ref).max() > 0.1


def test_host_grid_recipe_reproduces_water8_reference_grid():
    """The (H2O)8 configuration's whole USER 75 x 302 Becke grid: the host recipe
    (proteindf_b200.grids) with the oracle's Becke weights and the 1e-16 weight screen gives
    the reference's point count and weight sum."""
    from proteindf_b200 import basis, grids
    fx = golden("ref_water8_user75x302.npz")
    sh = basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"], basis.load_basis("cc-pVDZ"))
    P, W, A = grids.molecular_grid(fx["xyz"], sh.atom_z, **grids.PRESETS["USER-75x302"])
    w = W * oracle.becke(fx["xyz"], fx["radii"][:, 1], P, A)
    keep = np.abs(w) > 1e-16
    assert abs(int(keep.sum()) - int(fx["grid_npts"])) <= 5
    assert abs(w[keep].sum() - float(fx["grid_wsum"])) <= 1e-12 * float(fx["grid_wsum"])
