"""XC nuclear gradient on the GPU (pdfxc_xc_gradient) against the reference, the
CPU oracle and finite differences of the GPU energy.

Tolerances: the AO-centre term against the reference's own output on its SG-1 grid
1e-11 of the largest component (FP64, different summation order); the weight term
against the oracle 1e-11; central differences (h = 1e-4 bohr) 2e-6 of the
largest gradient component, the truncation error of the difference quotient.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle
from proteindf_b200 import basis, grids, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gradwater():
    return golden("ref_grad_water.npz")


def _engine(sh):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(device=0)
    eng.set_system(sh)
    return eng


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_orbital_term_vs_reference(gradwater, fn):
    fx = gradwater
    sh = basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"], basis.load_basis("cc-pVDZ"))
    eng = _engine(sh)
    w = fx["w_single"] * fx["w_partition"]
    eng.set_grid(np.c_[fx["points"], w], fx["atom"].astype(np.int32))
    go, gw, exc = eng.xc_gradient(fn, fx["PA"])
    eng.close()
    ref = fx[f"{fn}_grad_orbital"]
    assert gw is None
    assert abs(exc - float(fx[f"{fn}_exc"][0])) < 1e-11 * abs(float(fx[f"{fn}_exc"][0]))
    assert np.abs(go - ref).max() < 1e-11 * np.abs(ref).max()


def _small_system(nwater=2, seed=1, nrad=30, nang=86):
    syms, xyz = systems.water_cluster(nwater, seed=seed)
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    pts, ws, own = grids.molecular_grid(xyz, Z, nrad=nrad, nang=nang, radial="GC", mapping="TA", pruning=True)
    brad = np.array([grids.BECKE_RADIUS[z] for z in Z])
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    return syms, xyz, pts, ws, own, brad, sh


@pytest.mark.parametrize("fn", ["SVWN", "BLYP"])
def test_both_terms_vs_oracle(fn):
    syms, xyz, pts, ws, own, brad, sh = _small_system()
    PA = 0.5 * systems.density_matrix(sh.nao, 10, seed=2)
    w = ws * oracle.becke(xyz, brad, pts, own)
    eng = _engine(sh)
    eng.set_grid(np.c_[pts, w], own)
    go, gw, exc = eng.xc_gradient(fn, PA, w_single=ws, becke_radius=brad)
    eng.close()
    o = oracle.xc_grad(fn, sh, np.c_[pts, w], own, PA)
    ow = oracle.becke_grad(xyz, brad, pts, own, ws * o["f"])
    assert abs(exc - o["exc"]) < 1e-11 * abs(o["exc"])
    assert np.abs(go - o["grad"]).max() < 1e-11 * np.abs(o["grad"]).max()
    assert np.abs(gw - ow).max() < 1e-11 * max(np.abs(ow).max(), 1e-300)
    assert np.abs(gw.sum(axis=0)).max() < 1e-10 * np.abs(ow).max()


def test_total_gradient_finite_difference_chain():
    """30-atom chain (cc-pVDZ, USER 75x302 GC-TA grid, Becke partition), B3LYP at a
    fixed density: AO-centre + grid-weight terms against central differences of
    the GPU energy on 10 seeded Cartesian coordinates, the grid moving with the atoms."""
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(30, seed=11)
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    b = basis.load_basis("cc-pVDZ")
    pts, ws, own = grids.molecular_grid(xyz, Z, **grids.PRESETS["USER-75x302"])
    brad = np.array([grids.BECKE_RADIUS[z] for z in Z])
    d = pts - xyz[own]
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 60, seed=12)
    eng = XcEngine(device=0)

    def energy(X):
        eng.set_system(basis.ShellTable(syms, X, b))
        P = X[own] + d
        w = eng.becke_weights(P, own, ws, brad)
        eng.set_grid(np.c_[P, w], own)
        return eng.build_vxc("B3LYP", PA)[0]

    eng.set_system(sh)
    w = eng.becke_weights(pts, own, ws, brad)
    eng.set_grid(np.c_[pts, w], own)
    go, gw, _ = eng.xc_gradient("B3LYP", PA, w_single=ws, becke_radius=brad)
    g = go + gw
    rng = np.random.default_rng(13)
    h = 1e-4
    worst = 0.0
    for a, k in zip(rng.integers(0, len(xyz), 10), rng.integers(0, 3, 10)):
        X1, X2 = xyz.copy(), xyz.copy()
        X1[a, k] += h
        X2[a, k] -= h
        fd = (energy(X1) - energy(X2)) / (2 * h)
        worst = max(worst, abs(g[a, k] - fd))
    eng.close()
    assert worst < 2e-6 * np.abs(g).max(), worst


def test_vxc_is_the_density_derivative():
    """dExc/dPA_ij by central differences (h = 1e-5, PA perturbed symmetrically) against
    Vxc. The closed-shell energy moves both spin densities with PA, so dExc/dPA_ii =
    2 Vxc_ii and, with PA_ij and PA_ji moving together, 4 Vxc_ij off the diagonal (in
    terms of the total density P = 2 PA: Vxc_ii and 2 Vxc_ij)."""
    syms, xyz, pts, ws, own, brad, sh = _small_system(nwater=2, seed=3)
    PA = 0.5 * systems.density_matrix(sh.nao, 10, seed=4)
    w = ws * oracle.becke(xyz, brad, pts, own)
    eng = _engine(sh)
    eng.set_grid(np.c_[pts, w], own)
    _, _, V = eng.build_vxc("B3LYP", PA)
    rng = np.random.default_rng(5)
    h = 1e-5
    for i, j in zip(rng.integers(0, sh.nao, 20), rng.integers(0, sh.nao, 20)):
        E = []
        for s in (1, -1):
            P = PA.copy()
            P[i, j] += s * h
            if i != j:
                P[j, i] += s * h
            E.append(eng.build_vxc("B3LYP", P)[0])
        fd = (E[0] - E[1]) / (2 * h)
        want = V[i, j] * (2.0 if i == j else 4.0)
        assert abs(fd - want) < 1e-7 * max(1.0, np.abs(V).max()), (i, j, fd, want)
    eng.close()


def test_gradient_needs_owner_atoms(gradwater):
    from proteindf_b200.xc import XcEngine
    fx = gradwater
    sh = basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"], basis.load_basis("cc-pVDZ"))
    eng = XcEngine(device=0)
    eng.set_system(sh)
    eng.set_grid(np.c_[fx["points"], fx["w_single"] * fx["w_partition"]])
    with pytest.raises(RuntimeError, match="owner"):
        eng.xc_gradient("SVWN", fx["PA"])
    eng.close()


def test_weight_term_rows_in_device_memory_match_shared(monkeypatch):
    """The weight term's two forms (atom rows in shared memory, in device memory) give the same
    gradient on the same system (1e-12 relative: only the order of the atomic sums differs)."""
    syms, xyz, pts, ws, own, brad, sh = _small_system(nwater=3, seed=4)
    PA = 0.5 * systems.density_matrix(sh.nao, 15, seed=5)
    eng = _engine(sh)
    eng.set_grid(np.c_[pts, eng.becke_weights(pts, own, ws, brad)], own)
    _, gw_sm, _ = eng.xc_gradient("BLYP", PA, w_single=ws, becke_radius=brad)
    monkeypatch.setenv("PDFXC_GRAD_WEIGHT_ROWS", "dram")
    _, gw_dram, _ = eng.xc_gradient("BLYP", PA, w_single=ws, becke_radius=brad)
    eng.close()
    print(f"weight term, rows in shared vs device memory: max diff {np.abs(gw_dram - gw_sm).max():.3e} "
          f"(max |g| {np.abs(gw_sm).max():.3e})")
    assert np.abs(gw_dram - gw_sm).max() <= 1e-12 * np.abs(gw_sm).max()


def test_weight_term_beyond_400_atoms_finite_difference():
    """A 420-atom chain (above the shared-memory form's 400 atoms), SVWN, on a seeded sample of
    4000 rows of its USER 75x302 grid that moves with the atoms: the AO-centre plus weight
    terms against central differences of the GPU energy (h = 1e-4 bohr, 4 coordinates), and
    the weight term's sum over atoms (zero: translating the molecule moves its grid along)."""
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(420, seed=31)
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    b = basis.load_basis("cc-pVDZ")
    pts, ws, own = grids.molecular_grid(xyz, Z, **grids.PRESETS["USER-75x302"])
    rng = np.random.default_rng(32)
    rows = np.sort(rng.choice(len(pts), 4000, replace=False))
    pts, ws, own = pts[rows], ws[rows], own[rows]
    brad = np.array([grids.BECKE_RADIUS[z] for z in Z])
    d = pts - xyz[own]
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 200, seed=33)
    eng = XcEngine(device=0)

    def energy(X):
        eng.set_system(basis.ShellTable(syms, X, b))
        P = X[own] + d
        eng.set_grid(np.c_[P, eng.becke_weights(P, own, ws, brad)], own)
        return eng.build_vxc("SVWN", PA)[0]

    energy(xyz)
    go, gw, _ = eng.xc_gradient("SVWN", PA, w_single=ws, becke_radius=brad)
    g = go + gw
    h, worst = 1e-4, 0.0
    for a, k in zip(rng.choice(own, 4), rng.integers(0, 3, 4)):
        X1, X2 = xyz.copy(), xyz.copy()
        X1[a, k] += h
        X2[a, k] -= h
        worst = max(worst, abs(g[a, k] - (energy(X1) - energy(X2)) / (2 * h)))
    eng.close()
    print(f"420 atoms: max |g - FD| = {worst:.3e} (max |g| {np.abs(g).max():.3e}); "
          f"|sum of weight term| = {np.abs(gw.sum(axis=0)).max():.3e}")
    assert np.all(np.isfinite(gw)) and np.abs(gw).max() > 0
    assert worst < 2e-6 * np.abs(g).max()
    assert np.abs(gw.sum(axis=0)).max() < 1e-10 * np.abs(gw).max()
