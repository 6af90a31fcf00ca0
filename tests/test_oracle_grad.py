"""XC nuclear gradient: the CPU oracle against the reference and against finite
differences of its own energy (CPU only).

The reference's gradient (DfCalcGridX::energyGradient, src/libpdf/DfCalcGridX.cpp:
1073-1415) is an AO-centre term plus a grid-weight term. The fixture
tests/golden/ref_grad_water.npz holds both, from the reference itself on its own
SG-1 grid. Its weight term is exactly zero: JGP_t (src/libpdf/DfGenerateGrid.cpp:
2357-2372) returns 0 unless |mu| > 1, which a point never reaches. The weight
term here is the derivative of the partition function itself, pinned by
finite differences.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle
from proteindf_b200 import basis, grids, systems


@pytest.fixture(scope="module")
def gradwater():
    return golden("ref_grad_water.npz")


def _shells(fx, xyz=None):
    return basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"] if xyz is None else xyz,
                            basis.load_basis("cc-pVDZ"))


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_orbital_term_vs_reference(gradwater, fn):
    fx = gradwater
    sh = _shells(fx)
    w = fx["w_single"] * fx["w_partition"]
    o = oracle.xc_grad(fn, sh, np.c_[fx["points"], w], fx["atom"].astype(np.int32), fx["PA"])
    ref = fx[f"{fn}_grad_orbital"]
    assert abs(o["exc"] - float(fx[f"{fn}_exc"][0])) < 1e-12 * abs(float(fx[f"{fn}_exc"][0]))
    assert np.abs(o["grad"] - ref).max() < 1e-12 * np.abs(ref).max()
    # translational invariance of the AO-centre term
    assert np.abs(o["grad"].sum(axis=0)).max() < 1e-12 * np.abs(ref).max()


def test_reference_weight_term_is_zero(gradwater):
    for fn in ("SVWN", "B3LYP"):
        assert np.all(gradwater[f"{fn}_grad_weight"] == 0.0)


def test_sg1_partition_is_size_adjusted_becke(gradwater):
    fx = gradwater
    brad = np.array([grids.BECKE_RADIUS[z] for z in systems.nuclear_charges([str(s) for s in fx["symbols"]])])
    fac = oracle.becke(fx["xyz"], brad, fx["points"], fx["atom"].astype(np.int32), size_adjust=True)
    assert np.abs(fac - fx["w_partition"]).max() <= 1e-15


def _small_grid(syms, xyz):
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    pts, ws, own = grids.molecular_grid(xyz, Z, nrad=24, nang=50, radial="GC", mapping="TA", pruning=False)
    brad = np.array([grids.BECKE_RADIUS[z] for z in Z])
    return pts, ws, own, brad


@pytest.mark.parametrize("size_adjust", [True, False])
def test_weight_term_finite_difference(size_adjust):
    syms, xyz = systems.water_cluster(2, seed=1)
    pts, ws, own, brad = _small_grid(syms, xyz)
    d = pts - xyz[own]
    c = np.random.default_rng(0).uniform(-1, 1, len(pts)) * ws
    g = oracle.becke_grad(xyz, brad, pts, own, c, size_adjust=size_adjust)
    h = 1e-5
    fd = np.zeros_like(g)
    for a in range(len(xyz)):
        for k in range(3):
            e = []
            for s in (1, -1):
                X = xyz.copy()
                X[a, k] += s * h
                e.append(np.dot(c, oracle.becke(X, brad, X[own] + d, own, size_adjust=size_adjust)))
            fd[a, k] = (e[0] - e[1]) / (2 * h)
    # central differences, h = 1e-5 bohr: truncation ~h^2 times third derivatives
    assert np.abs(g - fd).max() < 1e-8 * max(1.0, np.abs(g).max())
    assert np.abs(g.sum(axis=0)).max() < 1e-10 * np.abs(g).max()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_total_gradient_finite_difference(fn):
    """d Exc / dR at fixed density matrix, the grid moving with the atoms:
    AO-centre term + grid-weight term against central differences."""
    syms, xyz = systems.water_cluster(1, seed=2)
    b = basis.load_basis("cc-pVDZ")
    pts, ws, own, brad = _small_grid(syms, xyz)
    d = pts - xyz[own]
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 5, seed=4)

    def energy(X):
        P = X[own] + d
        w = ws * oracle.becke(X, brad, P, own)
        return oracle.xc(fn, basis.ShellTable(syms, X, b), np.c_[P, w], PA)["exc"]

    w = ws * oracle.becke(xyz, brad, pts, own)
    o = oracle.xc_grad(fn, sh, np.c_[pts, w], own, PA)
    g = o["grad"] + oracle.becke_grad(xyz, brad, pts, own, ws * o["f"])
    rng = np.random.default_rng(5)
    h = 1e-4
    for a, k in zip(rng.integers(0, len(xyz), 5), rng.integers(0, 3, 5)):
        X1, X2 = xyz.copy(), xyz.copy()
        X1[a, k] += h
        X2[a, k] -= h
        fd = (energy(X1) - energy(X2)) / (2 * h)
        assert abs(g[a, k] - fd) < 2e-7 * max(1.0, np.abs(g).max()), (a, k, g[a, k], fd)
