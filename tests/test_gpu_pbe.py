"""PBE on the GPU (not in the reference; parity unpinned): the device's dual-number
PBE against the oracle's complex-step PBE through whole builds (closed and open
shell), and the 30-atom PBE configuration's finite-difference checks of the XC
nuclear gradient and of Vxc = dExc/dP. Tolerances: 1e-12 relative (Exc) and
1e-12 absolute (Vxc) between two FP64 implementations; central differences
(h = 1e-4 bohr) 2e-6 of the largest gradient component."""
import numpy as np
import pytest

from conftest import golden, shell_table
from oracle import oracle
from proteindf_b200 import basis, grids, systems

pytestmark = pytest.mark.gpu


def test_pbe_closed_and_open_shell_vs_oracle(water2):
    from proteindf_b200.xc import XcEngine
    sh = shell_table(water2)
    g = water2["grid"]
    eng = XcEngine(device=0)
    eng.set_system(sh)
    eng.set_grid(g[:, :4], g[:, 4].astype(np.int32))
    exc, nel, V = eng.build_vxc("PBE", water2["PA"])
    o = oracle.xc("PBE", sh, g[:, :4], water2["PA"])
    assert abs(exc - o["exc"]) < 1e-12 * abs(o["exc"])
    assert np.abs(V - o["vxc"]).max() < 1e-12
    uks = golden("ref_uks_water2.npz")
    e2, na, nb, FA, FB = eng.build_vxc_uks("PBE", uks["PA"], uks["PB"])
    ou = oracle.xc_uks("PBE", sh, g[:, :4], uks["PA"], uks["PB"])
    assert abs(e2 - ou["exc"]) < 1e-12 * abs(ou["exc"])
    assert np.abs(FA - ou["vxc_a"]).max() < 1e-12 and np.abs(FB - ou["vxc_b"]).max() < 1e-12
    eng.close()


def test_pbe_mixed_path_vs_fp64(water2):
    from proteindf_b200.xc import XcEngine
    sh = shell_table(water2)
    g = water2["grid"]
    out = []
    for prec in ("fp64", "mixed"):
        eng = XcEngine(device=0, precision=prec, split_terms=10)
        eng.set_system(sh)
        eng.set_grid(g[:, :4], g[:, 4].astype(np.int32))
        out.append(eng.build_vxc("PBE", water2["PA"]))
        eng.close()
    (e64, _, V64), (em, _, Vm) = out
    assert abs(em - e64) < 1e-8 * abs(e64)
    assert np.abs(Vm - V64).max() < 1e-7 * np.abs(V64).max()


@pytest.fixture(scope="module")
def chain30():
    syms, xyz = systems.peptide_chain(30, seed=11)
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    b = basis.load_basis("cc-pVDZ")
    pts, ws, own = grids.molecular_grid(xyz, Z, **grids.PRESETS["USER-75x302"])
    brad = np.array([grids.BECKE_RADIUS[z] for z in Z])
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 60, seed=12)
    return dict(syms=syms, xyz=xyz, b=b, pts=pts, ws=ws, own=own, brad=brad, sh=sh, PA=PA)


def test_pbe_gradient_finite_difference_chain30(chain30):
    """The PBE configuration: 30-atom chain, cc-pVDZ (standing in for the absent
    6-31G*), USER 75x302 grid with Becke partitioning; AO-centre + grid-weight terms
    against central differences of the GPU energy on 10 seeded Cartesian coordinates."""
    from proteindf_b200.xc import XcEngine
    c = chain30
    d = c["pts"] - c["xyz"][c["own"]]
    eng = XcEngine(device=0)

    def energy(X):
        eng.set_system(basis.ShellTable(c["syms"], X, c["b"]))
        P = X[c["own"]] + d
        w = eng.becke_weights(P, c["own"], c["ws"], c["brad"])
        eng.set_grid(np.c_[P, w], c["own"])
        return eng.build_vxc("PBE", c["PA"])[0]

    eng.set_system(c["sh"])
    w = eng.becke_weights(c["pts"], c["own"], c["ws"], c["brad"])
    eng.set_grid(np.c_[c["pts"], w], c["own"])
    go, gw, _ = eng.xc_gradient("PBE", c["PA"], w_single=c["ws"], becke_radius=c["brad"])
    g = go + gw
    rng = np.random.default_rng(13)
    h = 1e-4
    worst = 0.0
    for a, k in zip(rng.integers(0, len(c["xyz"]), 10), rng.integers(0, 3, 10)):
        X1, X2 = c["xyz"].copy(), c["xyz"].copy()
        X1[a, k] += h
        X2[a, k] -= h
        worst = max(worst, abs(g[a, k] - (energy(X1) - energy(X2)) / (2 * h)))
    eng.close()
    assert worst < 2e-6 * np.abs(g).max(), worst


def test_pbe_vxc_is_the_density_derivative_chain30(chain30):
    """dExc/dPA on 20 seeded entries (h = 1e-5, PA kept symmetric) against Vxc:
    2 Vxc_ii on the diagonal, 4 Vxc_ij off it (both spins move with PA)."""
    from proteindf_b200.xc import XcEngine
    c = chain30
    eng = XcEngine(device=0)
    eng.set_system(c["sh"])
    w = eng.becke_weights(c["pts"], c["own"], c["ws"], c["brad"])
    eng.set_grid(np.c_[c["pts"], w], c["own"])
    _, _, V = eng.build_vxc("PBE", c["PA"])
    rng = np.random.default_rng(14)
    h = 1e-5
    n = c["sh"].nao
    for i, j in zip(rng.integers(0, n, 20), rng.integers(0, n, 20)):
        E = []
        for s in (1, -1):
            P = c["PA"].copy()
            P[i, j] += s * h
            if i != j:
                P[j, i] += s * h
            E.append(eng.build_vxc("PBE", P)[0])
        fd = (E[0] - E[1]) / (2 * h)
        want = V[i, j] * (2.0 if i == j else 4.0)
        assert abs(fd - want) < 1e-7 * max(1.0, np.abs(V).max()), (i, j, fd, want)
    eng.close()
