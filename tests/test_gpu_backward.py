"""The hand-written adjoint of Exc(P, R) (pdfxc_xc_backward) on the differentiation
configuration: a 30-atom chain built as the 100-atom one (seed 21), the 6-31G*-shaped
stand-in basis (cc-pVDZ without the hydrogen p shell; 6-31G* is not in the reference's
library), PBE, USER 75 x 302 grid with Becke partitioning, P_A from 60 occupied orbitals.

* dExc/dP from the backward kernel equals the forward build's Vxc (absolute 1e-12: the same
  FP64 quantities through other kernels).
* Through the torch.autograd.Function wrapper (proteindf_b200.autograd.XcEnergy), the
  gradients match central finite differences of the GPU forward energy to an absolute 1e-6:
  h = 1e-4 bohr on 10 seeded Cartesian coordinates (the grid moves with the atoms and the
  Becke weights are recomputed), h = 1e-5 on 20 seeded P_A entries perturbed symmetrically
  (P_A[i, j] and P_A[j, i] together, so the difference measures the sum of both entries'
  derivatives).
* The cotangent scales every output.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_TOL = 1e-6


@pytest.fixture(scope="module")
def cfg3():
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.autograd import MovingGridSystem
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(30, seed=21)
    b = basis.load_basis("cc-pVDZ-noHp")
    sh = basis.ShellTable(syms, xyz, b)
    pts, ws, own = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["USER-75x302"])
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    PA = 0.5 * systems.density_matrix(sh.nao, 60, seed=22)
    eng = XcEngine(device=0)
    system = MovingGridSystem(eng, syms, xyz, b, pts, ws, own, brad, "PBE")
    yield dict(syms=syms, xyz=xyz, sh=sh, PA=PA, system=system, eng=eng, ws=ws, brad=brad)
    eng.close()


def test_backward_dexc_dP_equals_forward_vxc(cfg3):
    c = cfg3
    c["system"].place(c["xyz"])
    exc, _, V = c["eng"].build_vxc("PBE", c["PA"])
    dP, go, gw, e2 = c["eng"].xc_backward("PBE", c["PA"], w_single=c["ws"], becke_radius=c["brad"])
    dv = np.abs(dP - V).max()
    print(f"cfg3 PBE: {c['sh'].nao} AOs, Exc {exc:.10f}; max|dExc/dP (backward) - Vxc (forward)| = {dv:.3e}")
    assert dv <= 1e-12 and abs(e2 - exc) <= 1e-12 * abs(exc)
    assert np.array_equal(dP, dP.T)
    go1, gw1, _ = c["eng"].xc_gradient("PBE", c["PA"], w_single=c["ws"], becke_radius=c["brad"])
    assert np.abs(go - go1).max() <= 1e-12 and np.abs(gw - gw1).max() <= 1e-12


def test_backward_cotangent_scales_every_output(cfg3):
    c = cfg3
    c["system"].place(c["xyz"])
    a = c["eng"].xc_backward("PBE", c["PA"], dexc=1.0, w_single=c["ws"], becke_radius=c["brad"])
    b = c["eng"].xc_backward("PBE", c["PA"], dexc=-2.5, w_single=c["ws"], becke_radius=c["brad"])
    for x, y in zip(a[:3], b[:3]):
        assert np.abs(y + 2.5 * x).max() <= 1e-12 * max(1.0, np.abs(x).max())


def test_autograd_matches_finite_differences(cfg3):
    import torch
    from proteindf_b200.autograd import XcEnergy
    c = cfg3
    system = c["system"]
    PA = torch.tensor(c["PA"], requires_grad=True)
    R = torch.tensor(c["xyz"], requires_grad=True)
    E = XcEnergy.apply(PA, R, system)
    E.backward()
    gP, gR = PA.grad.numpy(), R.grad.numpy()
    rng = np.random.default_rng(23)
    h = 1e-4
    errR = []
    for a, k in zip(rng.integers(0, len(c["xyz"]), 10), rng.integers(0, 3, 10)):
        X1, X2 = c["xyz"].copy(), c["xyz"].copy()
        X1[a, k] += h
        X2[a, k] -= h
        fd = (system.energy(c["PA"], X1) - system.energy(c["PA"], X2)) / (2 * h)
        errR.append(abs(gR[a, k] - fd))
    h = 1e-5
    n = c["sh"].nao
    errP = []
    for i, j in zip(rng.integers(0, n, 20), rng.integers(0, n, 20)):
        E2 = []
        for s in (1, -1):
            P = c["PA"].copy()
            P[i, j] += s * h
            if i != j:
                P[j, i] += s * h
            E2.append(system.energy(P, c["xyz"]))
        fd = (E2[0] - E2[1]) / (2 * h)
        want = gP[i, j] + (gP[j, i] if i != j else 0.0)
        errP.append(abs(want - fd))
    print(f"cfg3 PBE finite differences: max |dE/dR - FD| = {max(errR):.3e} (h = 1e-4 bohr, 10 coordinates, "
          f"max |dE/dR| {np.abs(gR).max():.3e}); max |dE/dP_A - FD| = {max(errP):.3e} (h = 1e-5, 20 entries)")
    assert max(errR) <= FD_TOL and max(errP) <= FD_TOL
