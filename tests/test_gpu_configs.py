"""Parity at the benchmark's own configurations, against the reference itself.

* (H2O)8 (O uniform in a 9 A cube, seed 0), cc-pVDZ (192 AOs), the whole USER 75 x 302
  GC-TA Becke grid: the grid is made on the device (pdfxc_generate_grid) and compared with
  the reference's own grid (point count, weight sum); SVWN and B3LYP Exc, electron count and
  Vxc against the reference's DfCalcGridX on its grid (tests/golden/ref_water8_user75x302.npz).
* The 100-atom chain, cc-pVDZ (932 AOs), ULTRA_FINE 99 x 590, B3LYP, 380 occupied orbitals:
  a seeded sample of 20,000 rows of the final grid, built by the reference and here
  (tests/golden/ref_chain100_ultrafine_sample.npz): Exc, electron count, the Vxc diagonal,
  20,000 sampled Vxc entries and checksums of the whole Vxc.

FP64 drop-in: |dExc| <= 1e-8 Eh and max|dVxc| <= 1e-7. INT8 tensor-core path: the mixed
tolerances of the other tests, |dExc|/|Exc| <= 2e-10 and max|dVxc|/max|Vxc| <= 5e-9.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

EXC_TOL, VXC_TOL = 1e-8, 1e-7
OZ_TOL = (2e-10, 5e-9)


def _unpack(p, n):
    V = np.zeros((n, n))
    iu = np.triu_indices(n)
    V[iu] = p
    V.T[iu] = p
    return V


@pytest.fixture(scope="module")
def water8():
    return golden("ref_water8_user75x302.npz")


def _water8_engine(fx, precision):
    from proteindf_b200 import basis, grids
    from proteindf_b200.xc import XcEngine
    sh = basis.ShellTable([str(s) for s in fx["symbols"]], fx["xyz"], basis.load_basis("cc-pVDZ"))
    eng = XcEngine(device=0, precision=precision, split_terms=10)
    eng.set_system(sh)
    npts = eng.generate_grid(fx["radii"][:, 0], partition="Becke", becke_radius=fx["radii"][:, 1],
                             **grids.PRESETS["USER-75x302"])
    return eng, sh, npts


def test_water8_device_grid_is_the_reference_grid(water8):
    eng, sh, npts = _water8_engine(water8, "fp64")
    xyzw, _ = eng.get_grid()
    print(f"(H2O)8 grid: {npts} points (reference {int(water8['grid_npts'])}), "
          f"weight sum {xyzw[:, 3].sum():.12f} (reference {float(water8['grid_wsum']):.12f})")
    # the screen |w| > 1e-16 may differ on points whose weight rounds differently at the threshold
    assert abs(npts - int(water8["grid_npts"])) <= 5
    assert abs(xyzw[:, 3].sum() - float(water8["grid_wsum"])) <= 1e-12 * float(water8["grid_wsum"])
    eng.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_water8_full_grid_fp64_vs_reference(water8, fn):
    eng, sh, _ = _water8_engine(water8, "fp64")
    exc, nel, V = eng.build_vxc(fn, water8["PA"])
    Vr = _unpack(water8[f"{fn}_vxc_upper"], sh.nao)
    dE, dV = abs(exc - water8[f"{fn}_exc"][0]), np.abs(V - Vr).max()
    print(f"(H2O)8 {fn} FP64: |dExc|={dE:.3e} max|dVxc|={dV:.3e} |dN|={abs(nel - water8[f'{fn}_nelec_alpha'][0]):.3e}")
    assert dE <= EXC_TOL and dV <= VXC_TOL
    assert abs(nel - water8[f"{fn}_nelec_alpha"][0]) <= 1e-9
    eng.close()


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_water8_full_grid_int8_vs_reference(water8, fn):
    eng, sh, _ = _water8_engine(water8, "mixed")
    exc, nel, V = eng.build_vxc(fn, water8["PA"])
    Vr = _unpack(water8[f"{fn}_vxc_upper"], sh.nao)
    rE = abs(exc - water8[f"{fn}_exc"][0]) / abs(water8[f"{fn}_exc"][0])
    rV = np.abs(V - Vr).max() / np.abs(Vr).max()
    print(f"(H2O)8 {fn} INT8: |dExc|/|Exc|={rE:.3e} max|dVxc|/max|Vxc|={rV:.3e}")
    assert rE <= OZ_TOL[0] and rV <= OZ_TOL[1]
    eng.close()


@pytest.fixture(scope="module")
def chain100():
    from proteindf_b200 import basis, grids, systems
    fx = golden("ref_chain100_ultrafine_sample.npz")
    syms, xyz = systems.peptide_chain(100, seed=1)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P, _, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["ULTRA_FINE"])
    rows = fx["rows"]
    xyzw = np.concatenate([P[rows], fx["w"][:, None]], axis=1)
    PA = 0.5 * systems.density_matrix(sh.nao, 380, seed=1)
    return fx, sh, xyzw, A[rows], PA


def _chain100_compare(fx, V, PA):
    pairs = np.abs(V[fx["vxc_i"], fx["vxc_j"]] - fx["vxc_vals"]).max()
    diag = np.abs(np.diag(V) - fx["vxc_diag"]).max()
    sums = {"sum": abs(V.sum() - float(fx["vxc_sum"])), "trace": abs(np.trace(V) - float(fx["vxc_trace"])),
            "dot_pa": abs((PA * V).sum() - float(fx["vxc_dot_pa"])),
            "fro": abs(np.linalg.norm(V) - float(fx["vxc_fro"]))}
    return max(pairs, diag), sums


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chain100_ultrafine_sample_vs_reference(chain100, precision):
    from proteindf_b200.xc import XcEngine
    fx, sh, xyzw, atom, PA = chain100
    eng = XcEngine(device=0, precision=precision, split_terms=10)
    eng.set_system(sh)
    eng.set_grid(xyzw, atom)
    exc, nel, V = eng.build_vxc("B3LYP", PA)
    dV, sums = _chain100_compare(fx, V, PA)
    dE = abs(exc - fx["exc"][0])
    print(f"chain100 {precision} on {len(xyzw)} sampled points: |dExc|={dE:.3e} max|dVxc| (diag + sampled)="
          f"{dV:.3e} |dN|={abs(nel - fx['nelec_alpha'][0]):.3e} checksums {sums}")
    if precision == "fp64":
        assert dE <= EXC_TOL and dV <= VXC_TOL
        assert all(v <= 1e-7 * max(1.0, abs(float(fx[f"vxc_{k}"]))) for k, v in sums.items())
        assert abs(nel - fx["nelec_alpha"][0]) <= 1e-9
    else:
        vmax = max(np.abs(fx["vxc_vals"]).max(), np.abs(fx["vxc_diag"]).max())
        assert dE <= OZ_TOL[0] * abs(fx["exc"][0]) and dV <= OZ_TOL[1] * vmax
    eng.close()
