"""Mixed-precision path (tcgen05 split-BF16 contractions, FP32 accumulation,
FP64 weights / sums / Vxc accumulation) against the reference and the FP64
GPU path. The tensor cores' FP32 accumulation rounds toward zero, so rho
carries a small negative bias (about 1e-6 relative); the tolerances are
relative to |Exc| and max|Vxc| accordingly."""
import numpy as np
import pytest

from conftest import shell_table

pytestmark = pytest.mark.gpu

TOL = {6: (2e-6, 1e-5), 3: (2e-6, 1e-5)}  # split terms -> (|dExc|/|Exc|, max|dVxc|/max|Vxc|)


def within(exc, ref_exc, V, ref_V, tol):
    return abs(exc - ref_exc) <= tol[0] * abs(ref_exc) and np.abs(V - ref_V).max() <= tol[1] * np.abs(ref_V).max()


def engine(fx, **kw):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(**kw)
    eng.set_system(shell_table(fx))
    return eng


@pytest.mark.parametrize("terms", [6, 3])
@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_water2_mixed_vs_reference(water2, fn, terms):
    eng = engine(water2, precision="mixed", split_terms=terms)
    eng.set_grid(water2["grid"][:, :4])
    exc, nel, V = eng.build_vxc(fn, water2["PA"])
    dE = abs(exc - water2[f"{fn}_exc"][0])
    dV = np.abs(V - water2[f"{fn}_vxc"]).max()
    print(f"{fn} split{terms}: |dExc|={dE:.3e} max|dVxc|={dV:.3e}")
    assert within(exc, water2[f"{fn}_exc"][0], V, water2[f"{fn}_vxc"], TOL[terms])
    assert np.allclose(V, V.T, atol=0, rtol=0)


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_chain12_mixed_vs_reference(chain12, fn):
    eng = engine(chain12, precision="mixed", split_terms=6)
    eng.set_grid(chain12["grid"][:, :4])
    exc, nel, V = eng.build_vxc(fn, chain12["PA"])
    dE = abs(exc - chain12[f"{fn}_exc"][0])
    dV = np.abs(V - chain12[f"{fn}_vxc"]).max()
    print(f"chain12 {fn}: |dExc|={dE:.3e} max|dVxc|={dV:.3e}")
    assert within(exc, chain12[f"{fn}_exc"][0], V, chain12[f"{fn}_vxc"], TOL[6])


def test_mixed_vs_fp64_gpu_water8():
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.water_cluster(8, seed=0)
    sh = basis.ShellTable(syms, xyz, basis.load_basis())
    z = [1 if s == "H" else 8 for s in syms]
    P, W, A = grids.molecular_grid(xyz, z, nrad=40, nang=146, radial="GC", mapping="TA", pruning=True)
    e64 = XcEngine()
    e64.set_system(sh)
    brad = np.array([grids.BECKE_RADIUS[zz] for zz in z])
    w = e64.becke_weights(P, A, W, brad)
    P, W, A = grids.screen_by_weight(P, w, A)
    xyzw = np.concatenate([P, W[:, None]], axis=1)
    PA = 0.5 * systems.density_matrix(sh.nao, 40, seed=0)
    e64.set_grid(xyzw, A)
    exc64, nel64, V64 = e64.build_vxc("B3LYP", PA)
    em = XcEngine(precision="mixed", split_terms=6)
    em.set_system(sh)
    em.set_grid(xyzw, A)
    excm, nelm, Vm = em.build_vxc("B3LYP", PA)
    print(f"(H2O)8 B3LYP mixed vs FP64: |dExc|={abs(excm - exc64):.3e} max|dVxc|={np.abs(Vm - V64).max():.3e}")
    assert within(excm, exc64, Vm, V64, TOL[6])
    assert abs(nelm - nel64) <= 2e-6 * abs(nel64)


# INT8 fixed-point slices (split_terms = 10): operands cut from the FP64 AO values
# into four radix-254 digits (~31 bits), exact integer accumulation; only the
# unbiased digit truncation and the dropped digit products of order >= 6 remain
# (measured: 2e-11 of Exc on the 100-atom chain, 5e-14 on the 2000-atom chain). The
# Vxc contraction accumulates a group of up to 4 blocks (512 points) under one scale
# per AO row; measured max|dVxc|/max|Vxc|: 1.0e-9 to 1.3e-9 on (H2O)2 and 2.0e-9 to
# 3.4e-9 on the 12-atom chain (a CPU emulation of the digit arithmetic gives 3.0e-9 for
# 128-point and 3.2e-9 for 512-point accumulation on the chain).
OZ_TOL = (2e-10, 5e-9)  # (|dExc|/|Exc|, max|dVxc|/max|Vxc|)


@pytest.mark.parametrize("fn", ["SVWN", "HFB", "B3LYP"])
def test_water2_int8_slices_vs_reference(water2, fn):
    eng = engine(water2, precision="mixed", split_terms=10)
    eng.set_grid(water2["grid"][:, :4])
    exc, nel, V = eng.build_vxc(fn, water2["PA"])
    dE = abs(exc - water2[f"{fn}_exc"][0])
    dV = np.abs(V - water2[f"{fn}_vxc"]).max()
    print(f"{fn} int8 slices: |dExc|={dE:.3e} max|dVxc|={dV:.3e} rel {dV / np.abs(water2[f'{fn}_vxc']).max():.3e}")
    assert within(exc, water2[f"{fn}_exc"][0], V, water2[f"{fn}_vxc"], OZ_TOL)
    assert abs(nel - water2[f"{fn}_nelec_alpha"][0]) <= 1e-10 * abs(nel)


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_chain12_int8_slices_vs_reference(chain12, fn):
    eng = engine(chain12, precision="mixed", split_terms=10)
    eng.set_grid(chain12["grid"][:, :4])
    exc, nel, V = eng.build_vxc(fn, chain12["PA"])
    dV = np.abs(V - chain12[f"{fn}_vxc"]).max() / np.abs(chain12[f"{fn}_vxc"]).max()
    print(f"chain12 {fn} int8 slices: |dExc|={abs(exc - chain12[f'{fn}_exc'][0]):.3e} max|dVxc|/max|Vxc|={dV:.3e}")
    assert within(exc, chain12[f"{fn}_exc"][0], V, chain12[f"{fn}_vxc"], OZ_TOL)


@pytest.mark.parametrize("terms", [6, 10])
def test_mixed_incremental(water2, terms):
    eng = engine(water2, precision="mixed", split_terms=terms)
    eng.set_grid(water2["grid"][:, :4])
    PA = water2["PA"]
    eng.build_vxc("B3LYP", 0.5 * PA)
    exc_i, _, V_i = eng.build_vxc("B3LYP", 0.5 * PA, incremental=True)
    exc_f, _, V_f = eng.build_vxc("B3LYP", PA)
    assert within(exc_i, exc_f, V_i, V_f, TOL[6])


def test_int8_accuracy_target_chain300():
    """The accuracy target of the INT8 path, |dExc| <= 1e-6 Eh against the FP64 path, on a 300-atom
    chain with the settings of the 2000-atom benchmark (device grid producer, USER 75x302, SS
    weights, AO cut-off 1e-10); also Vxc and the electron count."""
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(300, seed=11)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    PA = 0.5 * systems.density_matrix(sh.nao, int(0.4 * sh.nao), seed=11)
    radius = [grids.BRAGG_SLATER[int(z)] for z in sh.atom_z]
    res = {}
    for precision in ("fp64", "mixed"):
        e = XcEngine(device=0, precision=precision, ao_cutoff=1e-10)
        e.set_system(sh)
        npts = e.generate_grid(radius, partition="SSWeight", **grids.PRESETS["USER-75x302"])
        assert npts > 3_000_000
        res[precision] = e.build_vxc("B3LYP", PA)
        e.close()
    (xf, nf, Vf), (xm, nm, Vm) = res["fp64"], res["mixed"]
    assert abs(xm - xf) <= 1e-6
    assert np.abs(Vm - Vf).max() <= OZ_TOL[1] * np.abs(Vf).max()
    assert abs(nm - nf) <= 1e-6
