"""CUDA path (libpdfxc through its C ABI) against the reference fixtures and the
CPU oracle. Tolerances (FP64 drop-in): |dExc| <= 1e-8 Eh, max|dVxc| <= 1e-7
against the reference; the AO screening cutoff (1e-14) is the only approximation
the GPU path makes beyond summation order."""
import numpy as np
import pytest

from conftest import golden, shell_table

pytestmark = pytest.mark.gpu

EXC_TOL = 1e-8
VXC_TOL = 1e-7


def engine(fx, **kw):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(**kw)
    eng.set_system(shell_table(fx))
    return eng


@pytest.mark.parametrize("fn", ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"])
def test_water2_vs_reference(water2, fn):
    eng = engine(water2)
    eng.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
    exc, nel, V = eng.build_vxc(fn, water2["PA"])
    assert abs(exc - water2[f"{fn}_exc"][0]) <= EXC_TOL
    assert np.abs(V - water2[f"{fn}_vxc"]).max() <= VXC_TOL
    assert abs(nel - water2[f"{fn}_nelec_alpha"][0]) <= 1e-9
    rho = eng.get_rho(fn not in ("SVWN", "HFS"))
    assert np.abs(rho - water2[f"{fn}_rho"]).max() <= 1e-9


@pytest.mark.parametrize("fn", ["SVWN", "B3LYP"])
def test_chain12_vs_reference(chain12, fn):
    eng = engine(chain12)
    eng.set_grid(chain12["grid"][:, :4])
    exc, nel, V = eng.build_vxc(fn, chain12["PA"])
    assert abs(exc - chain12[f"{fn}_exc"][0]) <= EXC_TOL
    assert np.abs(V - chain12[f"{fn}_vxc"]).max() <= VXC_TOL


def test_vxc_accumulates_into_F(water2):
    eng = engine(water2)
    eng.set_grid(water2["grid"][:, :4])
    F0 = np.arange(water2["PA"].size, dtype=np.float64).reshape(water2["PA"].shape) * 1e-3
    F = F0.copy()
    eng.build_vxc("B3LYP", water2["PA"], F=F)
    assert np.abs((F - F0) - water2["B3LYP_vxc"]).max() <= VXC_TOL


def test_full_grid_vs_oracle_water8():
    """(H2O)8 on a full Becke grid sample: GPU vs the CPU oracle."""
    from oracle import oracle
    from proteindf_b200 import basis, grids, systems
    syms, xyz = systems.water_cluster(8, seed=0)
    sh = basis.ShellTable(syms, xyz, basis.load_basis())
    z = [1 if s == "H" else 8 for s in syms]
    P, W, A = grids.molecular_grid(xyz, z, nrad=30, nang=110, radial="GC", mapping="TA", pruning=True)
    from proteindf_b200.xc import XcEngine
    eng = XcEngine()
    eng.set_system(sh)
    brad = np.array([grids.BECKE_RADIUS[zz] for zz in z])
    w = eng.becke_weights(P, A, W, brad)
    fac = oracle.becke(xyz, brad, P, A)
    assert np.all(np.abs(w - W * fac) <= 1e-13 * np.abs(W))
    P, W, A = grids.screen_by_weight(P, w, A)
    rng = np.random.default_rng(1)
    sel = np.sort(rng.choice(len(W), 20000, replace=False))
    xyzw = np.concatenate([P[sel], W[sel, None]], axis=1)
    PA = 0.5 * systems.density_matrix(sh.nao, 40, seed=0)
    eng.set_grid(xyzw, A[sel])
    for fn in ("SVWN", "B3LYP"):
        exc, nel, V = eng.build_vxc(fn, PA)
        ref = oracle.xc(fn, sh, xyzw, PA)
        assert abs(exc - ref["exc"]) <= EXC_TOL
        assert np.abs(V - ref["vxc"]).max() <= VXC_TOL
        assert abs(nel - ref["nelec_alpha"]) <= 1e-9


def test_becke_vs_reference(water2):
    eng = engine(water2)
    w = eng.becke_weights(water2["becke_points"], water2["becke_atom"], water2["becke_w_single"],
                          water2["radii"][:, 1])
    # FP64 with a different operation order (fused multiply-adds): relative to each point's weight
    assert np.all(np.abs(w - water2["becke_w_final"]) <= 1e-13 * np.abs(water2["becke_w_single"]))


def test_becke_equals_oracle_bit_for_bit():
    """The device's Becke weights (compiled without fused multiply-adds) equal the CPU
    restatement's bit for bit, so both sides keep the same points under the 1e-16 weight screen;
    a 30-atom chain on a USER 40 x 110 grid, the warp-per-point table form."""
    from oracle import oracle
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(30, seed=5)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, nrad=40, nang=110, radial="GC", mapping="TA", pruning=True)
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    eng = XcEngine()
    eng.set_system(sh)
    w = eng.becke_weights(P, A, W, brad)
    ref = W * oracle.becke(xyz, brad, P, A)
    assert np.array_equal(w, ref), np.abs(w - ref).max()
    eng.close()


def test_becke_warp_form_equals_oracle_bit_for_bit():
    """Above 48 atoms the Becke weights come from the warp-per-point kernel (its lanes over the
    atoms); they equal the CPU restatement's bit for bit too: a 56-atom chain on a USER 20 x 50 grid."""
    from oracle import oracle
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(56, seed=7)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, nrad=20, nang=50, radial="GC", mapping="TA", pruning=True)
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    eng = XcEngine()
    eng.set_system(sh)
    w = eng.becke_weights(P, A, W, brad)
    ref = W * oracle.becke(xyz, brad, P, A)
    assert np.array_equal(w, ref), np.abs(w - ref).max()
    eng.close()


def test_becke_dummy_atom_vs_reference():
    """A dummy atom (atomic number 0) is left out of the partition products, as the reference's
    Ps_uij does (src/libpdf/DfGenerateGrid.cpp:2056); equal to the oracle bit for bit."""
    from oracle import oracle
    from proteindf_b200 import basis
    from proteindf_b200.xc import XcEngine
    fx = golden("ref_becke_ghost_water2.npz")
    syms = [str(s) for s in fx["symbols"]]
    sh = basis.ShellTable(syms, fx["xyz"], basis.load_basis("cc-pVDZ"))
    assert sh.atom_z[-1] == 0
    eng = XcEngine()
    eng.set_system(sh)
    brad = fx["radii"][:, 1]
    w = eng.becke_weights(fx["points"], fx["atom"], fx["w_single"], brad)
    assert np.all(np.abs(w - fx["w_final"]) <= 1e-13 * np.abs(fx["w_single"]))
    ref = fx["w_single"] * oracle.becke(fx["xyz"], brad, fx["points"], fx["atom"], ghost=sh.atom_z == 0)
    assert np.array_equal(w, ref)
    eng.close()


def test_incremental_density_update(water2):
    """xc-update = yes: a build on dP adds rho(dP) to the stored rho(P_prev)."""
    eng = engine(water2)
    eng.set_grid(water2["grid"][:, :4])
    PA = water2["PA"]
    rng = np.random.default_rng(3)
    dP = rng.normal(scale=1e-3, size=PA.shape)
    dP = 0.5 * (dP + dP.T)
    eng.build_vxc("B3LYP", PA - dP)
    exc_i, _, V_i = eng.build_vxc("B3LYP", dP, incremental=True)
    exc_f, _, V_f = eng.build_vxc("B3LYP", PA)
    assert abs(exc_i - exc_f) <= 1e-10
    assert np.abs(V_i - V_f).max() <= 1e-9


def test_rho_restart_roundtrip(water2):
    eng = engine(water2)
    eng.set_grid(water2["grid"][:, :4])
    eng.build_vxc("BLYP", water2["PA"])
    rho = eng.get_rho(True)
    eng2 = engine(water2)
    eng2.set_grid(water2["grid"][:, :4])
    eng2.set_rho(rho, True)
    exc, _, V = eng2.build_vxc("BLYP", np.zeros_like(water2["PA"]), incremental=True)
    assert abs(exc - water2["BLYP_exc"][0]) <= EXC_TOL
    assert np.abs(V - water2["BLYP_vxc"]).max() <= VXC_TOL


def test_device_build_matches_host_build(water2):
    import torch
    eng = engine(water2)
    eng.set_grid(water2["grid"][:, :4])
    exc_h, nel_h, V_h = eng.build_vxc("B3LYP", water2["PA"])
    dP = torch.tensor(water2["PA"], device="cuda", dtype=torch.float64)
    dV = torch.empty_like(dP)
    torch.cuda.synchronize()
    exc_d, nel_d = eng.build_vxc_device("B3LYP", dP.data_ptr(), dV.data_ptr())
    # Vxc is accumulated with FP64 atomics: equal up to summation order
    assert abs(exc_d - exc_h) <= 1e-13 and abs(nel_d - nel_h) <= 1e-13
    assert np.abs(dV.cpu().numpy() - V_h).max() <= 1e-13


def test_small_blocks_and_ragged_grid(water2):
    """Blocks of 37 points (ragged last block) give the same result."""
    eng = engine(water2, block_points=37)
    g = water2["grid"][:4001]
    eng.set_grid(g[:, :4])
    exc, _, V = eng.build_vxc("SVWN", water2["PA"])
    eng2 = engine(water2)
    eng2.set_grid(g[:, :4])
    exc2, _, V2 = eng2.build_vxc("SVWN", water2["PA"])
    assert abs(exc - exc2) <= 1e-12
    assert np.abs(V - V2).max() <= 1e-12


def test_single_point_grid(water2):
    eng = engine(water2)
    g = water2["grid"][:1]
    eng.set_grid(g[:, :4])
    exc, nel, V = eng.build_vxc("B3LYP", water2["PA"])
    from oracle import oracle
    ref = oracle.xc("B3LYP", shell_table(water2), g[:, :4], water2["PA"])
    assert abs(exc - ref["exc"]) <= 1e-12
    assert np.abs(V - ref["vxc"]).max() <= 1e-12


def test_errors_are_status_codes(water2):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine()
    with pytest.raises(RuntimeError, match="set_system"):
        eng.set_grid(water2["grid"][:10, :4])
    eng.set_system(shell_table(water2))
    with pytest.raises(RuntimeError, match="set_grid"):
        eng.build_vxc("SVWN", water2["PA"])
    eng.set_grid(water2["grid"][:10, :4])
    with pytest.raises(RuntimeError, match="incremental"):
        eng.build_vxc("SVWN", water2["PA"], incremental=True)
    with pytest.raises(RuntimeError, match="owner atom"):
        eng.becke_weights(np.zeros((2, 3)), np.array([0, 99]), np.ones(2), np.ones(6))


def test_ss_weights_vs_reference(water2):
    """Device Stratmann-Scuseria weights on the reference's SSWeight grid sample, and
    on a 30-atom chain against the oracle (relative 1e-13 per weight)."""
    from oracle import oracle
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    fx = golden("ref_ss_water2.npz")
    eng = XcEngine(device=0)
    eng.set_system(shell_table(water2))
    w = eng.ss_weights(fx["points"], fx["atom"], fx["w_single"])
    assert np.all(np.abs(w - fx["w_final"]) <= 1e-13 * np.abs(fx["w_single"]))
    eng.close()
    syms, xyz = systems.peptide_chain(30, seed=5)
    Z = [int(z) for z in systems.nuclear_charges(syms)]
    P, W, A = grids.molecular_grid(xyz, Z, nrad=30, nang=110, radial="GC", mapping="TA", pruning=True)
    eng = XcEngine(device=0)
    eng.set_system(basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ")))
    w = eng.ss_weights(P, A, W)
    ref = W * oracle.ss(xyz, P, A)
    assert np.all(np.abs(w - ref) <= 1e-13 * np.abs(W))
    eng.close()
