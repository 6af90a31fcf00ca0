"""Grid generation on the device (pdfxc_generate_grid) against the host generator of
proteindf_b200.grids with the device partition weights (the same recipe, pinned against
the reference by tests/test_oracle_pins.py), and the SG-1 grid against the reference's own
gradient grid (tests/golden/ref_grad_water.npz)."""
import numpy as np
import pytest

from conftest import golden, shell_table
from oracle import refio

pytestmark = pytest.mark.gpu


def _engine(fx):
    from proteindf_b200.xc import XcEngine
    e = XcEngine(device=0)
    e.set_system(shell_table(fx))
    return e


def _host_grid(e, xyz, Z, partition, **kw):
    from proteindf_b200 import grids
    P, W, A = grids.molecular_grid(xyz, Z, **kw)
    if partition == "Becke":
        w = e.becke_weights(P, A, W, np.array([grids.BECKE_RADIUS[z] for z in Z]))
    else:
        w = e.ss_weights(P, A, W)
    P, w, A = grids.screen_by_weight(P, w, A)
    return np.c_[P, w], A


@pytest.mark.parametrize("partition,preset", [("Becke", "USER-75x302"), ("SSWeight", "USER-75x302"),
                                              ("Becke", "ULTRA_FINE")])
def test_device_grid_equals_host_recipe(water2, partition, preset):
    from proteindf_b200 import grids
    Z = [int(z) for z in shell_table(water2).atom_z]
    e = _engine(water2)
    kw = grids.PRESETS[preset]
    ref, refA = _host_grid(e, water2["xyz"], Z, partition, **kw)
    n = e.generate_grid([grids.BRAGG_SLATER[z] for z in Z], partition=partition,
                        becke_radius=[grids.BECKE_RADIUS[z] for z in Z], **kw)
    g, A = e.get_grid()
    assert n == len(ref)
    assert np.array_equal(A, refA)
    assert np.abs(g[:, :3] - ref[:, :3]).max() == 0.0  # same operations in the same order
    assert np.all(np.abs(g[:, 3] - ref[:, 3]) <= 1e-14 * np.abs(ref[:, 3]))
    e.close()


def test_sg1_grid_vs_reference_gradient_grid():
    """The reference's SG-1 gradient grid (DfGenerateGrid::getGrids): 50 Euler-Maclaurin
    shells scaled by the SG-1 radii, SG-1 angular regions, rotated by the reference's
    orientation matrix (recovered here from the first shell of atom 0, the 6-point grid on
    the axes), Becke partition with size adjustment, weight screen."""
    from proteindf_b200 import grids
    fx = golden("ref_grad_water.npz")
    Z = [int(z) for z in shell_table(fx).atom_z]
    r1, _ = grids.radial_em(grids.SG1_RADIUS[Z[0]], 50, 1)
    u6 = grids.lebedev_table()[6]
    O = np.zeros((3, 3))
    for k in range(6):
        ax = int(np.argmax(np.abs(u6[k, :3])))
        O[:, ax] = (fx["points"][k] - fx["xyz"][0]) / r1 * np.sign(u6[k, ax])
    U, _, Vt = np.linalg.svd(O)
    O = U @ Vt  # nearest rotation
    e = _engine(fx)
    n = e.generate_grid([grids.SG1_RADIUS[z] for z in Z], nrad=50, nang=194, radial="EM", pruning="SG1",
                        partition="Becke", becke_radius=[grids.BECKE_RADIUS[z] for z in Z], orientation=O)
    g, A = e.get_grid()
    assert n == len(fx["points"])
    assert np.array_equal(A, fx["atom"].astype(np.int32))
    assert np.abs(g[:, :3] - fx["points"]).max() <= 1e-9  # the orientation is recovered to ~1e-12
    # the points carry the ~1e-11 bohr error of the recovered orientation; where the partition
    # factor is ~1e-18 (deep in another atom's cell) that moves it by ~1 % of itself, so the
    # weights are compared to 1e-8 relative plus 1e-11 of the largest weight
    ref_w = fx["w_single"] * fx["w_partition"]
    assert np.all(np.abs(g[:, 3] - ref_w) <= 1e-8 * np.abs(ref_w) + 1e-11 * np.abs(ref_w).max())
    e.close()


def test_build_on_generated_grid(water2):
    """A build on the generated grid equals a build on the same grid passed in."""
    from proteindf_b200 import grids
    from proteindf_b200.xc import XcEngine
    Z = [int(z) for z in shell_table(water2).atom_z]
    e = _engine(water2)
    e.generate_grid([grids.BRAGG_SLATER[z] for z in Z], becke_radius=[grids.BECKE_RADIUS[z] for z in Z])
    exc, nel, V = e.build_vxc("B3LYP", water2["PA"])
    g, A = e.get_grid()
    f = XcEngine(device=0)
    f.set_system(shell_table(water2))
    f.set_grid(g, A)
    exc2, nel2, V2 = f.build_vxc("B3LYP", water2["PA"])
    assert abs(exc - exc2) <= 1e-12 and abs(nel - nel2) <= 1e-12 and np.abs(V - V2).max() <= 1e-13
    e.close(), f.close()


def test_get_grid_returns_input_order(water2):
    e = _engine(water2)
    g = water2["grid"][:5000]
    e.set_grid(g[:, :4], g[:, 4].astype(np.int32))
    xyzw, A = e.get_grid()
    assert np.array_equal(xyzw, g[:, :4])
    assert np.array_equal(A, g[:, 4].astype(np.int32))
    e.close()


def test_generate_grid_errors(water2):
    from proteindf_b200 import grids
    Z = [int(z) for z in shell_table(water2).atom_z]
    e = _engine(water2)
    with pytest.raises(RuntimeError, match="parameter"):
        e.generate_grid([grids.BRAGG_SLATER[z] for z in Z], partition="Becke", becke_radius=None)
    with pytest.raises(RuntimeError, match="ascending"):  # an empty order
        e.generate_grid([grids.BRAGG_SLATER[z] for z in Z], partition="SSWeight",
                        unit_grids={0: np.zeros((0, 4)), 6: grids.lebedev_table()[6]})
    with pytest.raises(RuntimeError, match="not tabulated"):  # SG-1 needs orders 38, 86, 194
        e.generate_grid([grids.SG1_RADIUS[z] for z in Z], partition="SSWeight", nrad=50, radial="EM",
                        pruning="SG1", unit_grids={6: grids.lebedev_table()[6], 590: grids.lebedev_table()[590]})
    with pytest.raises(RuntimeError, match="radius"):
        e.generate_grid([-1.0] * len(Z), partition="SSWeight")
    with pytest.raises(RuntimeError, match="screened out"):  # radius 0: no grid on any atom
        e.generate_grid([0.0] * len(Z), partition="SSWeight")
    e.close()


def _match_grids(ref, b200):
    """Rows of the two grid matrices matched by position (the weight screens may differ on a
    point whose weight sits at the cut); returns (ref rows, b200 rows, unmatched weights)."""
    from scipy.spatial import cKDTree
    d, idx = cKDTree(b200[:, :3]).query(ref[:, :3])
    hit = d <= 1e-9
    lost = np.concatenate([ref[~hit, 3], np.delete(b200[:, 3], idx[hit])])
    return ref[hit], b200[idx[hit]], lost


@pytest.mark.skipif(not refio.dropin_available(), reason="oracle/_ref/pdfxc_dropin not built")
@pytest.mark.parametrize("kv", [
    dict(grid_type="USER", nrad=75, nang=302, radial="GC", gc_mapping="TA", partition="Becke", pruning="yes"),
    dict(grid_type="USER", nrad=40, nang=194, radial="GC", gc_mapping="BECKE", partition="SSWeight", pruning="no"),
    dict(grid_type="FINE"),
    dict(grid_type="SG-1"),
], ids=["user-becke-ta", "user-ss-becke-map", "fine", "sg1"])
def test_dfgenerategrid_b200_matches_reference_producer(tmp_path, water2, kv):
    """DfGenerateGrid_B200::dfGrdMain beside the reference's DfGenerateGrid::dfGrdMain: the
    same parameter set, orientation matrix and Lebedev tables, the same grid matrix file
    (x, y, z, weight, atom, zeroed density columns)."""
    from proteindf_b200 import basis, systems
    syms = [str(s) for s in water2["symbols"]]
    ref, b200 = refio.run_dropin_gengrid(str(tmp_path), syms, systems.nuclear_charges(syms), water2["xyz"],
                                         basis.load_basis("cc-pVDZ"), kv)
    assert ref.shape[1] == b200.shape[1] and abs(len(ref) - len(b200)) <= 4
    r, b, lost = _match_grids(ref, b200)
    # a point deep in another atom's cell has a partition product of ~1e-17 relative, which
    # neither side computes to relative accuracy: the screens may differ there, at weights
    # below 1e-12 (the largest weights are ~1e3)
    assert np.all(np.abs(lost) <= 1e-12)
    assert len(r) >= len(ref) - 4
    assert np.array_equal(r[:, 4], b[:, 4])  # owner atoms
    assert np.all(r[:, 5:] == 0.0) and np.all(b[:, 5:] == 0.0)
    assert np.abs(r[:, :3] - b[:, :3]).max() <= 1e-13
    assert np.all(np.abs(r[:, 3] - b[:, 3]) <= 1e-10 * np.abs(r[:, 3]) + 1e-13 * np.abs(r[:, 3]).max())
