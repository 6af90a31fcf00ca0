"""Generate the reference golden fixtures for the parity tests.

Runs the ProteinDF reference itself (oracle/_ref/pdfxc_ref, built from the
reference sources by oracle/ref/Makefile) on small seeded systems and stores
its inputs and outputs as compressed .npz files beside this script:

  ref_water2.npz   (H2O)2, cc-pVDZ (48 AOs), USER 75x302 GC-TA grid with Becke
                   partitioning: single-centre and Becke weights of a point
                   sample, the reference's final grid (a seeded sample of it),
                   and per functional (SVWN, HFS, HFB, BLYP, B3LYP) Exc, Vxc,
                   rho / grad rho; AO table and AO values at five points.
  ref_chain12.npz  a 12-atom C/N/O/H chain, cc-pVDZ, same grid recipe, B3LYP
                   and SVWN on a point sample.
  ref_functionals.npz  functional values and first derivatives of all five
                   functionals on a seeded log-uniform (rho, gamma) set, both
                   the open-shell and the closed-shell overloads.
  ref_uks_water2.npz  the (H2O)2 grid sample of ref_water2.npz with two different
                   spin densities (10 alpha, 9 beta occupied): the reference's
                   open-shell Exc, Vxc_A, Vxc_B and electron counts for all five
                   functionals, the rho columns for SVWN and B3LYP.
  ref_ss_water2.npz  the (H2O)2 USER 75x302 grid with the Stratmann-Scuseria
                   partition (grid/partitioning_method = SSWeight): single-centre and
                   final weights of a seeded point sample.
  ref_grad_water.npz  one H2O, cc-pVDZ: the reference's XC nuclear gradient
                   (DfCalcGridX::energyGradient_part, AO-centre and grid-weight
                   terms apart) for SVWN and B3LYP, with the SG-1 grid it
                   integrates on (points, single-centre and partition weights).
  ref_becke_ghost_water2.npz  (H2O)2 with a dummy atom X: the reference's Becke weights
                   (dummy atoms left out of the partition products) on a point sample.
  ref_water8_user75x302.npz  the (H2O)8 configuration in full: the reference's whole
                   USER 75x302 Becke grid (point count, weight sum) and its SVWN and B3LYP
                   Exc, electron count and Vxc on it (about a minute of reference CPU).
  ref_chain100_ultrafine_sample.npz  the 100-atom chain, ULTRA_FINE grid, B3LYP: the
                   reference on a seeded 20,000-row sample of the grid (Exc, electron count,
                   Vxc diagonal, sampled entries and checksums).
  ref_density_water2.npz  (H2O)2 with the alpha density of ref_water2.npz: the
                   reference's DfCalcGridX::gridDensity at a seeded set of points
                   (a box around the molecules, points near and on the nuclei, far
                   points where rho vanishes).

usage (needs the reference tree): make -C oracle/ref && python tests/golden/make_ref_fixtures.py [name ...]
(names: system functional uks ss grad density ghost water8 chain100; none = all)
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from oracle import refio  # noqa: E402
from proteindf_b200 import basis, systems  # noqa: E402

GRID = {"nrad": 75, "nang": 302, "radial": "GC", "gc_mapping": "TA", "partition": "Becke", "pruning": "yes"}
FUNCS = ["SVWN", "HFS", "HFB", "BLYP", "B3LYP"]


def system_fixture(name, syms, xyz, nsample, funcs, nocc, seed):
    b = basis.load_basis("cc-pVDZ")
    q = systems.nuclear_charges(syms)
    rng = np.random.default_rng(seed)
    out = {"symbols": np.array(syms), "xyz": xyz, "grid_params": np.array([f"{k}={v}" for k, v in GRID.items()])}
    with tempfile.TemporaryDirectory() as d:
        g = refio.run_grid(d, syms, q, xyz, b, GRID)
        pts = g["points"].reshape(-1, 3)
        sel = np.sort(rng.choice(len(pts), min(4000, len(pts)), replace=False))
        out["becke_points"] = pts[sel]
        out["becke_atom"] = g["atom"][sel].astype(np.int32)
        out["becke_w_single"] = g["w_single"][sel]
        out["becke_w_final"] = g["w_final"][sel]
        out["radii"] = g["radii"].reshape(-1, 2)  # Bragg-Slater, Becke radius per atom
        full = g["grid"].reshape(-1, 5)
        out["grid_npts_full"] = np.array(len(full))
        out["grid_wsum_full"] = np.array(full[:, 3].sum())
        sel = np.sort(rng.choice(len(full), min(nsample, len(full)), replace=False))
        grid = full[sel]
        out["grid"] = grid
        sh = basis.ShellTable(syms, xyz, b)
        P = systems.density_matrix(sh.nao, nocc, seed=seed)
        PA = 0.5 * P
        out["PA"] = PA
        for fn in funcs:
            r = refio.run_xc(d, syms, q, xyz, b, fn, grid, PA, ao_dump=5)
            out[f"{fn}_exc"] = r["exc"]
            out[f"{fn}_vxc"] = r["vxc"].reshape(sh.nao, sh.nao)
            out[f"{fn}_rho"] = r["rho"].reshape(len(grid), -1)
            out[f"{fn}_nelec_alpha"] = r["nelec_alpha"]
        for k in ("ao_atom", "ao_type", "ao_nprim", "ao_exp", "ao_coef", "phi", "dphi"):
            out[k] = r[k]
    np.savez_compressed(os.path.join(HERE, name), **out)


def functional_fixture():
    rng = np.random.default_rng(7)
    n = 400
    ra = 10 ** rng.uniform(-12, 2, n)
    rb = np.where(rng.random(n) < 0.5, ra, 10 ** rng.uniform(-12, 2, n))
    gaa = 10 ** rng.uniform(-14, 3, n)
    gbb = np.where(rb == ra, gaa, 10 ** rng.uniform(-14, 3, n))
    gab = np.where(rb == ra, gaa, np.sqrt(gaa * gbb) * rng.uniform(-1, 1, n))
    inp = np.stack([ra, rb, gaa, gab, gbb], axis=1)
    out = {"inputs": inp}
    with tempfile.TemporaryDirectory() as d:
        for fn in FUNCS:
            out[fn] = refio.run_func(d, fn, inp)
    np.savez_compressed(os.path.join(HERE, "ref_functionals.npz"), **out)


def uks_fixture():
    w2 = dict(np.load(os.path.join(HERE, "ref_water2.npz")))
    syms = [str(s) for s in w2["symbols"]]
    xyz = w2["xyz"]
    b = basis.load_basis("cc-pVDZ")
    q = systems.nuclear_charges(syms)
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 10, seed=20)
    PB = 0.5 * systems.density_matrix(sh.nao, 9, seed=21)
    out = {"PA": PA, "PB": PB}
    with tempfile.TemporaryDirectory() as d:
        for fn in FUNCS:
            r = refio.run_xc_uks(d, syms, q, xyz, b, fn, w2["grid"], PA, PB)
            out[f"{fn}_exc"] = r["exc"]
            out[f"{fn}_vxc_a"] = r["vxc"].reshape(sh.nao, sh.nao)
            out[f"{fn}_vxc_b"] = r["vxc_b"].reshape(sh.nao, sh.nao)
            if fn in ("SVWN", "B3LYP"):  # the rho columns depend only on LDA / GGA
                out[f"{fn}_rho"] = r["rho"].reshape(len(w2["grid"]), -1)
            out[f"{fn}_nelec_alpha"] = r["nelec_alpha"]
            out[f"{fn}_nelec_beta"] = r["nelec_beta"]
    np.savez_compressed(os.path.join(HERE, "ref_uks_water2.npz"), **out)


def ss_fixture():
    w2 = dict(np.load(os.path.join(HERE, "ref_water2.npz")))
    syms = [str(s) for s in w2["symbols"]]
    kv = dict(GRID)
    kv["partition"] = "SSWeight"
    rng = np.random.default_rng(30)
    with tempfile.TemporaryDirectory() as d:
        g = refio.run_grid(d, syms, systems.nuclear_charges(syms), w2["xyz"], basis.load_basis("cc-pVDZ"), kv)
    pts = g["points"].reshape(-1, 3)
    sel = np.sort(rng.choice(len(pts), 4000, replace=False))
    np.savez_compressed(os.path.join(HERE, "ref_ss_water2.npz"), points=pts[sel],
                        atom=g["atom"][sel].astype(np.int32), w_single=g["w_single"][sel],
                        w_final=g["w_final"][sel])


def grad_fixture():
    b = basis.load_basis("cc-pVDZ")
    syms, xyz = systems.water_cluster(1, seed=0)
    q = systems.nuclear_charges(syms)
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 5, seed=0)
    out = {"symbols": np.array(syms), "xyz": xyz, "PA": PA}
    with tempfile.TemporaryDirectory() as d:
        for fn in ("SVWN", "B3LYP"):
            r = refio.run_grad(d, syms, q, xyz, b, fn, PA)
            out[f"{fn}_grad_orbital"] = r["grad_orbital"].reshape(-1, 3)
            out[f"{fn}_grad_weight"] = r["grad_weight"].reshape(-1, 3)
            out[f"{fn}_exc"] = r["exc"]
    out["points"] = r["points"].reshape(-1, 3)
    out["w_single"] = r["w_single"]
    out["w_partition"] = r["w_partition"]
    out["atom"] = r["atom"].astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "ref_grad_water.npz"), **out)


def density_fixture():
    w2 = dict(np.load(os.path.join(HERE, "ref_water2.npz")))
    syms = [str(s) for s in w2["symbols"]]
    xyz = w2["xyz"]
    rng = np.random.default_rng(40)
    lo, hi = xyz.min(0) - 6.0, xyz.max(0) + 6.0
    box = lo + (hi - lo) * rng.random((400, 3))
    near = xyz[rng.integers(0, len(xyz), 60)] + rng.normal(scale=0.05, size=(60, 3))
    d = rng.normal(size=(20, 3))
    far = xyz.mean(0) + (25.0 + 15.0 * rng.random((20, 1))) * d / np.linalg.norm(d, axis=1, keepdims=True)
    pts = np.concatenate([box, near, xyz, far])
    with tempfile.TemporaryDirectory() as dd:
        rho = refio.run_density(dd, syms, systems.nuclear_charges(syms), xyz, basis.load_basis("cc-pVDZ"),
                                w2["PA"], pts)
    np.savez_compressed(os.path.join(HERE, "ref_density_water2.npz"), symbols=np.array(syms), xyz=xyz,
                        P=w2["PA"], points=pts, rho=rho)


def ghost_fixture():
    """(H2O)2 with a dummy atom X between the molecules: the reference's Becke weights leave
    atoms of atomic number 0 out of every partition product (DfGenerateGrid::Ps_uij,
    src/libpdf/DfGenerateGrid.cpp:2056); a dummy atom has no grid of its own."""
    syms, xyz = systems.water_cluster(2, seed=0)
    syms = syms + ["X"]
    xyz = np.vstack([xyz, xyz.mean(0) + np.array([0.3, 0.2, -0.1])])
    rng = np.random.default_rng(50)
    with tempfile.TemporaryDirectory() as d:
        g = refio.run_grid(d, syms, systems.nuclear_charges(syms), xyz, basis.load_basis("cc-pVDZ"), GRID)
    pts = g["points"].reshape(-1, 3)
    sel = np.sort(rng.choice(len(pts), 4000, replace=False))
    full = g["grid"].reshape(-1, 5)
    np.savez_compressed(os.path.join(HERE, "ref_becke_ghost_water2.npz"), symbols=np.array(syms), xyz=xyz,
                        points=pts[sel], atom=g["atom"][sel].astype(np.int32), w_single=g["w_single"][sel],
                        w_final=g["w_final"][sel], radii=g["radii"].reshape(-1, 2),
                        grid_npts_full=np.array(len(full)), grid_wsum_full=np.array(full[:, 3].sum()))


def _packed_upper(V):
    return np.concatenate([V[i, i:] for i in range(V.shape[0])])


def water8_fixture():
    """The (H2O)8 configuration in full: O uniform in a 9 A cube (seed 0, min O-O 2.6 A), cc-pVDZ
    (192 AOs), P = 2 C C^T from the QR of a seeded N(0,1) 192 x 40 matrix (P_A = P / 2), the
    reference's own whole USER 75 x 302 GC-TA Becke grid (identity orientation), SVWN and
    B3LYP: the reference's Exc, electron count and Vxc (upper triangle) on that grid."""
    syms, xyz = systems.water_cluster(8, seed=0)
    b = basis.load_basis("cc-pVDZ")
    q = systems.nuclear_charges(syms)
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 40, seed=0)
    out = {"symbols": np.array(syms), "xyz": xyz, "PA": PA}
    with tempfile.TemporaryDirectory() as d:
        g = refio.run_grid(d, syms, q, xyz, b, GRID)
        full = g["grid"].reshape(-1, 5)
        out["grid_npts"] = np.array(len(full))
        out["grid_wsum"] = np.array(full[:, 3].sum())
        out["radii"] = g["radii"].reshape(-1, 2)
        for fn in ("SVWN", "B3LYP"):
            r = refio.run_xc(d, syms, q, xyz, b, fn, full, PA, threads=os.cpu_count())
            out[f"{fn}_exc"] = r["exc"]
            out[f"{fn}_nelec_alpha"] = r["nelec_alpha"]
            out[f"{fn}_vxc_upper"] = _packed_upper(r["vxc"].reshape(sh.nao, sh.nao))
            out[f"{fn}_seconds"] = np.array([r["t_rho"][0] + r["t_vxc"][0]])
    out["threads"] = np.array(os.cpu_count())
    np.savez_compressed(os.path.join(HERE, "ref_water8_user75x302.npz"), **out)


def chain100_fixture(nsample=20000):
    """The 100-atom chain configuration on a sample of its grid: the chain (seed 1), cc-pVDZ
    (932 AOs), P_A from 380 occupied orbitals, the ULTRA_FINE 99 x 590 grid (Euler-Maclaurin,
    MHL pruning; single-centre points from proteindf_b200.grids, Becke weights from the CPU
    restatement, weight screen 1e-16), a seeded uniform sample of nsample final rows (seed 0).
    The reference's B3LYP build on the sampled rows: Exc, electron count, the diagonal of Vxc,
    Vxc at 20000 seeded upper-triangle entries, and checksums of the whole Vxc (sum, trace,
    sum P_A * Vxc, Frobenius norm). The rows are stored as indices into the single-centre
    grid with their final weights."""
    from oracle import oracle
    from proteindf_b200 import grids
    syms, xyz = systems.peptide_chain(100, seed=1)
    b = basis.load_basis("cc-pVDZ")
    q = systems.nuclear_charges(syms)
    sh = basis.ShellTable(syms, xyz, b)
    PA = 0.5 * systems.density_matrix(sh.nao, 380, seed=1)
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["ULTRA_FINE"])
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    w = W * oracle.becke(xyz, brad, P, A)
    keep = np.nonzero(np.abs(w) > 1e-16)[0]
    rng = np.random.default_rng(0)
    sel = keep[np.sort(rng.choice(len(keep), nsample, replace=False))]
    grid5 = np.concatenate([P[sel], w[sel, None], A[sel, None].astype(np.float64)], axis=1)
    with tempfile.TemporaryDirectory() as d:
        r = refio.run_xc(d, syms, q, xyz, b, "B3LYP", grid5, PA, threads=os.cpu_count())
    V = r["vxc"].reshape(sh.nao, sh.nao)
    iu = np.triu_indices(sh.nao)
    pick = np.sort(np.random.default_rng(1).choice(len(iu[0]), 20000, replace=False))
    np.savez_compressed(os.path.join(HERE, "ref_chain100_ultrafine_sample.npz"),
                        rows=sel.astype(np.int64), w=grid5[:, 3], grid_npts=np.array(len(keep)),
                        exc=r["exc"], nelec_alpha=r["nelec_alpha"], vxc_diag=np.diag(V).copy(),
                        vxc_i=iu[0][pick].astype(np.int32), vxc_j=iu[1][pick].astype(np.int32),
                        vxc_vals=V[iu[0][pick], iu[1][pick]],
                        vxc_sum=np.array(V.sum()), vxc_trace=np.array(np.trace(V)),
                        vxc_dot_pa=np.array((PA * V).sum()), vxc_fro=np.array(np.linalg.norm(V)),
                        seconds=np.array([r["t_rho"][0] + r["t_vxc"][0]]), threads=np.array(os.cpu_count()))


def main(names):
    if not refio.ref_available():
        raise SystemExit("build the reference harness first: make -C oracle/ref")
    if not names or "system" in names:
        syms, xyz = systems.water_cluster(2, seed=0)
        system_fixture("ref_water2.npz", syms, xyz, 6000, FUNCS, nocc=10, seed=0)
        syms, xyz = systems.peptide_chain(12, seed=3)
        system_fixture("ref_chain12.npz", syms, xyz, 5000, ["SVWN", "B3LYP"], nocc=20, seed=3)
    steps = {"functional": functional_fixture, "uks": uks_fixture, "ss": ss_fixture, "grad": grad_fixture,
             "density": density_fixture, "ghost": ghost_fixture, "water8": water8_fixture,
             "chain100": chain100_fixture}
    for name, f in steps.items():
        if not names or name in names:
            f()


if __name__ == "__main__":
    main(sys.argv[1:])
