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
  ref_density_water2.npz  (H2O)2 with the alpha density of ref_water2.npz: the
                   reference's DfCalcGridX::gridDensity at a seeded set of points
                   (a box around the molecules, points near and on the nuclei, far
                   points where rho vanishes).

usage (needs the reference tree): make -C oracle/ref && python tests/golden/make_ref_fixtures.py [name ...]
(names: system functional uks ss grad density; none = all)
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


def main(names):
    if not refio.ref_available():
        raise SystemExit("build the reference harness first: make -C oracle/ref")
    if not names or "system" in names:
        syms, xyz = systems.water_cluster(2, seed=0)
        system_fixture("ref_water2.npz", syms, xyz, 6000, FUNCS, nocc=10, seed=0)
        syms, xyz = systems.peptide_chain(12, seed=3)
        system_fixture("ref_chain12.npz", syms, xyz, 5000, ["SVWN", "B3LYP"], nocc=20, seed=3)
    steps = {"functional": functional_fixture, "uks": uks_fixture, "ss": ss_fixture, "grad": grad_fixture,
             "density": density_fixture}
    for name, f in steps.items():
        if not names or name in names:
            f()


if __name__ == "__main__":
    main(sys.argv[1:])
