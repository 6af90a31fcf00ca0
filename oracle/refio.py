"""I/O for the reference-oracle harness (oracle/_ref/pdfxc_ref).

TEST INFRASTRUCTURE ONLY: used by tests/, the fixture generators under
tests/golden/ and bench.py's reference arm. Writes the harness's case files
(text key/value lines, atoms in bohr, raw basis-library contractions) and reads
its flat output records ([char name[32]][int64 n][n float64]).
"""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "pdfxc_ref")


def ref_available():
    return os.path.exists(REF_BIN)


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        while True:
            name = f.read(32)
            if len(name) < 32:
                break
            n = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            out[name.rstrip(b"\0").decode()] = np.frombuffer(f.read(8 * n), dtype=np.float64).copy()
    return out


def write_case(path, symbols, charges, xyz_bohr, basis, kv):
    """basis: {element: [{"shell": "s", "prims": [[exp, coef], ...]}, ...]}"""
    with open(path, "w") as f:
        for k, v in kv.items():
            f.write(f"{k} {v}\n")
        for s, q, r in zip(symbols, charges, np.asarray(xyz_bohr).reshape(-1, 3)):
            f.write(f"atom {s} {q:.1f} {r[0]:.17g} {r[1]:.17g} {r[2]:.17g}\n")
        for el in sorted(set(symbols), key=list(symbols).index):
            for sh in basis.get(el, []) if el == "X" else basis[el]:  # X: a dummy atom, no basis
                f.write(f"cgto {el} {sh['shell']} {len(sh['prims'])}\n")
                for e, c in sh["prims"]:
                    f.write(f"{e:.17g} {c:.17g}\n")


def run(mode, case_path, out_path, threads=None, timeout=None):
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    env.setdefault("OMP_SCHEDULE", "dynamic")
    # the reference writes its log file into the working directory
    subprocess.run([REF_BIN, mode, case_path, out_path], check=True, env=env, timeout=timeout,
                   cwd=os.path.dirname(os.path.abspath(out_path)), stdout=subprocess.DEVNULL)
    return read_records(out_path)


def run_xc(workdir, symbols, charges, xyz_bohr, basis, functional, grid5, PA, ao_dump=0,
           threads=1, timeout=None):
    """Reference rho + Vxc pass. grid5: (npts, 5) [x, y, z, w, atom]; PA: alpha density."""
    os.makedirs(workdir, exist_ok=True)
    gpath = os.path.join(workdir, "grid.bin")
    ppath = os.path.join(workdir, "P.bin")
    np.ascontiguousarray(grid5, dtype=np.float64).tofile(gpath)
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    case = os.path.join(workdir, "case.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {
        "functional": functional, "npts": len(grid5), "grid_file": gpath,
        "density_file": ppath, "ao_dump": ao_dump, "threads": threads})
    return run("xc", case, os.path.join(workdir, "out.bin"), threads=threads, timeout=timeout)


def run_xc_uks(workdir, symbols, charges, xyz_bohr, basis, functional, grid5, PA, PB, threads=1, timeout=None):
    """Reference open-shell rho + Vxc pass (the P_A, P_B overloads)."""
    os.makedirs(workdir, exist_ok=True)
    gpath = os.path.join(workdir, "grid.bin")
    ppath = os.path.join(workdir, "P.bin")
    pbpath = os.path.join(workdir, "PB.bin")
    np.ascontiguousarray(grid5, dtype=np.float64).tofile(gpath)
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    np.ascontiguousarray(PB, dtype=np.float64).tofile(pbpath)
    case = os.path.join(workdir, "case.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {
        "functional": functional, "npts": len(grid5), "grid_file": gpath, "density_file": ppath,
        "density_file_b": pbpath, "uks": 1, "threads": threads})
    return run("xc", case, os.path.join(workdir, "out.bin"), threads=threads, timeout=timeout)


def run_grid(workdir, symbols, charges, xyz_bohr, basis, grid_kv):
    os.makedirs(workdir, exist_ok=True)
    case = os.path.join(workdir, "case.txt")
    kv = {"functional": "SVWN"}
    kv.update(grid_kv)
    write_case(case, symbols, charges, xyz_bohr, basis, kv)
    return run("grid", case, os.path.join(workdir, "grid_out.bin"))


def run_grad(workdir, symbols, charges, xyz_bohr, basis, functional, PA, timeout=None):
    """Reference XC nuclear gradient (DfCalcGridX::energyGradient_part over all
    atoms) and the SG-1 grid it integrates on. Returns the harness records:
    grad_orbital (x2 for RKS), grad_weight, exc, points, w_single, w_partition, atom."""
    os.makedirs(workdir, exist_ok=True)
    ppath = os.path.join(workdir, "P.bin")
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    case = os.path.join(workdir, "grad.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {"functional": functional, "density_file": ppath})
    # one thread: the SG-1 grid generator of the reference races with several (see _dropin_env)
    return run("grad", case, os.path.join(workdir, "grad_out.bin"), threads=1, timeout=timeout)


def _density_case(workdir, symbols, charges, xyz_bohr, basis, P, points):
    os.makedirs(os.path.join(workdir, "fl_Work"), exist_ok=True)
    ppath, xpath = os.path.join(workdir, "P.bin"), os.path.join(workdir, "points.bin")
    np.ascontiguousarray(P, dtype=np.float64).tofile(ppath)
    np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3).tofile(xpath)
    case = os.path.join(workdir, "density.txt")
    write_case(case, symbols, charges, xyz_bohr, basis,
               {"density_file": ppath, "points_file": xpath, "npts": len(np.reshape(points, (-1, 3)))})
    return case


def run_density(workdir, symbols, charges, xyz_bohr, basis, P, points, timeout=None):
    """rho(r) = phi^T P phi at the points through the reference's DfCalcGridX::gridDensity."""
    case = _density_case(workdir, symbols, charges, xyz_bohr, basis, P, points)
    return run("density", case, os.path.join(workdir, "density_out.bin"), timeout=timeout)["rho"]


def run_func(workdir, functional, inputs5):
    os.makedirs(workdir, exist_ok=True)
    ipath = os.path.join(workdir, "func_in.bin")
    np.ascontiguousarray(inputs5, dtype=np.float64).tofile(ipath)
    case = os.path.join(workdir, "func.txt")
    with open(case, "w") as f:
        f.write(f"functional {functional}\nnpts {len(inputs5)}\ninput_file {ipath}\n")
    r = run("func", case, os.path.join(workdir, "func_out.bin"))
    return r["values"].reshape(-1, 10)


DROPIN_BIN = os.path.join(HERE, "_ref", "pdfxc_dropin")


def dropin_available():
    return os.path.exists(DROPIN_BIN)


def _dropin_env():
    """One OpenMP thread for the harness that links the reference classes: the reference's
    DfGenerateGrid::getGrids builds its orientation matrix in an OpenMP loop that adds into
    one shared matrix without a reduction (src/libpdf/DfGenerateGrid.cpp:1768-1795), so with
    several threads the SG-1 gradient grid of either class can come out rotated."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "1"
    return env


def run_dropin(workdir, symbols, charges, xyz_bohr, basis, functional, grid5, PA, timeout=None):
    """Reference DfCalcGridX and DfCalcGridX_B200 on the same inputs, two SCF
    iterations (P_A/2, then the difference P_A/2 with xc-update)."""
    os.makedirs(os.path.join(workdir, "fl_Work"), exist_ok=True)
    gpath = os.path.join(workdir, "grid.bin")
    ppath = os.path.join(workdir, "P.bin")
    np.ascontiguousarray(grid5, dtype=np.float64).tofile(gpath)
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    case = os.path.join(workdir, "case.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {
        "functional": functional, "npts": len(grid5), "grid_file": gpath, "density_file": ppath})
    out = os.path.join(workdir, "dropin.bin")
    subprocess.run([DROPIN_BIN, "dropin", case, out], check=True, timeout=timeout, cwd=workdir,
                   stdout=subprocess.DEVNULL, env=_dropin_env())
    return read_records(out)


def run_dropin_grad(workdir, symbols, charges, xyz_bohr, basis, functional, PA, timeout=None):
    """energyGradient of the reference DfCalcGridX and of DfCalcGridX_B200 (without and
    with the grid-weight term) on the same parameter set and density."""
    os.makedirs(os.path.join(workdir, "fl_Work"), exist_ok=True)
    ppath = os.path.join(workdir, "P.bin")
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    case = os.path.join(workdir, "case.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {"functional": functional, "density_file": ppath})
    out = os.path.join(workdir, "dropin_grad.bin")
    subprocess.run([DROPIN_BIN, "dropin_grad", case, out], check=True, timeout=timeout, cwd=workdir,
                   stdout=subprocess.DEVNULL, env=_dropin_env())
    return read_records(out)


def run_dropin_density(workdir, symbols, charges, xyz_bohr, basis, P, points, timeout=None):
    """gridDensity of the reference DfCalcGridX and of DfCalcGridX_B200 (per point for the first
    8 points, and batched) on the same points: records ref_rho, b200_rho, b200_rho_single."""
    case = _density_case(workdir, symbols, charges, xyz_bohr, basis, P, points)
    out = os.path.join(workdir, "dropin_density.bin")
    subprocess.run([DROPIN_BIN, "dropin_density", case, out], check=True, timeout=timeout, cwd=workdir,
                   stdout=subprocess.DEVNULL, env=_dropin_env())
    return read_records(out)


def run_dropin_gengrid(workdir, symbols, charges, xyz_bohr, basis, grid_kv, timeout=None):
    """The grid producer: DfGenerateGrid::dfGrdMain of the reference, then DfGenerateGrid_B200's,
    on the same parameter set (grid_kv: grid_type, nrad, nang, radial, gc_mapping, partition,
    pruning). Returns (ref_grid, b200_grid) as (rows, ncol) arrays of the grid matrix."""
    os.makedirs(os.path.join(workdir, "fl_Work"), exist_ok=True)
    case = os.path.join(workdir, "gengrid.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, dict(grid_kv, functional="SVWN"))
    out = os.path.join(workdir, "dropin_gengrid.bin")
    subprocess.run([DROPIN_BIN, "dropin_gengrid", case, out], check=True, timeout=timeout, cwd=workdir,
                   stdout=subprocess.DEVNULL, env=_dropin_env())
    r = read_records(out)
    return (r["ref_grid"].reshape(-1, int(r["ref_ncol"][0])), r["b200_grid"].reshape(-1, int(r["b200_ncol"][0])))


def run_dropin_uks(workdir, symbols, charges, xyz_bohr, basis, functional, grid5, PA, PB, timeout=None):
    """The open-shell overloads of the reference DfCalcGridX and of DfCalcGridX_B200, two
    SCF iterations (PA/2, PB/2, then the same again with xc-update)."""
    os.makedirs(os.path.join(workdir, "fl_Work"), exist_ok=True)
    gpath = os.path.join(workdir, "grid.bin")
    ppath = os.path.join(workdir, "P.bin")
    pbpath = os.path.join(workdir, "PB.bin")
    np.ascontiguousarray(grid5, dtype=np.float64).tofile(gpath)
    np.ascontiguousarray(PA, dtype=np.float64).tofile(ppath)
    np.ascontiguousarray(PB, dtype=np.float64).tofile(pbpath)
    case = os.path.join(workdir, "case.txt")
    write_case(case, symbols, charges, xyz_bohr, basis, {
        "functional": functional, "npts": len(grid5), "grid_file": gpath, "density_file": ppath,
        "density_file_b": pbpath})
    out = os.path.join(workdir, "dropin_uks.bin")
    subprocess.run([DROPIN_BIN, "dropin_uks", case, out], check=True, timeout=timeout, cwd=workdir,
                   stdout=subprocess.DEVNULL, env=_dropin_env())
    return read_records(out)
