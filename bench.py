#!/usr/bin/env python
"""Vxc build throughput of the B200 XC quadrature (grid points/s, ms per SCF iteration).

Workload (default): a seeded 100-atom peptide-like chain (C:N:O:H = 30:8:10:52),
cc-pVDZ (5d; the 6-31G** stand-in, ~930 AOs), B3LYP, ULTRA_FINE 99x590 grid
(Euler-Maclaurin radial, pruned, Becke partition computed on the GPU), alpha
density P_A = C C^T from the QR of a seeded N(0,1) N x 380 matrix. One step is
one closed-shell Vxc build (rho pass + Vxc pass) of the whole grid.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
  python bench.py --impl reference ...   (the reference's CPU DfCalcGridX, sampled)

With --precision both (default) the same grid is built with the FP64 drop-in and
the mixed path (INT8 fixed-point slices on the tensor cores by default); the
headline value is the FP64 drop-in (the plain FP64 path is the configuration the
metric is quoted on), the line carries the mixed path's numbers, the
mixed-vs-FP64 speed-up and |dExc| / max|dVxc| between them.

Under torchrun (N > 1) every rank builds its own chain (seed + rank): the units
are independent molecules, no data-path collective; value = all ranks' points
/ the slowest rank's time (weak scaling).

--shard builds ONE chain over all ranks instead (the reference's distributed
DfCalcGridX): every rank builds its cost-balanced range of grid blocks, then one
NCCL all-reduce sums the packed upper triangle of Vxc with Exc and the electron
count appended. A step is the rank's build (library CUDA events) plus the
all-reduce (CUDA events on torch's stream), max over ranks; value = the chain's
points / that time (strong scaling: the total work is fixed).

The same line (N = 1, unless --no-large) carries the adjoint on the differentiation
configuration (a 30-atom chain, PBE: forward and backward host-API times) and the two
large configurations,
each built with the FP64 drop-in and the INT8 path, their speed-up and |dExc|:
  chain2000  one 2000-atom chain, cc-pVDZ (~18,600 AOs), B3LYP, USER 75x302 grid with
             Stratmann-Scuseria weights, AO cut-off 1e-10
  batch64    64 independent chains of 10-120 atoms (seeded sizes), cc-pVDZ, B3LYP,
             USER 75x302 grid with Becke weights, one batched build per step
             (pdfxc_build_vxc_batched: one graph per build for all molecules)
--workload chain2000 / batch64 runs one of them alone.

cpu_baseline: the reference's own DfCalcGridX (oracle/_ref/pdfxc_ref, built from its
sources) on seeded samples of the grid's rows, all host cores (two sample sizes, whose
rates must agree) and one thread; its Exc and Vxc on the first sample are compared
with the GPU builds on the same rows (vs_reference_parity).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Vxc build grid points/s"
UNIT = "grid points/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--split-terms", type=int, default=10, choices=[3, 6, 10],
                    help="mixed path: 3/6 split-BF16 products, 10 = INT8 fixed-point slices")
    ap.add_argument("--natoms", type=int, default=100)
    ap.add_argument("--functional", default="B3LYP")
    ap.add_argument("--grid", default="ULTRA_FINE")
    ap.add_argument("--nocc", type=int, default=380)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample", type=int, default=4000, help="grid points for the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="chain", choices=["chain", "batch64", "chain2000"])
    ap.add_argument("--no-large", action="store_true", help="leave the 2000-atom chain and the batch out")
    ap.add_argument("--partition", default="Becke", choices=["Becke", "SSWeight"],
                    help="partition weights of the chain workload's grid")
    ap.add_argument("--shard", action="store_true",
                    help="one chain over all ranks: block ranges + one NCCL all-reduce (strong scaling)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload(args, seed):
    """Seeded chain, basis table, single-centre grid, density."""
    from proteindf_b200 import basis, grids, systems
    syms, xyz = systems.peptide_chain(args.natoms, seed=seed)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS[args.grid])
    PA = 0.5 * systems.density_matrix(sh.nao, args.nocc, seed=seed)
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    return syms, xyz, sh, P, W, A, PA, brad


def final_grid(eng, P, W, A, brad, partition="Becke"):
    from proteindf_b200 import grids
    w = eng.ss_weights(P, A, W) if partition == "SSWeight" else eng.becke_weights(P, A, W, brad)
    P2, W2, A2 = grids.screen_by_weight(P, w, A)
    return np.concatenate([P2, W2[:, None]], axis=1), A2


def config(args, npts, nao, **extra):
    c = {"workload": f"{args.natoms}-atom peptide-like chain, cc-pVDZ, {args.functional}, {args.grid} grid",
         "atoms": args.natoms, "n_ao": nao, "grid_points": int(npts), "functional": args.functional,
         "grid": args.grid, "partition": args.partition, "precision": args.precision, "nocc": args.nocc,
         "split_terms": args.split_terms if args.precision != "fp64" else None,
         "l2": "flushed between timed steps (512 MiB write)"}
    c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def fp64_gemm_peak(torch):
    """Measured cuBLAS DGEMM throughput on this GPU (TFLOP/s), burst, best of 5."""
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float64)
    b = torch.randn(n, n, device="cuda", dtype=torch.float64)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def sample_rows(n_total, n, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n_total, min(n, n_total), replace=False))


def reference_on_rows(args, syms, xyz, grid5, PA, rows, threads):
    """The reference engine (or, without it, the CPU restatement) on the given grid rows:
    (seconds, kind, exc, vxc)."""
    import tempfile
    from oracle import refio
    from proteindf_b200 import basis, systems
    g = grid5[rows]
    if refio.ref_available():
        with tempfile.TemporaryDirectory() as d:
            r = refio.run_xc(d, syms, systems.nuclear_charges(syms), xyz, basis.load_basis("cc-pVDZ"),
                             args.functional, g, PA, threads=threads)
        n = int(round(np.sqrt(r["vxc"].size)))
        return float(r["t_rho"][0] + r["t_vxc"][0]), "reference", float(r["exc"][0]), r["vxc"].reshape(n, n)
    from oracle import oracle
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ"))
    t0 = time.perf_counter()
    r = oracle.xc(args.functional, sh, g[:, :4], PA, threads=threads)
    return time.perf_counter() - t0, "port", r["exc"], r["vxc"]


def cpu_baseline(args, syms, xyz, grid5, PA, sample):
    """Reference DfCalcGridX (oracle/_ref/pdfxc_ref) on seeded samples of grid rows. Its
    per-point cost is position-independent (it evaluates every AO at every point), so
    points/s extrapolates linearly: two samples (sample/2 rows, seed 0; sample rows, seed 1)
    on all host cores, whose rates must agree, and one sample on one thread (seed 2). The
    seed-0 sample's Exc and Vxc are returned for the parity check."""
    cores = os.cpu_count() or 1
    runs = []
    keep = None
    for n, seed, threads in ((sample // 2, 0, cores), (sample, 1, cores), (max(100, sample // 16), 2, 1)):
        rows = sample_rows(len(grid5), n, seed)
        t, kind, exc, vxc = reference_on_rows(args, syms, xyz, grid5, PA, rows, threads)
        runs.append({"points": int(len(rows)), "seed": seed, "threads": threads, "seconds": t,
                     "points_per_s": len(rows) / t})
        if seed == 0:
            keep = {"rows": rows, "exc": exc, "vxc": vxc}
    full = runs[:2]
    value = sum(r["points"] for r in full) / sum(r["seconds"] for r in full)
    spread = abs(full[0]["points_per_s"] - full[1]["points_per_s"]) / value
    out = {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
           "sample": (f"{full[0]['points']} + {full[1]['points']} of {len(grid5)} grid points (seeds 0, 1), "
                      f"rho pass + Vxc pass on {cores} threads, {sum(r['seconds'] for r in full):.1f} s; "
                      "extrapolated (cost per point is position-independent)"),
           "samples": runs, "sample_rate_spread": spread,
           "one_thread": {"value": runs[2]["points_per_s"], "unit": UNIT, "points": runs[2]["points"]}}
    return out, keep


def parity_vs_reference(args, sh, grid4, owner, keep, precisions):
    """The GPU builds on the reference's seed-0 sample rows: |dExc| and max|dVxc| per path."""
    from proteindf_b200.xc import XcEngine
    rows = keep["rows"]
    out = {"points": int(len(rows)), "functional": args.functional}
    for p in precisions:
        eng = XcEngine(device=0, precision=p, split_terms=args.split_terms)
        eng.set_system(sh)
        eng.set_grid(grid4[rows], owner[rows])
        exc, _, V = eng.build_vxc(args.functional, keep["PA"])
        eng.close()
        out[p] = {"abs_dexc": abs(exc - keep["exc"]), "max_abs_dvxc": float(np.abs(V - keep["vxc"]).max()),
                  "reference_exc_on_sample": keep["exc"]}
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from proteindf_b200 import grids
    from oracle import oracle
    syms, xyz, sh, P, W, A, PA, brad = workload(args, args.seed)
    # Becke weights from the CPU restatement: bit for bit the device's (same IEEE operations in
    # the same order), so the weight screen keeps the same points as the GPU arm's grid
    fac = oracle.ss(xyz, P, A) if args.partition == "SSWeight" else oracle.becke(xyz, brad, P, A)
    P2, W2, A2 = grids.screen_by_weight(P, W * fac, A)
    grid5 = np.concatenate([P2, W2[:, None], A2[:, None]], axis=1)
    per_step = max(200, args.cpu_sample // 2)
    cores = os.cpu_count() or 1
    vals, kind = [], "reference"
    first = None
    for i in range(args.warmup + args.steps):
        rows = sample_rows(len(grid5), per_step, i)
        t, kind, exc, vxc = reference_on_rows(args, syms, xyz, grid5, PA, rows, cores)
        if i == 0:
            first = {"points": int(len(rows)), "seed": 0, "exc": exc, "vxc_trace": float(np.trace(vxc)),
                     "vxc_sum": float(vxc.sum())}
        if i >= args.warmup:
            vals.append(len(rows) / t)
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": len(grid5) / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded chain and density, ProteinDF grid recipe)",
            "config": config(args, len(grid5), sh.nao),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
                             "sample": f"{per_step} grid points per step (seed = step), extrapolated to "
                                       f"{len(grid5)}"},
            "reference_on_sample": first,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "chain":
        return run_large(args)
    if args.shard:
        return run_shard(args)
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from proteindf_b200.xc import XcEngine

    syms, xyz, sh, P, W, A, PA, brad = workload(args, args.seed + rank)
    dev = f"cuda:{local}"
    nao = sh.nao
    dP = torch.tensor(PA, device=dev)
    dV = torch.empty_like(dP)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    precisions = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    engines = {p: XcEngine(device=local, precision=p, split_terms=args.split_terms) for p in precisions}
    for e in engines.values():
        e.set_system(sh)
    grid4, owner = final_grid(next(iter(engines.values())), P, W, A, brad, args.partition)
    npts = len(grid4)
    res = {}
    clk_summary = None
    for p, eng in engines.items():
        eng.set_grid(grid4, owner)
        for _ in range(args.warmup):
            eng.build_vxc_device(args.functional, dP.data_ptr(), dV.data_ptr())
        dev_ms, launches = 0.0, 0
        barrier()
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                exc, nel = eng.build_vxc_device(args.functional, dP.data_ptr(), dV.data_ptr())
                prof = eng.last_profile()
                dev_ms += prof["total_ms"]
                launches += prof["launches"]
            barrier()
        if p == precisions[-1]:
            clk_summary = clk.summary()
        V = dV.cpu().numpy()
        # one build launched stage by stage for the per-stage times (same kernels, no graph)
        eng.set_profiling(True)
        flush.zero_()
        torch.cuda.synchronize()
        eng.build_vxc_device(args.functional, dP.data_ptr(), dV.data_ptr())
        stage = eng.last_profile()
        eng.set_profiling(False)
        ms = max_over_ranks(dev_ms) / args.steps
        res[p] = {"ms": ms, "value": world * npts / (ms * 1e-3), "exc": exc, "nel": nel, "V": V, "stage": stage,
                  "launches": launches, "stats": eng.grid_stats()}

    head = precisions[-1]
    eng = engines[head]
    # end to end through the host API: P from pinned host memory in, Vxc (F += Vxc) back
    pin_P = torch.empty((nao, nao), dtype=torch.float64, pin_memory=True)
    pin_P.copy_(torch.from_numpy(PA))
    pin_F = torch.zeros((nao, nao), dtype=torch.float64, pin_memory=True)
    e2e_t = []
    for i in range(max(1, args.steps)):
        pin_F.zero_()
        barrier()
        t0 = time.perf_counter()
        eng.build_vxc(args.functional, pin_P.numpy(), F=pin_F.numpy())
        e2e_t.append(time.perf_counter() - t0)
    t_e2e = max_over_ranks(float(np.mean(e2e_t)))

    if rank == 0:
        peaks = measured_peaks()
        rooflines = {p: roofline(args, torch, peaks, res[p], p) for p in precisions}
        cpu, parity = None, None
        if not args.no_cpu_baseline:
            grid5 = np.concatenate([grid4, owner[:, None].astype(np.float64)], axis=1)
            cpu, keep = cpu_baseline(args, syms, xyz, grid5, PA, args.cpu_sample)
            keep["PA"] = PA
            parity = parity_vs_reference(args, sh, grid4, owner, keep, precisions)
        h = res[head]
        dtype = "f64" if head == "fp64" else ("int8 fixed-point slices/i32/f64" if args.split_terms == 10
                                              else "bf16 split/f32/f64")
        line = {"metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": h["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype,
                "data": "synthetic (seeded chain and density, ProteinDF grid recipe)",
                "config": config(args, npts, nao, blocks=h["stats"]["nblocks"],
                                 mean_screened_aos=h["stats"]["mean_nb"], headline=head),
                "exc": h["exc"], "nelec_alpha": h["nel"],
                "e2e": {"value": world * npts / t_e2e, "unit": UNIT,
                        "h2d_bytes_per_step": nao * nao * 8, "d2h_bytes_per_step": nao * nao * 8 + 16},
                "roofline": rooflines[head], "cpu_baseline": cpu, "gpu_launches": h["launches"],
                "clocks": clk_summary, "vs_reference_parity": parity}
        if "fp64" in res and "mixed" in res:
            f, m = res["fp64"], res["mixed"]
            line["mixed"] = {"value": m["value"], "ms_per_step": m["ms"], "exc": m["exc"], "dtype": (
                "int8 fixed-point slices/i32/f64" if args.split_terms == 10 else "bf16 split/f32/f64"),
                "roofline": rooflines["mixed"]}
            line["mixed_vs_fp64"] = {"speedup": f["ms"] / m["ms"], "abs_dexc": abs(m["exc"] - f["exc"]),
                                     "max_abs_dvxc": float(np.abs(m["V"] - f["V"]).max()),
                                     "abs_dnelec_alpha": abs(m["nel"] - f["nel"])}
    for e in engines.values():
        e.close()
    if rank == 0 and world == 1 and not args.no_large:
        del dP, dV
        torch.cuda.empty_cache()
        for name in ("chain2000", "batch64"):
            line[name] = large_workload(args, name, flush)
        line["adjoint"] = adjoint_workload()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_shard(args):
    """One chain over all ranks (ShardedXcEngine): block ranges + one NCCL all-reduce per build."""
    import datetime
    import torch
    import torch.distributed as dist
    from proteindf_b200.sharded import ShardedXcEngine, allreduce_partials
    from proteindf_b200.xc import XcEngine
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:  # a group of one, so that the same reduce runs
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=600))
    prec = "fp64" if args.precision == "both" else args.precision
    syms, xyz, sh, P, W, A, PA, brad = workload(args, args.seed)  # the same molecule on every rank
    dev = f"cuda:{local}"
    dP = torch.tensor(PA, device=dev)
    dV = torch.empty_like(dP)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    eng = XcEngine(device=local, precision=prec, split_terms=args.split_terms)
    eng.set_system(sh)
    grid4, owner = final_grid(eng, P, W, A, brad, args.partition)
    shard = ShardedXcEngine(eng)
    shard.set_grid(grid4, owner)
    npts = len(grid4)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def step():
        exc, nel = eng.build_vxc_device(args.functional, dP.data_ptr(), dV.data_ptr())
        t_build = eng.last_profile()["total_ms"]
        ev[0].record()
        _, sc = allreduce_partials(dV, [exc, nel], None)
        ev[1].record()
        torch.cuda.synchronize()
        return t_build, ev[0].elapsed_time(ev[1]), sc

    for _ in range(args.warmup):
        step()
    t_build = t_red = 0.0
    launches = 0
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            tb, tr, sc = step()
            t_build += tb
            t_red += tr
            launches += eng.last_profile()["launches"]
        dist.barrier()
        torch.cuda.synchronize()
    mine = torch.tensor([(t_build + t_red) / args.steps, t_build / args.steps, t_red / args.steps],
                        dtype=torch.float64, device=dev)
    dist.all_reduce(mine, op=dist.ReduceOp.MAX)
    ms, ms_build, ms_red = (float(x) for x in mine.cpu())
    # end to end through the sharded host API: P from host memory, Vxc of the whole molecule back on every rank
    e2e_t = []
    for _ in range(max(1, args.steps)):
        dist.barrier()
        t0 = time.perf_counter()
        shard.build_vxc(args.functional, PA)
        e2e_t.append(time.perf_counter() - t0)
    t_e2e = torch.tensor([float(np.mean(e2e_t))], dtype=torch.float64, device=dev)
    dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    nao = sh.nao
    if rank == 0:
        b = shard.bounds
        line = {"metric": METRIC, "value": npts / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "int8 fixed-point slices/i32/f64",
                "data": "synthetic (seeded chain and density, ProteinDF grid recipe)",
                "config": config(args, npts, nao, sharding="one chain, cost-balanced block ranges, "
                                 "one NCCL all-reduce of the packed Vxc upper triangle + Exc, N",
                                 block_ranges=[int(x) for x in b], headline=prec),
                "exc": float(sc[0]), "nelec_alpha": float(sc[1]),
                "ms_build_max": ms_build, "ms_allreduce_max": ms_red,
                "allreduce_bytes": 8 * (nao * (nao + 1) // 2 + 2),
                "e2e": {"value": npts / float(t_e2e.item()), "unit": UNIT,
                        "h2d_bytes_per_step": nao * nao * 8, "d2h_bytes_per_step": nao * nao * 8 + 16},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    eng.close()
    dist.destroy_process_group()


def adjoint_workload(reps=3):
    """The differentiation configuration: a 30-atom chain (seed 21), the 6-31G*-shaped cc-pVDZ
    without hydrogen p shells, PBE, USER 75x302 grid with Becke weights. Host-API wall time (the calls
    synchronise) of the forward build and of pdfxc_xc_backward (dExc/dP, the AO-centre and the
    Becke-weight gradient terms), best of `reps` after a warm-up, on one GPU."""
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    syms, xyz = systems.peptide_chain(30, seed=21)
    sh = basis.ShellTable(syms, xyz, basis.load_basis("cc-pVDZ-noHp"))
    P, W, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["USER-75x302"])
    brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
    PA = 0.5 * systems.density_matrix(sh.nao, 60, seed=22)
    eng = XcEngine(device=0)
    eng.set_system(sh)
    eng.set_grid(np.c_[P, eng.becke_weights(P, A, W, brad)], A)
    fwd, bwd = [], []
    for k in range(reps + 1):
        t0 = time.perf_counter()
        exc, _, V = eng.build_vxc("PBE", PA)
        t1 = time.perf_counter()
        dP, go, gw, e2 = eng.xc_backward("PBE", PA, w_single=W, becke_radius=brad)
        t2 = time.perf_counter()
        if k:
            fwd.append(t1 - t0), bwd.append(t2 - t1)
    eng.close()
    return {"workload": "30-atom peptide-like chain (seed 21), cc-pVDZ without H p shells, PBE, USER 75x302, "
                        "Becke weights", "atoms": 30, "n_ao": int(sh.nao), "grid_points": int(len(P)),
            "forward_ms": 1e3 * min(fwd), "backward_ms": 1e3 * min(bwd),
            "max_abs_dexc_dP_minus_vxc": float(np.abs(dP - V).max()), "timing": "host API wall time"}


def large_workload(args, name, flush):
    """The 64-molecule batch or the 2000-atom chain, FP64 drop-in and INT8 path, device time
    per build (CUDA events of the library on its stream, L2 flushed between steps); one GPU."""
    import torch
    from proteindf_b200 import basis, grids, systems
    from proteindf_b200.xc import XcEngine
    b = basis.load_basis("cc-pVDZ")
    t0 = time.perf_counter()
    dP = dV = None
    if name == "batch64":
        rng = np.random.default_rng(args.seed)
        sizes = rng.integers(10, 121, 64)
        mols, PAs = [], []
        tmp = XcEngine(device=0)
        for k, n in enumerate(sizes):
            syms, xyz = systems.peptide_chain(int(n), seed=args.seed + 1000 + k)
            sh = basis.ShellTable(syms, xyz, b)
            P, W, A = grids.molecular_grid(xyz, sh.atom_z, **grids.PRESETS["USER-75x302"])
            brad = np.array([grids.BECKE_RADIUS[int(z)] for z in sh.atom_z])
            tmp.set_system(sh)
            w = tmp.becke_weights(P, A, W, brad)
            P2, W2, A2 = grids.screen_by_weight(P, w, A)
            mols.append((sh, np.c_[P2, W2], A2))
            PAs.append(0.5 * systems.density_matrix(sh.nao, max(1, int(0.4 * sh.nao)), seed=args.seed + 2000 + k))
        tmp.close()
        npts = sum(len(g) for _, g, _ in mols)
        nao = sum(sh.nao for sh, _, _ in mols)
        desc = {"workload": "64 independent peptide-like chains of 10-120 atoms (seeded), cc-pVDZ, B3LYP, "
                            "USER 75x302 grid, Becke weights, one batched build",
                "molecules": 64, "atoms": int(sizes.sum()), "n_ao_total": int(nao), "grid_points": int(npts)}
    else:
        # the grid comes from the device producer (pdfxc_generate_grid: USER 75x302 GC-TA,
        # MHL pruning, Stratmann-Scuseria weights, weight screen), as each engine's own grid
        syms, xyz = systems.peptide_chain(2000, seed=args.seed)
        sh = basis.ShellTable(syms, xyz, b)
        radius = [grids.BRAGG_SLATER[int(z)] for z in sh.atom_z]
        dP = 0.5 * systems.density_matrix_device(sh.nao, int(0.4 * sh.nao), seed=args.seed, device="cuda:0")
        dV = torch.empty_like(dP)
        npts, nao = None, sh.nao
        desc = {"workload": "2000-atom peptide-like chain, cc-pVDZ, B3LYP, USER 75x302 grid, "
                            "Stratmann-Scuseria weights, AO cut-off 1e-10",
                "atoms": 2000, "n_ao": int(nao)}
    t_setup = time.perf_counter() - t0
    out = {}
    Vs = {}
    for prec in (["fp64", "mixed"] if args.precision == "both" else [args.precision]):
        eng = XcEngine(device=0, precision=prec, split_terms=args.split_terms,
                       ao_cutoff=1e-10 if name == "chain2000" else 1e-14)
        t1 = time.perf_counter()
        if name == "batch64":
            eng.set_batch(mols)
            build = lambda: eng.build_vxc_batched(args.functional, PAs)
        else:
            eng.set_system(sh)
            npts = eng.generate_grid(radius, partition="SSWeight", **grids.PRESETS["USER-75x302"])
            desc["grid_points"] = int(npts)
            build = lambda: eng.build_vxc_device(args.functional, dP.data_ptr(), dV.data_ptr())
        t_grid = time.perf_counter() - t1
        for _ in range(args.warmup):
            r = build()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = build()
            ms.append(eng.last_profile()["total_ms"])
        if name == "batch64":
            exc = float(np.sum(r[0]))
            Vs[prec] = r[2]
        else:
            exc = float(r[0])
            Vs[prec] = dV.clone()
        st = eng.grid_stats()
        eng.set_profiling(True)  # one more build, stage by stage, for the stage times (not timed above)
        build()
        prof = eng.last_profile()
        eng.set_profiling(False)
        out[prec] = {"ms_per_step": float(np.mean(ms)), "value": npts / (np.mean(ms) * 1e-3), "exc": exc,
                     "blocks": st["nblocks"], "mean_screened_aos": st["mean_nb"],
                     ("grid_generation_s" if name == "chain2000" else "set_grid_s"): t_grid,
                     "stage_ms": {k: prof[k] for k in ("ao_ms", "gemm_x_ms", "rho_ms", "gemm_v_ms", "finish_ms")}}
        eng.close()
    res = {"metric": METRIC, "unit": UNIT, "steps": args.steps, "warmup": args.warmup,
           "config": dict(desc, functional=args.functional, l2="flushed between timed steps (512 MiB write)",
                          host_setup_s=t_setup)}
    res.update(out)
    if "fp64" in out and "mixed" in out:
        if name == "batch64":
            dv = max(float(np.abs(a - b).max()) for a, b in zip(Vs["fp64"], Vs["mixed"]))
        else:
            dv = float((Vs["fp64"] - Vs["mixed"]).abs().max())
        res["mixed_vs_fp64"] = {"speedup": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
                                "abs_dexc": abs(out["mixed"]["exc"] - out["fp64"]["exc"]), "max_abs_dvxc": dv}
    del Vs, dP, dV
    torch.cuda.empty_cache()
    return res


def run_large(args):
    """One large configuration alone (--workload chain2000 | batch64)."""
    import torch
    torch.cuda.set_device(0)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    res = large_workload(args, args.workload, flush)
    head = res.get("mixed", res.get("fp64"))
    line = {"metric": METRIC, "unit": UNIT, "value": head["value"], "ms_per_step": head["ms_per_step"],
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "int8 fixed-point slices/i32/f64" if "mixed" in res else "f64",
            "data": "synthetic (seeded chains and densities)"}
    line.update(res)
    print(json.dumps(line), flush=True)


def measured_traffic(kernel):
    """DRAM bytes per build of an FP64 contraction kernel from the committed ncu summary
    (profiles/traffic_fp64_contractions_chain100_b3lyp_ultrafine.md), for the default workload."""
    import re
    try:
        txt = open(os.path.join(ROOT, "profiles", "traffic_fp64_contractions_chain100_b3lyp_ultrafine.md")).read()
    except OSError:
        return None
    mt = re.search(r"traffic_bytes_per_build k_" + kernel + r" = (\d+)", txt)
    return int(mt.group(1)) if mt else None


def roofline(args, torch, peaks, r, precision):
    """Dominant contraction kernel of one build: algorithmic FLOPs (2 nb^2 np per block per
    contraction) over its CUDA-event time, against the measured peak of the unit it runs on."""
    per = {k: r["stage"][k] for k in ("ao_ms", "gemm_x_ms", "rho_ms", "gemm_v_ms", "finish_ms")}
    top = max(("gemm_x_ms", "gemm_v_ms"), key=lambda k: per[k])
    flops = 0.5 * r["stats"]["contraction_flops"]
    achieved = flops / (per[top] * 1e-3) / 1e12 if per[top] > 0 else None
    if precision == "fp64":
        peak = fp64_gemm_peak(torch)
        note = "measured cuBLAS FP64 DGEMM 8192^3 on this GPU (burst), FP64 tensor cores"
    elif args.split_terms == 10:
        bf = peaks.get("bf16_tflops", 1590.0)
        peak = 2.0 * bf
        note = ("2 x MEASURED_PEAKS.json bf16_tflops (dense INT8 rate is twice BF16 on B200); achieved counts "
                "useful FP64-equivalent FLOPs, the tensor cores issue 10 slice products per useful product")
    else:
        peak = peaks.get("bf16_tflops", 1590.0)
        note = "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback 1.59 PFLOP/s"
    default = (args.natoms == 100 and args.grid == "ULTRA_FINE" and args.functional == "B3LYP" and args.nocc == 380
               and args.seed == 1)
    traffic = measured_traffic(top.replace("_ms", "")) if (precision == "fp64" and default) else None
    return {"bound": "tensor", "kernel": top.replace("_ms", ""), "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "traffic_note": ("DRAM bytes of the kernel's launches in one build, one ncu capture "
                             "(profiles/traffic_fp64_contractions_chain100_b3lyp_ultrafine.md)") if traffic else None,
            "peak_source": note, "flops_per_launch_set": flops, "stage_ms": per}


if __name__ == "__main__":
    main()
