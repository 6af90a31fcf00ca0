"""Multi-rank logic on CPU (gloo, world_size 2): the grid's blocks are split
into contiguous ranges of near-equal cost by the library's
pdfxc_partition_blocks (host code, no device), each rank builds its partial
Vxc, Exc and electron count -- with the CPU oracle standing in for the rank's
GPU build -- and proteindf_b200.sharded.allreduce_partials sums them in one
collective; the result equals the single-rank build. This is the exchange step
of the sharded GPU build (the reference's MPI variant:
src/libpdf/DfCalcGridX_Parallel.cpp:191-239)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch.distributed as dist
    from conftest import golden, shell_table
    from oracle import oracle
    from proteindf_b200.sharded import allreduce_partials
    from proteindf_b200.xc import partition_blocks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fx = golden("ref_water2.npz")
    g = fx["grid"][:, :4]
    sh = shell_table(fx)
    blocks = np.array_split(np.arange(len(g)), (len(g) + 127) // 128)
    cost = np.array([4.0 * sh.nao ** 2 * len(b) for b in blocks])
    bounds = partition_blocks(cost, world)
    mine = np.concatenate(blocks[bounds[rank]:bounds[rank + 1]])
    r = oracle.xc("B3LYP", sh, g[mine], fx["PA"])
    V, sc = allreduce_partials(r["vxc"], [r["exc"], r["nelec_alpha"]])
    if rank == 0:
        np.save(out_path, np.concatenate([V.ravel(), sc]))
    dist.barrier()
    dist.destroy_process_group()


def test_block_sharded_build_allreduce(tmp_path):
    import torch.multiprocessing as mp
    from conftest import golden
    out = str(tmp_path / "sum.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    s = np.load(out)
    fx = golden("ref_water2.npz")
    n = fx["PA"].shape[0]
    assert np.abs(s[:n * n].reshape(n, n) - fx["B3LYP_vxc"]).max() < 1e-12
    assert abs(s[n * n] - fx["B3LYP_exc"][0]) < 1e-12
    assert abs(s[n * n + 1] - fx["B3LYP_nelec_alpha"][0]) < 1e-10


class _OracleRankEngine:
    """The XcEngine interface that ShardedXcEngine drives, with the CPU oracle standing in for
    the rank's GPU build: blocks of 128 rows in input order, each rank builds its block range."""

    def __init__(self, sh):
        self.sh = sh

    def set_system(self, sh):
        self.sh = sh

    def set_grid(self, xyzw, atom=None):
        self.g, self.atom = np.asarray(xyzw)[:, :4], atom
        self.blocks = np.array_split(np.arange(len(self.g)), (len(self.g) + 127) // 128)
        self.rows = np.arange(len(self.g))

    def block_costs(self):
        return np.array([4.0 * self.sh.nao ** 2 * len(b) for b in self.blocks])

    def set_block_range(self, lo, hi):
        self.rows = np.concatenate(self.blocks[lo:hi])

    def build_vxc(self, fn, PA, incremental=False):
        from oracle import oracle
        r = oracle.xc(fn, self.sh, self.g[self.rows], PA)
        return r["exc"], r["nelec_alpha"], r["vxc"]

    def build_vxc_uks(self, fn, PA, PB, incremental=False):
        from oracle import oracle
        r = oracle.xc_uks(fn, self.sh, self.g[self.rows], PA, PB)
        return r["exc"], r["nelec_alpha"], r["nelec_beta"], r["vxc_a"], r["vxc_b"]

    def xc_gradient(self, fn, PA, w_single=None, becke_radius=None, size_adjust=True):
        from oracle import oracle
        r = oracle.xc_grad(fn, self.sh, self.g[self.rows], self.atom[self.rows], PA)
        return r["grad"], None, r["exc"]


def _sharded_worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch.distributed as dist
    from conftest import golden, shell_table
    from proteindf_b200.sharded import ShardedXcEngine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fx, uks = golden("ref_water2.npz"), golden("ref_uks_water2.npz")
    sh = shell_table(fx)
    eng = ShardedXcEngine(_OracleRankEngine(sh))
    eng.set_grid(fx["grid"][:, :4], fx["grid"][:, 4].astype(np.int32))
    e, n, V = eng.build_vxc("B3LYP", fx["PA"])
    eu, na, nb, FA, FB = eng.build_vxc_uks("BLYP", uks["PA"], uks["PB"])
    g, gw, eg = eng.xc_gradient("SVWN", fx["PA"])
    assert gw is None
    if rank == 0:
        np.savez(out_path, e=e, n=n, V=V, eu=eu, na=na, nb=nb, FA=FA, FB=FB, g=g, eg=eg)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_engine_host_builds_two_ranks(tmp_path):
    """ShardedXcEngine over two gloo ranks: the closed-shell build, the open-shell build and
    the XC gradient on host arrays (the packed upper triangles and the scalars in one
    all-reduce per build) equal the one-rank result."""
    import torch.multiprocessing as mp
    from conftest import golden, shell_table
    from oracle import oracle
    out = str(tmp_path / "sharded.npz")
    mp.start_processes(_sharded_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = dict(np.load(out))
    fx, uks = golden("ref_water2.npz"), golden("ref_uks_water2.npz")
    sh = shell_table(fx)
    g = fx["grid"]
    assert abs(r["e"] - fx["B3LYP_exc"][0]) < 1e-12
    assert abs(r["n"] - fx["B3LYP_nelec_alpha"][0]) < 1e-10
    assert np.abs(r["V"] - fx["B3LYP_vxc"]).max() < 1e-12
    assert abs(r["eu"] - uks["BLYP_exc"][0]) < 1e-12
    assert abs(r["na"] - uks["BLYP_nelec_alpha"][0]) < 1e-10 and abs(r["nb"] - uks["BLYP_nelec_beta"][0]) < 1e-10
    assert np.abs(r["FA"] - uks["BLYP_vxc_a"]).max() < 1e-12 and np.abs(r["FB"] - uks["BLYP_vxc_b"]).max() < 1e-12
    full = oracle.xc_grad("SVWN", sh, g[:, :4], g[:, 4].astype(np.int32), fx["PA"])
    assert np.abs(r["g"] - full["grad"]).max() < 1e-11
    assert abs(r["eg"] - full["exc"]) < 1e-12


def test_packed_upper_host_round_trip():
    from proteindf_b200.sharded import _pack_host, _unpack_host
    rng = np.random.default_rng(3)
    for n in (1, 2, 7, 33):
        A = rng.normal(size=(n, n))
        S = A + A.T
        p = _pack_host(S)
        assert p.shape == (n * (n + 1) // 2,)
        assert np.array_equal(_unpack_host(p, n), S)


def test_partition_blocks_properties():
    from proteindf_b200.xc import partition_blocks
    rng = np.random.default_rng(0)
    for nblk, nparts in [(1000, 4), (7, 3), (3, 8), (0, 2), (500, 1)]:
        cost = rng.uniform(0, 10, nblk) ** 3
        b = partition_blocks(cost, nparts)
        assert b[0] == 0 and b[-1] == nblk and np.all(np.diff(b) >= 0)
        if nblk >= 10 * nparts:
            parts = np.array([cost[b[i]:b[i + 1]].sum() for i in range(nparts)])
            # contiguous cuts at the cost quantiles: each part within one block of the mean
            assert np.all(np.abs(parts - cost.sum() / nparts) <= cost.max())
    with pytest.raises(RuntimeError):
        partition_blocks(np.array([1.0, -1.0]), 2)


def _local_worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch.distributed as dist
    from conftest import golden, shell_table
    from proteindf_b200.sharded import BlockCyclic, ShardedXcEngine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fx = golden("ref_water2.npz")
    sh = shell_table(fx)
    layout = BlockCyclic(sh.nao, 5, 2, world // 2)
    PA = fx["PA"]
    mine = PA[np.ix_(layout.rows(rank), layout.cols(rank))]
    eng = ShardedXcEngine(_OracleRankEngine(sh))
    eng.set_grid(fx["grid"][:, :4], fx["grid"][:, 4].astype(np.int32))
    e, n, piece = eng.build_vxc_local("B3LYP", mine, layout)
    np.savez(out_path + f".{rank}.npz", e=e, n=n, piece=piece, rows=layout.rows(rank), cols=layout.cols(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_block_cyclic_local_matrices_four_ranks(tmp_path):
    """The distributed-matrix form over four gloo ranks (a 2 x 2 process grid, blocks of 5):
    each rank passes only its block-cyclic piece of P_A and receives only its piece of Vxc,
    which equals the one-rank Vxc at those rows and columns; Exc and the electron count are
    the whole molecule's on every rank."""
    import torch.multiprocessing as mp
    from conftest import golden
    out = str(tmp_path / "local")
    mp.start_processes(_local_worker, args=(4, _free_port(), out), nprocs=4, join=True, start_method="spawn")
    fx = golden("ref_water2.npz")
    seen = np.zeros(fx["PA"].shape, dtype=int)
    for r in range(4):
        d = np.load(out + f".{r}.npz")
        ref = fx["B3LYP_vxc"][np.ix_(d["rows"], d["cols"])]
        assert d["piece"].shape == ref.shape
        assert np.abs(d["piece"] - ref).max() < 1e-12
        assert abs(float(d["e"]) - fx["B3LYP_exc"][0]) < 1e-12
        assert abs(float(d["n"]) - fx["B3LYP_nelec_alpha"][0]) < 1e-10
        seen[np.ix_(d["rows"], d["cols"])] += 1
    assert np.all(seen == 1)  # the pieces tile the matrix


def test_block_cyclic_layout_matches_scalapack_rule():
    from proteindf_b200.sharded import BlockCyclic
    L = BlockCyclic(10, 3, 2, 2)
    assert list(L.rows(0)) == [0, 1, 2, 6, 7, 8] and list(L.cols(1)) == [3, 4, 5, 9]
    assert [L.local_shape(r) for r in range(4)] == [(6, 6), (6, 4), (4, 6), (4, 4)]
    cover = np.zeros(100, dtype=int)
    for r in range(4):
        cover[L.flat_index(r)] += 1
    assert np.all(cover == 1)
    with pytest.raises(ValueError):
        BlockCyclic(10, 0, 2, 2)
