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
