"""Multi-rank logic on CPU (gloo, world_size 2): the grid is sharded by
blocks of points across ranks, each rank builds its partial Vxc, Exc and
electron count with the CPU oracle, and one all-reduce sums them; the result
equals the single-rank build. This is the exchange step the sharded GPU build
uses (the reference's MPI variant: src/libpdf/DfCalcGridX_Parallel.cpp:191-239)."""
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
    import torch
    import torch.distributed as dist
    from conftest import golden, shell_table
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fx = golden("ref_water2.npz")
    g = fx["grid"][:, :4]
    blocks = np.array_split(np.arange(len(g)), (len(g) + 127) // 128)
    mine = np.concatenate([b for i, b in enumerate(blocks) if i % world == rank])
    r = oracle.xc("B3LYP", shell_table(fx), g[mine], fx["PA"])
    buf = torch.tensor(np.concatenate([r["vxc"].ravel(), [r["exc"], r["nelec_alpha"]]]), dtype=torch.float64)
    dist.all_reduce(buf)
    if rank == 0:
        np.save(out_path, buf.numpy())
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
