"""Sharded build on the GPU. With one GPU per test run, two ranks are emulated as
two contexts over complementary block ranges, run one after the other: their
partial results must sum to the whole build (closed shell FP64 and INT8, open
shell, XC gradient). No kernel waits on another rank. The NCCL front end
(proteindf_b200.sharded) runs on a process group of world size 1."""
import os
import socket

import numpy as np
import pytest

from conftest import golden, shell_table

pytestmark = pytest.mark.gpu


def _engines(fx, precision="fp64"):
    from proteindf_b200.xc import XcEngine, partition_blocks
    out = []
    g = fx["grid"]
    for r in range(2):
        e = XcEngine(device=0, precision=precision, split_terms=10)
        e.set_system(shell_table(fx))
        e.set_grid(g[:, :4], g[:, 4].astype(np.int32))
        b = partition_blocks(e.block_costs(), 2)
        e.set_block_range(b[r], b[r + 1])
        out.append(e)
    full = XcEngine(device=0, precision=precision, split_terms=10)
    full.set_system(shell_table(fx))
    full.set_grid(g[:, :4], g[:, 4].astype(np.int32))
    return out, full


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_ranges_sum_to_the_whole_build(water2, precision):
    parts, full = _engines(water2, precision)
    e, n, V = full.build_vxc("B3LYP", water2["PA"])
    ps = [p.build_vxc("B3LYP", water2["PA"]) for p in parts]
    assert abs(sum(x[0] for x in ps) - e) < 1e-12 * abs(e)
    assert abs(sum(x[1] for x in ps) - n) < 1e-12 * abs(n)
    assert np.abs(ps[0][2] + ps[1][2] - V).max() < 1e-12
    # xc-update on each rank's own points
    ps2 = [p.build_vxc("B3LYP", 0.5 * water2["PA"], incremental=True) for p in parts]
    e2, _, V2 = full.build_vxc("B3LYP", 0.5 * water2["PA"], incremental=True)
    assert abs(sum(x[0] for x in ps2) - e2) < 1e-12 * abs(e2)
    assert np.abs(ps2[0][2] + ps2[1][2] - V2).max() < 1e-12
    for x in parts + [full]:
        x.close()


def test_two_ranges_open_shell_and_gradient(water2):
    uks = golden("ref_uks_water2.npz")
    parts, full = _engines(water2)
    e, na, nb, FA, FB = full.build_vxc_uks("BLYP", uks["PA"], uks["PB"])
    ps = [p.build_vxc_uks("BLYP", uks["PA"], uks["PB"]) for p in parts]
    assert abs(ps[0][0] + ps[1][0] - e) < 1e-12 * abs(e)
    assert np.abs(ps[0][3] + ps[1][3] - FA).max() < 1e-12
    assert np.abs(ps[0][4] + ps[1][4] - FB).max() < 1e-12
    go, _, eg = full.xc_gradient("PBE", water2["PA"])
    gs = [p.xc_gradient("PBE", water2["PA"]) for p in parts]
    assert abs(gs[0][2] + gs[1][2] - eg) < 1e-12 * abs(eg)
    assert np.abs(gs[0][0] + gs[1][0] - go).max() < 1e-11 * np.abs(go).max()
    for x in parts + [full]:
        x.close()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_nccl_front_end_world_one(water2):
    import torch
    import torch.distributed as dist
    from proteindf_b200.sharded import ShardedXcEngine
    from proteindf_b200.xc import XcEngine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda:0"))
    try:
        eng = XcEngine(device=0)
        sh = ShardedXcEngine(eng)
        sh.set_system(shell_table(water2))
        sh.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
        PA = torch.tensor(water2["PA"], device="cuda:0")
        V = torch.zeros_like(PA)
        exc, nel = sh.build_vxc_device("B3LYP", PA, V)
        assert abs(exc - water2["B3LYP_exc"][0]) < 1e-8
        assert (V.cpu().numpy() - water2["B3LYP_vxc"]).__abs__().max() < 1e-7
        # the host-array builds reduce through a CUDA tensor on the NCCL group
        exc, nel, Vh = sh.build_vxc("B3LYP", water2["PA"])
        assert abs(exc - water2["B3LYP_exc"][0]) < 1e-8
        assert np.abs(Vh - water2["B3LYP_vxc"]).max() < 1e-7
        uks = golden("ref_uks_water2.npz")
        eu, na, nb, FA, FB = sh.build_vxc_uks("BLYP", uks["PA"], uks["PB"])
        assert abs(eu - uks["BLYP_exc"][0]) < 1e-8
        assert np.abs(FA - uks["BLYP_vxc_a"]).max() < 1e-7 and np.abs(FB - uks["BLYP_vxc_b"]).max() < 1e-7
        # the distributed-matrix form: the local piece of a 1 x 1 process grid is the whole matrix
        from proteindf_b200.sharded import BlockCyclic
        layout = BlockCyclic(water2["PA"].shape[0], 8, 1, 1)
        el, nl, piece = sh.build_vxc_local("B3LYP", water2["PA"], layout)
        assert abs(el - water2["B3LYP_exc"][0]) < 1e-8
        assert np.abs(piece - water2["B3LYP_vxc"]).max() < 1e-7
        go, gw, eg = sh.xc_gradient("SVWN", water2["PA"])
        go1, _, eg1 = eng.xc_gradient("SVWN", water2["PA"])
        # two builds differ by the order of their FP64 atomic additions only
        assert gw is None and np.abs(go - go1).max() <= 1e-13 * np.abs(go1).max() and abs(eg - eg1) <= 1e-12 * abs(eg1)
        eng.close()
    finally:
        dist.destroy_process_group()
