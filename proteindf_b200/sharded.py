"""One molecule's XC build sharded over GPUs, one process per GPU.

The reference's distributed variant gives every MPI rank a share of the grid
rows and all-reduces F and E (src/libpdf/DfCalcGridX_Parallel.cpp:191-239).
Here every rank holds the whole system, grid and density (they are small next
to the per-block intermediates), builds only its contiguous range of grid
blocks, and one all-reduce (NCCL over NVLink for CUDA tensors, gloo for CPU
tensors) sums the partial Vxc with Exc and the electron count appended. Ranges
come from pdfxc_partition_blocks over the blocks' contraction costs
4 nb^2 np, so ranks get near-equal work; the blocks are in Morton order, so a
range is also a compact region of space. The stored densities of xc-update stay
on the rank that owns the points, so incremental builds need no exchange.
"""
import numpy as np

from .xc import partition_blocks


def _dist():
    import torch.distributed as dist
    return dist


def allreduce_partials(V, scalars, group=None):
    """Sum a rank's partial Vxc (array or torch tensor, n x n) and scalars (Exc,
    electron counts) over the process group in one collective. Host arrays go
    through a CPU tensor; torch tensors are reduced where they live. Returns
    (V_sum, scalars_sum) of the input's kind."""
    import torch
    dist = _dist()
    if isinstance(V, torch.Tensor):
        sc = torch.as_tensor(np.asarray(scalars, dtype=np.float64), device=V.device)
        buf = torch.cat([V.reshape(-1), sc])
        dist.all_reduce(buf, group=group)
        n = V.numel()
        V.copy_(buf[:n].view_as(V))
        return V, buf[n:].cpu().numpy()
    V = np.ascontiguousarray(V, dtype=np.float64)
    buf = torch.from_numpy(np.concatenate([V.ravel(), np.asarray(scalars, dtype=np.float64)]))
    dist.all_reduce(buf, group=group)
    out = buf.numpy()
    return out[:V.size].reshape(V.shape), out[V.size:]


class ShardedXcEngine:
    """Wraps an XcEngine of this rank's GPU; rank and world come from torch.distributed."""

    def __init__(self, engine, group=None):
        dist = _dist()
        self.eng = engine
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.bounds = None

    def set_system(self, sh):
        self.eng.set_system(sh)

    def set_grid(self, xyzw, atom=None):
        self.eng.set_grid(xyzw, atom)
        self.bounds = partition_blocks(self.eng.block_costs(), self.world)
        self.eng.set_block_range(self.bounds[self.rank], self.bounds[self.rank + 1])

    def build_vxc(self, functional, PA, incremental=False):
        """Host build: returns (exc, nelec_alpha, Vxc) of the whole molecule on every rank."""
        exc, nel, V = self.eng.build_vxc(functional, PA, incremental=incremental)
        V, sc = allreduce_partials(V, [exc, nel], self.group)
        return sc[0], sc[1], V

    def build_vxc_device(self, functional, PA, V, incremental=False):
        """Device build on torch CUDA tensors PA (input) and V (output, n x n FP64): V
        holds the whole molecule's Vxc after the all-reduce. Returns (exc, nelec_alpha)."""
        exc, nel = self.eng.build_vxc_device(functional, PA.data_ptr(), V.data_ptr(), incremental=incremental)
        _, sc = allreduce_partials(V, [exc, nel], self.group)
        return sc[0], sc[1]

    def build_vxc_uks(self, functional, PA, PB, incremental=False):
        exc, na, nb, FA, FB = self.eng.build_vxc_uks(functional, PA, PB, incremental=incremental)
        n = FA.size
        both, sc = allreduce_partials(np.concatenate([FA.ravel(), FB.ravel()]), [exc, na, nb], self.group)
        return sc[0], sc[1], sc[2], both[:n].reshape(FA.shape), both[n:].reshape(FB.shape)

    def xc_gradient(self, functional, PA, w_single=None, becke_radius=None, size_adjust=True):
        go, gw, exc = self.eng.xc_gradient(functional, PA, w_single=w_single, becke_radius=becke_radius,
                                           size_adjust=size_adjust)
        stack = np.concatenate([go.ravel(), (gw if gw is not None else np.zeros_like(go)).ravel()])
        tot, sc = allreduce_partials(stack, [exc], self.group)
        k = go.size
        return tot[:k].reshape(go.shape), (tot[k:].reshape(go.shape) if gw is not None else None), sc[0]
