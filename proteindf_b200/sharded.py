"""One molecule's XC build sharded over GPUs, one process per GPU.

The reference's distributed variant gives every MPI rank a share of the grid
rows and all-reduces F and E (src/libpdf/DfCalcGridX_Parallel.cpp:191-239).
Here every rank holds the whole system, grid and density (they are small next
to the per-block intermediates), builds only its contiguous range of grid
blocks, and one all-reduce sums the partial results. Ranges come from
pdfxc_partition_blocks over the blocks' contraction costs 4 nb^2 np, so ranks
get near-equal work; the blocks are in Morton order, so a range is also a
compact region of space. The stored densities of xc-update stay on the rank
that owns the points, so incremental builds need no exchange.

The exchange: each symmetric partial Vxc is packed to its upper triangle
(n (n + 1) / 2 values, row by row; pdfxc_pack_upper on the device), the scalars
(Exc, electron counts) are appended, and one all-reduce sums the buffer, which
is then unpacked into both triangles. On an NCCL group the buffer is a CUDA
tensor on the rank's device (host partials are copied there and back); on a
gloo group host partials are reduced as CPU tensors.
"""
import ctypes

import numpy as np

from .xc import load_library, partition_blocks


def _dist():
    import torch.distributed as dist
    return dist


def _is_nccl(group):
    return _dist().get_backend(group) == "nccl"


def _packed_size(n):
    return n * (n + 1) // 2


def _pack_host(V):
    n = V.shape[0]
    return np.concatenate([V[i, i:] for i in range(n)]) if n else np.zeros(0)


def _unpack_host(p, n):
    V = np.empty((n, n), dtype=np.float64)
    o = 0
    for i in range(n):
        V[i, i:] = p[o:o + n - i]
        V[i:, i] = p[o:o + n - i]
        o += n - i
    return V


def _reduce_device(mats, scalars, device, group):
    """mats: list of symmetric (n, n) CUDA float64 tensors, reduced in place; returns the summed scalars."""
    import torch
    L = load_library()
    stream = torch.cuda.current_stream(device).cuda_stream
    m = [_packed_size(V.shape[0]) for V in mats]
    k = len(scalars)
    buf = torch.empty(sum(m) + k, dtype=torch.float64, device=device)
    o = 0
    for V, mi in zip(mats, m):
        if L.pdfxc_pack_upper(ctypes.c_void_p(V.data_ptr()), V.shape[0], ctypes.c_void_p(buf[o:].data_ptr()),
                              ctypes.c_void_p(stream)) != 0:
            raise RuntimeError("pdfxc_pack_upper failed")
        o += mi
    buf[o:] = torch.as_tensor(np.asarray(scalars, dtype=np.float64), device=device)
    _dist().all_reduce(buf, group=group)
    o = 0
    for V, mi in zip(mats, m):
        if L.pdfxc_unpack_upper(ctypes.c_void_p(buf[o:].data_ptr()), V.shape[0], ctypes.c_void_p(V.data_ptr()),
                                ctypes.c_void_p(stream)) != 0:
            raise RuntimeError("pdfxc_unpack_upper failed")
        o += mi
    return buf[o:].cpu().numpy()


def allreduce_partials(mats, scalars, group=None, device=None):
    """Sum the ranks' partial symmetric matrices and scalars in one collective.

    mats: one matrix or a list of them, each a host array or a CUDA tensor (n x n,
    symmetric; only the upper triangle travels). CUDA tensors are reduced in place.
    Host arrays on an NCCL group go through a CUDA tensor on `device`. Returns
    (summed matrices in the input's kind -- one or a list, as given --, summed scalars)."""
    import torch
    dist = _dist()
    single = not isinstance(mats, (list, tuple))
    mats = [mats] if single else list(mats)
    if all(isinstance(V, torch.Tensor) and V.is_cuda for V in mats):
        sc = _reduce_device(mats, scalars, mats[0].device, group)
        return (mats[0] if single else mats), sc
    host = [np.ascontiguousarray(V, dtype=np.float64) for V in mats]
    if _is_nccl(group):
        dev = torch.device("cuda", device if device is not None else torch.cuda.current_device())
        dmats = [torch.from_numpy(V).to(dev) for V in host]
        sc = _reduce_device(dmats, scalars, dev, group)
        out = [V.cpu().numpy() for V in dmats]
    else:
        buf = torch.from_numpy(np.concatenate([_pack_host(V) for V in host] + [np.asarray(scalars, np.float64)]))
        dist.all_reduce(buf, group=group)
        b = buf.numpy()
        out, o = [], 0
        for V in host:
            mi = _packed_size(V.shape[0])
            out.append(_unpack_host(b[o:o + mi], V.shape[0]))
            o += mi
        sc = b[o:]
    return (out[0] if single else out), sc


def allreduce_vector(v, group=None, device=None):
    """Sum a small host vector (gradients, energies) over the group (a CUDA tensor on NCCL)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).copy())
    if _is_nccl(group):
        dev = torch.device("cuda", device if device is not None else torch.cuda.current_device())
        t = t.to(dev)
    _dist().all_reduce(t, group=group)
    return t.cpu().numpy()


class ShardedXcEngine:
    """Wraps an XcEngine of this rank's GPU; rank and world come from torch.distributed."""

    def __init__(self, engine, group=None):
        dist = _dist()
        self.eng = engine
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.bounds = None

    @property
    def _device(self):
        return getattr(self.eng, "device", None)

    def set_system(self, sh):
        self.eng.set_system(sh)

    def set_grid(self, xyzw, atom=None):
        self.eng.set_grid(xyzw, atom)
        self.bounds = partition_blocks(self.eng.block_costs(), self.world)
        self.eng.set_block_range(self.bounds[self.rank], self.bounds[self.rank + 1])

    def build_vxc(self, functional, PA, incremental=False):
        """Host build: returns (exc, nelec_alpha, Vxc) of the whole molecule on every rank."""
        exc, nel, V = self.eng.build_vxc(functional, PA, incremental=incremental)
        V, sc = allreduce_partials(V, [exc, nel], self.group, self._device)
        return sc[0], sc[1], V

    def build_vxc_device(self, functional, PA, V, incremental=False):
        """Device build on torch CUDA tensors PA (input) and V (output, n x n FP64): V
        holds the whole molecule's Vxc after the all-reduce. Returns (exc, nelec_alpha)."""
        exc, nel = self.eng.build_vxc_device(functional, PA.data_ptr(), V.data_ptr(), incremental=incremental)
        _, sc = allreduce_partials(V, [exc, nel], self.group)
        return sc[0], sc[1]

    def build_vxc_uks(self, functional, PA, PB, incremental=False):
        exc, na, nb, FA, FB = self.eng.build_vxc_uks(functional, PA, PB, incremental=incremental)
        (FA, FB), sc = allreduce_partials([FA, FB], [exc, na, nb], self.group, self._device)
        return sc[0], sc[1], sc[2], FA, FB

    def xc_gradient(self, functional, PA, w_single=None, becke_radius=None, size_adjust=True):
        go, gw, exc = self.eng.xc_gradient(functional, PA, w_single=w_single, becke_radius=becke_radius,
                                           size_adjust=size_adjust)
        stack = np.concatenate([go.ravel(), (gw if gw is not None else np.zeros_like(go)).ravel(), [exc]])
        tot = allreduce_vector(stack, self.group, self._device)
        k = go.size
        return tot[:k].reshape(go.shape), (tot[k:2 * k].reshape(go.shape) if gw is not None else None), tot[-1]
