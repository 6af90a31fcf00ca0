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

The distributed-matrix form (build_vxc_local) takes P_A and returns Vxc as each
rank's block-cyclic piece (BlockCyclic): an all-gather assembles P_A, the rank
builds its block range, and a reduce-scatter returns the summed pieces.
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


class BlockCyclic:
    """The 2-D block-cyclic layout of an n x n matrix over a pr x pc process grid (ScaLAPACK's,
    square blocks of nb; rank r sits at grid row r // pc, column r % pc). A rank's local
    matrix holds the global rows i with (i // nb) % pr == its grid row and the global columns j
    with (j // nb) % pc == its grid column, in ascending order: the reference's
    TlDenseGeneralMatrix_Scalapack::getLocalMatrix with getRowIndexTable / getColIndexTable
    (src/libpdf/DfCalcGridX_Parallel.cpp:481-487)."""

    def __init__(self, n, nb, pr, pc):
        if n < 0 or nb < 1 or pr < 1 or pc < 1:
            raise ValueError("BlockCyclic: n >= 0, nb >= 1 and a positive process grid")
        self.n, self.nb, self.pr, self.pc = int(n), int(nb), int(pr), int(pc)

    @property
    def world(self):
        return self.pr * self.pc

    def rows(self, rank):
        idx = np.arange(self.n)
        return idx[(idx // self.nb) % self.pr == rank // self.pc]

    def cols(self, rank):
        idx = np.arange(self.n)
        return idx[(idx // self.nb) % self.pc == rank % self.pc]

    def local_shape(self, rank):
        return len(self.rows(rank)), len(self.cols(rank))

    def flat_index(self, rank):
        """Global flat indices (i n + j) of the rank's local matrix, row-major."""
        return (self.rows(rank)[:, None] * self.n + self.cols(rank)[None, :]).ravel()


def gather_block_cyclic(local, layout, group=None, device=None):
    """The whole n x n matrix from every rank's local block-cyclic piece, on every rank: one
    all-gather of the pieces (padded to the largest), then each placed at its global indices.
    `local` is a host array or a CUDA tensor; the result is of the same kind (a CUDA tensor on
    `device` for an NCCL group)."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    if world != layout.world:
        raise ValueError(f"gather_block_cyclic: the layout is for {layout.world} ranks, the group has {world}")
    cuda = isinstance(local, torch.Tensor) and local.is_cuda
    nccl = _is_nccl(group)
    dev = (local.device if cuda else torch.device("cuda", device if device is not None else torch.cuda.current_device())
           if nccl else torch.device("cpu"))
    t = local if isinstance(local, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64))
    t = t.to(dev, dtype=torch.float64).reshape(-1)
    m = max(int(np.prod(layout.local_shape(r))) for r in range(world))
    buf = torch.zeros(m, dtype=torch.float64, device=dev)
    buf[:t.numel()] = t
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    full = torch.empty(layout.n * layout.n, dtype=torch.float64, device=dev)
    for r in range(world):
        fi = torch.as_tensor(layout.flat_index(r), device=dev)
        full[fi] = parts[r][:fi.numel()]
    full = full.reshape(layout.n, layout.n)
    return full if cuda else full.cpu().numpy()


def reduce_scatter_block_cyclic(full, layout, group=None, device=None):
    """Each rank's local block-cyclic piece of the sum over ranks of `full` (n x n partial
    sums, host array or CUDA tensor). On NCCL one reduce-scatter of the pieces packed in rank
    order (padded to the largest); on gloo, which has no reduce-scatter, an all-reduce of the
    matrix and this rank's piece taken from it. Returns the piece (local rows x local columns)
    in the input's kind."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    if world != layout.world:
        raise ValueError(f"reduce_scatter_block_cyclic: the layout is for {layout.world} ranks, the group has {world}")
    cuda = isinstance(full, torch.Tensor) and full.is_cuda
    shape = layout.local_shape(rank)
    if _is_nccl(group):
        dev = full.device if cuda else torch.device("cuda", device if device is not None else torch.cuda.current_device())
        f = (full if cuda else torch.from_numpy(np.ascontiguousarray(full, dtype=np.float64))).to(dev).reshape(-1)
        m = max(int(np.prod(layout.local_shape(r))) for r in range(world))
        send = torch.zeros(world * m, dtype=torch.float64, device=dev)
        for r in range(world):
            fi = torch.as_tensor(layout.flat_index(r), device=dev)
            send[r * m:r * m + fi.numel()] = f[fi]
        out = torch.empty(m, dtype=torch.float64, device=dev)
        dist.reduce_scatter_tensor(out, send, group=group)
        piece = out[:shape[0] * shape[1]].reshape(shape)
        return piece if cuda else piece.cpu().numpy()
    f = (full.cpu() if cuda else torch.from_numpy(np.ascontiguousarray(full, dtype=np.float64)).clone()).reshape(-1)
    dist.all_reduce(f, group=group)
    piece = f[torch.as_tensor(layout.flat_index(rank))].reshape(shape)
    return piece.to(full.device) if cuda else piece.numpy()


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

    def build_vxc_local(self, functional, PA_local, layout, incremental=False):
        """The distributed-matrix form (the reference's DfCalcGridX_Parallel with ScaLAPACK
        matrices, src/libpdf/DfCalcGridX_Parallel.cpp:481-664): P_A arrives as this rank's
        block-cyclic piece and Vxc leaves as this rank's piece. P_A is all-gathered, the rank
        builds its range of grid blocks, and one reduce-scatter sums the partial Vxc into the
        pieces (the reference instead evaluates every grid point on every rank for its local
        rows and columns and all-reduces the grid matrix's densities). Returns (exc,
        nelec_alpha, Vxc piece)."""
        PA = gather_block_cyclic(PA_local, layout, self.group, self._device)
        exc, nel, V = self.eng.build_vxc(functional, PA, incremental=incremental)
        piece = reduce_scatter_block_cyclic(V, layout, self.group, self._device)
        sc = allreduce_vector(np.array([exc, nel]), self.group, self._device)
        return sc[0], sc[1], piece

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
