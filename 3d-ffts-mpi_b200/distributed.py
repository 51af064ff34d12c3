"""The a2afft distribution layer across processes: the P virtual ranks of the
reference's brick grid spread over the processes of a ``torch.distributed``
group, one process per GPU, each holding a contiguous block of
``L = P / G`` ranks (``[g L, (g+1) L)``).

The reference runs one MPI rank per GPU and exchanges with ``MPI_Alltoall``
(``src/a2afft/distribution/a2adistribution.cpp:115-215``), either staged
through host memory (its default, ``:160-163``) or on device buffers with
CUDA-aware MPI (``-Dcudampi``, ``:164-166``).  Here the alltoall over the P
virtual ranks is one ``all_to_all_single`` between the G processes (NCCL over
NVLink for CUDA tensors in ``mode="device"``; ``mode="host"`` stages through
host memory like the reference's default) bracketed by two local chunk
reorders; the per-rank remaps, fast-axis changes and batched 1D transforms
run on this process's block through ``liba2afft_b200`` (its rank range set
with ``a2a_distribution_set_rank_range``).  ``DistributedDfft.forward`` /
``inverse`` follow ``a2adfft::forward``/``inverse`` (``dfft/a2adfft.cpp:26-158``)
step for step: 12 exchanges per transform, as in the reference.

Every process takes the same collective steps in the same order.
"""
from __future__ import annotations

from . import (a2aDistribution, a2adfft, decompose, fast_copy_fft, forward_1d_fft, inverse_1d_fft, ipc_export,
               ipc_import, ipc_release, scale_fft)


class CudaLocal:
    """The per-rank kernels of this process's block, on its GPU."""

    def __init__(self, world_size, Ng, blockSize, precision, first, count):
        self.dist = a2aDistribution(world_size, Ng, blockSize, precision)
        self.dist.set_rank_range(first, count)

    def launch(self, kernel, src, dst):
        self.dist.launch(kernel, src, dst)

    def fft1d(self, data, inverse):
        (inverse_1d_fft if inverse else forward_1d_fft)(self.dist, data)

    def scale(self, out, data):
        scale_fft(self.dist, out, data)

    def copy(self, out, data):
        fast_copy_fft(self.dist, out, data)


class DistributedDistribution:
    """``a2aDistribution`` over a process group.  Buffers are this process's
    ``L * nlocal`` elements (its ranks' bricks or pencils, rank-major)."""

    def __init__(self, world_size: int, Ng: int, blockSize: int = 64, precision: str = "c128", group=None,
                 mode: str = "device", local=None):
        import torch.distributed as tdist

        if mode not in ("device", "host"):
            raise ValueError("mode is 'device' (collective on the buffers' device) or 'host' (staged)")
        self.group = group
        self.G = tdist.get_world_size(group)
        self.g = tdist.get_rank(group)
        if world_size % self.G:
            raise ValueError(f"world_size={world_size} virtual ranks do not split over {self.G} processes")
        self.world_size = world_size
        self.Ng = Ng
        self.L = world_size // self.G
        self.first_rank = self.g * self.L
        dec = decompose(Ng, world_size)
        self.dims = dec["dims"]
        self.local_grid_size = dec["local_grid_size"]
        self.nlocal = dec["nlocal"]
        self.nsends = self.nlocal // world_size
        self.mode = mode
        self.local = local if local is not None else CudaLocal(world_size, Ng, blockSize, precision,
                                                               self.first_rank, self.L)

    # -- MPI_Alltoall over the virtual ranks --------------------------------
    def alltoall(self, send, recv):
        """``recv[q][r] = send[r][q]`` (chunks of ``nsends``) over all P virtual
        ranks: chunks bound for process h gathered, one all_to_all_single,
        received chunks put in sender order."""
        import torch
        import torch.distributed as tdist

        L, G, C = self.L, self.G, self.nsends
        out = send.view(L, G, L, C).permute(1, 0, 2, 3).contiguous()  # [dest proc][sender][dest rank][chunk]
        if self.mode == "host":
            staged = out.cpu()
            back = torch.empty_like(staged)
            tdist.all_to_all_single(back, staged, group=self.group)
            back = back.to(recv.device)
        else:
            back = torch.empty_like(out)
            tdist.all_to_all_single(back, out, group=self.group)
        recv.view(L, G, L, C).copy_(back.permute(2, 0, 1, 3))  # [dest rank][source proc][sender][chunk]

    # -- the six steps (a2adistribution.cpp:115-215) -------------------------
    def getZPencils(self, b1, b2):
        self.alltoall(b1, b2)
        self.local.launch("d_z_a2a_to_z_pencils", b2, b1)

    def returnZPencils(self, b1, b2):
        self.local.launch("d_z_pencils_to_z_a2a", b1, b2)
        self.alltoall(b2, b1)

    def getXPencils(self, b1, b2):
        self.local.launch("d_fast_z_to_x", b1, b2)
        self.alltoall(b2, b1)
        self.local.launch("d_x_a2a_to_x_pencils", b1, b2)

    def returnXPencils(self, b1, b2):
        self.local.launch("d_x_pencils_to_x_a2a", b2, b1)
        self.alltoall(b1, b2)

    def getYPencils(self, b1, b2):
        self.local.launch("d_fast_x_to_y", b2, b1)
        self.alltoall(b1, b2)
        self.local.launch("d_y_a2a_to_y_pencils", b2, b1)

    def returnYPencils(self, b1, b2):
        self.local.launch("d_y_pencils_to_y_a2a", b2, b1)
        self.alltoall(b1, b2)
        self.local.launch("d_fast_y_to_z", b2, b1)


class DistributedDfft:
    """``a2adfft`` over a ``DistributedDistribution`` (``dfft/a2adfft.cpp``)."""

    def __init__(self, dist: DistributedDistribution):
        self.distribution = dist
        self.d_scratch = None
        self.plans_made = 0

    def make_plans(self, d_scratch) -> None:
        self.d_scratch = d_scratch
        self.plans_made = 1

    def _run(self, d_data, inverse):
        if not self.plans_made:
            raise RuntimeError("make_plans has not been called")
        d, s, loc = self.distribution, self.d_scratch, self.distribution.local
        d.getZPencils(d_data, s)
        loc.fft1d(d_data, inverse)
        d.returnZPencils(d_data, s)
        d.getXPencils(d_data, s)
        loc.fft1d(s, inverse)
        d.returnXPencils(d_data, s)
        d.getYPencils(d_data, s)
        loc.fft1d(d_data, inverse)
        if inverse:
            loc.scale(s, d_data)  # a2adfft.cpp:147
        else:
            loc.copy(s, d_data)  # a2adfft.cpp:79
        d.returnYPencils(d_data, s)

    def forward(self, d_data) -> None:
        self._run(d_data, False)

    def inverse(self, d_data) -> None:
        self._run(d_data, True)

    backward = inverse


class FusedDistributedDfft:
    """The transform across processes (one per GPU) with the fused pass: no
    alltoall.  Process g holds virtual ranks ``[g L, (g+1) L)`` (L = P / G) in
    one device buffer; ``bind`` maps every other process's buffer into this
    one (CUDA IPC), then each of the 3 passes of a transform is one kernel per
    process over its share of the pass's tiles, reading and writing the
    owners' bricks directly (peer loads and stores over NVLink), with a
    group barrier between passes.  Same result as ``DistributedDfft``; each
    element crosses the link once each way per pass, as in the reference's
    get/return alltoall pair, without the separate pack/unpack passes."""

    def __init__(self, world_size: int, Ng, precision: str = "c64", group=None):
        import torch.distributed as tdist

        self.group = group
        self.G = tdist.get_world_size(group)
        self.g = tdist.get_rank(group)
        if world_size % self.G:
            raise ValueError(f"world_size={world_size} virtual ranks do not split over {self.G} processes")
        self.world_size = world_size
        self.dist = a2aDistribution(world_size, Ng, 64, precision)
        self.dfft = a2adfft(self.dist)
        self.L = world_size // self.G
        self.block_elems = self.L * self.dist.nlocal
        self.blocks = None
        self._imported = []

    def _check_block(self, d_data):
        """Why ``d_data`` cannot serve as this process's block ('' if it can):
        the fused kernels of every process index it as ``block_elems``
        elements of the distribution's own element type, so a buffer of the
        wrong type, shape or length would let peer loads and stores run past
        its allocation."""
        import torch

        want = self.dist.dtype
        if not isinstance(d_data, torch.Tensor) or not d_data.is_cuda:
            return "the block must be a CUDA tensor"
        if d_data.dtype != want:
            return f"the block must be {want} for this distribution, not {d_data.dtype}"
        if not d_data.is_contiguous():
            return "the block must be contiguous"
        if d_data.numel() * d_data.element_size() < self.block_elems * self.dist.element_bytes:
            return f"the block needs {self.block_elems} elements, it has {d_data.numel()}"
        return ""

    def bind(self, d_data) -> None:
        """Exchange buffer handles with every process (collective).  Every
        process checks its own block first and all of them raise if any
        block is unusable, so no process maps a bad buffer or waits alone."""
        import torch.distributed as tdist

        why = self._check_block(d_data)
        mine = (why, None if why else ipc_export(d_data))
        allh = [None] * self.G
        tdist.all_gather_object(allh, mine, group=self.group)
        bad = [(q, w) for q, (w, _) in enumerate(allh) if w]
        if bad:
            raise ValueError("; ".join(f"process {q}: {w}" for q, w in bad))
        self.release()
        blocks = []
        for q, (_, (h, off)) in enumerate(allh):
            if q == self.g:
                blocks.append(d_data.data_ptr())
            else:
                p = ipc_import(h, off)
                self._imported.append(p)
                blocks.append(p)
        self.blocks = blocks

    def _run(self, inverse: bool) -> None:
        import torch
        import torch.distributed as tdist

        if self.blocks is None:
            raise RuntimeError("bind() first")
        if self.G == 1:  # one process: the passes are ordered by its stream
            for p in range(3):
                self.dfft.execute_pass_blocks(self.blocks, p, inverse, 0, 1)
            return
        torch.cuda.synchronize()
        tdist.barrier(group=self.group)  # every block holds its input
        for p in range(3):
            self.dfft.execute_pass_blocks(self.blocks, p, inverse, self.g, self.G)
            torch.cuda.synchronize()
            tdist.barrier(group=self.group)  # pass p complete everywhere

    def forward(self) -> None:
        self._run(False)

    def inverse(self) -> None:
        self._run(True)

    def release(self) -> None:
        for p in self._imported:
            ipc_release(p)
        self._imported = []
        self.blocks = None

