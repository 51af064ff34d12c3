"""a2afft_b200: B200-native drop-in for the a2afft pencil-decomposed 3D FFT of
humz2k/3D-FFTs-MPI.

Host-side mirror of the reference's two classes over the C ABI of
``liba2afft_b200.so`` (``include/a2afft_b200.h``):

* ``a2aDistribution`` -- ``src/a2afft/distribution/a2adistribution.h:5-41``:
  brick decomposition of an ``Ng^3`` grid over ``world_size`` ranks and the six
  pencil transpose steps.  The ranks are virtual: one device buffer holds every
  rank's brick, rank-major, each brick in the reference's ``[x][y][z]``
  layout.
* ``a2adfft`` -- ``src/a2afft/dfft/a2adfft.h:9-30``: ``make_plans`` /
  ``forward`` / ``inverse`` in place on such a buffer.

plus the 1D helpers of ``src/a2afft/dfft/kernels/kernels.h:5-11``
(``forward_1d_fft``, ``inverse_1d_fft``, ``scale_fft``, ``fast_copy_fft``).

Buffers are CUDA tensors (``complex128`` for ``precision="c128"``, the
reference's ``fftPrecision double``; ``complex64`` for ``"c64"``) with
``world_size * nlocal`` elements, or raw device pointers (``int``).  Every call
goes to the CUDA library; errors raise ``A2AError`` with the library's status
and message.
"""
from __future__ import annotations

import ctypes

from ._lib import (  # noqa: F401
    A2AError,
    C64,
    C128,
    Desc,
    LIB_PATH,
    METHOD_PLAIN,
    METHOD_SPLIT_BF16,
    METHOD_SPLIT_FP16,
    bufptr,
    call,
    lib,
)

__all__ = [
    "A2AError",
    "a2aDistribution",
    "a2adfft",
    "a2aBatch",
    "ipc_export",
    "ipc_import",
    "ipc_release",
    "batch_shapes",
    "forward_1d_fft",
    "inverse_1d_fft",
    "scale_fft",
    "fast_copy_fft",
    "version",
    "decompose",
    "write_dims",
    "write_rank_dumps",
]

_KERNELS = {"d_z_a2a_to_z_pencils", "d_z_pencils_to_z_a2a", "d_x_a2a_to_x_pencils", "d_x_pencils_to_x_a2a",
            "d_y_a2a_to_y_pencils", "d_y_pencils_to_y_a2a", "d_fast_z_to_x", "d_fast_x_to_y", "d_fast_y_to_z"}
_PREC = {"c128": C128, "complex128": C128, "double": C128, "c64": C64, "complex64": C64, "float": C64}
_METHODS = {"plain": METHOD_PLAIN, "split_bf16": METHOD_SPLIT_BF16, "split_fp16": METHOD_SPLIT_FP16}


def ipc_export(buf) -> tuple[bytes, int]:
    """(handle, offset) that lets another process map this CUDA tensor (or
    device address)."""
    ptr = buf if isinstance(buf, int) else buf.data_ptr()
    h = ctypes.create_string_buffer(64)
    off = ctypes.c_uint64()
    call("a2a_ipc_export", ctypes.c_void_p(ptr), h, ctypes.byref(off))
    return h.raw, off.value


def ipc_import(handle: bytes, offset: int) -> int:
    """Device address, in this process, of a buffer another process exported."""
    h = ctypes.create_string_buffer(handle, 64)
    p = ctypes.c_void_p()
    call("a2a_ipc_import", h, ctypes.c_uint64(offset), ctypes.byref(p))
    return p.value


def ipc_release(ptr: int) -> None:
    call("a2a_ipc_release", ctypes.c_void_p(ptr))


def version() -> int:
    return lib().a2a_version()


def _host_ptr(a) -> int:
    """Address of a contiguous host array (numpy array or CPU tensor)."""
    if hasattr(a, "data_ptr"):
        if a.is_cuda or not a.is_contiguous():
            raise ValueError("host buffers must be contiguous CPU tensors")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host buffers must be C-contiguous")
    return a.ctypes.data


def _torch_dtype(prec: int):
    import torch

    return torch.complex128 if prec == C128 else torch.complex64


class a2aDistribution:
    """``a2aDistribution(MPI_Comm, int Ng, int blockSize)``
    (``a2adistribution.cpp:44-113``) over ``world_size`` virtual ranks.

    ``Ng`` may be a 3-tuple ``(nx, ny, nz)`` for a box (an extension the
    reference does not have; only ``a2adfft`` accepts boxes)."""

    def __init__(self, world_size: int, Ng, blockSize: int = 64, precision: str = "c128"):
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        self.precision = _PREC[precision]
        h = ctypes.c_void_p()
        if isinstance(Ng, (tuple, list)):
            nx, ny, nz = (int(v) for v in Ng)
            call("a2a_distribution_create_box", nx, ny, nz, int(world_size), int(blockSize), self.precision,
                 ctypes.byref(h))
        else:
            call("a2a_distribution_create", int(Ng), int(world_size), int(blockSize), self.precision, ctypes.byref(h))
        self._h = h
        d = Desc()
        call("a2a_distribution_describe", self._h, ctypes.byref(d))
        self.ndims = d.ndims
        self.ng = tuple(d.ng)
        self.Ng = self.ng[0]
        self.world_size = d.world_size
        self.dims = list(d.dims)
        self.local_grid_size = list(d.local_grid_size)
        self.nlocal = int(d.nlocal)
        self.nsends = int(d.nsends)
        self.blockSize = d.block_size
        self.element_bytes = int(d.element_bytes)
        self.buffer_bytes = int(d.buffer_bytes)
        self.first_rank = int(d.first_rank)
        self.local_ranks = int(d.local_ranks)
        self._stream = None

    def set_rank_range(self, first: int, count: int) -> None:
        """Hold only virtual ranks [first, first+count) in the buffers passed to
        the per-rank kernels (remaps, fast-axis changes, 1D transforms, scale,
        copy) -- the layout of one process of a distributed run."""
        call("a2a_distribution_set_rank_range", self._h, int(first), int(count))
        self.first_rank, self.local_ranks = int(first), int(count)

    # -- reference public fields per rank (a2adistribution.h:8-17) ----------
    def coords(self, rank: int) -> list[int]:
        c, s = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        call("a2a_rank_coords", self._h, int(rank), c, s)
        return list(c)

    def local_coordinates_start(self, rank: int) -> list[int]:
        c, s = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        call("a2a_rank_coords", self._h, int(rank), c, s)
        return list(s)

    @property
    def handle(self):
        return self._h

    @property
    def dtype(self):
        return _torch_dtype(self.precision)

    def empty(self, device="cuda"):
        """A device buffer of ``local_ranks * nlocal`` elements (all ranks by
        default)."""
        import torch

        return torch.empty(self.local_ranks * self.nlocal, dtype=self.dtype, device=device)

    def set_stream(self, stream) -> None:
        """CUDA stream for the calls that take none (a ``torch.cuda.Stream``,
        a raw handle or ``None`` for the default stream)."""
        self._stream = stream
        handle = getattr(stream, "cuda_stream", stream)
        call("a2a_distribution_set_stream", self._h, ctypes.c_void_p(handle or 0))

    def _buf(self, t):
        if isinstance(t, int):
            return bufptr(t)
        if not t.is_cuda:
            raise ValueError("buffers must be CUDA tensors (or raw device pointers)")
        if t.dtype != self.dtype:
            raise TypeError(f"buffer dtype {t.dtype} does not match the distribution's {self.dtype}")
        n = getattr(self, "local_ranks", self.world_size) * self.nlocal
        if not t.is_contiguous() or t.numel() != n:
            raise ValueError(f"buffer must be contiguous with local_ranks*nlocal = {n} elements")
        return bufptr(t.data_ptr())

    # -- the six steps (a2adistribution.cpp:115-215) -------------------------
    def getZPencils(self, d_Buff1, d_Buff2):
        call("a2a_get_z_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    def returnZPencils(self, d_Buff1, d_Buff2):
        call("a2a_return_z_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    def getXPencils(self, d_Buff1, d_Buff2):
        call("a2a_get_x_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    def returnXPencils(self, d_Buff1, d_Buff2):
        call("a2a_return_x_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    def getYPencils(self, d_Buff1, d_Buff2):
        call("a2a_get_y_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    def returnYPencils(self, d_Buff1, d_Buff2):
        call("a2a_return_y_pencils", self._h, self._buf(d_Buff1), self._buf(d_Buff2))

    # -- the individual kernels (distribution/kernels/kernels.h:3-17) -------
    def alltoall(self, source, dest):
        """``MPI_Alltoall`` of ``nsends`` complexes per peer over the virtual ranks."""
        call("a2a_alltoall", self._h, self._buf(source), self._buf(dest))

    def launch(self, kernel: str, source, dest):
        """One remap kernel by its reference name: ``d_z_a2a_to_z_pencils``,
        ``d_z_pencils_to_z_a2a``, ``d_x_...``, ``d_y_...``, ``d_fast_z_to_x``,
        ``d_fast_x_to_y``, ``d_fast_y_to_z``."""
        if kernel not in _KERNELS:
            raise ValueError(f"unknown kernel {kernel!r}; one of {sorted(_KERNELS)}")
        call("a2a_" + kernel, self._h, self._buf(source), self._buf(dest))

    def write_dims(self, path: str) -> None:
        """The reference's ``dims`` file (``a2adistribution.cpp:101-111``)."""
        write_dims(self.Ng, self.world_size, path)

    def finalize(self) -> None:
        """``a2aDistribution::finalize`` (``a2adistribution.cpp:217-224``)."""
        if self._h:
            call("a2a_distribution_finalize", self._h)
            self._h = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass


def decompose(Ng: int, world_size: int) -> dict:
    """Host-only decomposition: dims, local_grid_size, nlocal (raises
    A2AError where the reference asserts)."""
    dims, loc, n = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), ctypes.c_int64()
    call("a2a_decompose", int(Ng), int(world_size), dims, loc, ctypes.byref(n))
    return {"dims": list(dims), "local_grid_size": list(loc), "nlocal": int(n.value)}


def write_dims(Ng: int, world_size: int, path: str) -> None:
    """Write the reference's ``dims`` file: nine int32 (world_size, Ng,
    nlocal, dims[3], local_grid_size[3]); host only."""
    call("a2a_write_dims", int(Ng), int(world_size), str(path).encode())


def write_rank_dumps(Ng: int, world_size: int, folder: str, inp, fwd, inv) -> None:
    """Write ``<folder>/proc<r>`` for every rank: its brick of ``inp``,
    ``fwd`` and ``inv`` (rank-major host arrays or CUDA tensors, complex128
    or complex64), the layout of the reference test's dumps
    (``tests/test.cpp:69-125``)."""
    import numpy as np

    arrs = []
    for a in (inp, fwd, inv):
        if hasattr(a, "detach"):
            a = a.detach().cpu().numpy()
        arrs.append(np.ascontiguousarray(a).ravel())
    dt = arrs[0].dtype
    if dt not in (np.complex128, np.complex64) or any(a.dtype != dt for a in arrs):
        raise TypeError("dumps are complex128 or complex64, all three the same")
    prec = C128 if dt == np.complex128 else C64
    call("a2a_write_rank_dumps", int(Ng), int(world_size), prec, str(folder).encode(),
         arrs[0].ctypes.data_as(ctypes.c_void_p), arrs[1].ctypes.data_as(ctypes.c_void_p),
         arrs[2].ctypes.data_as(ctypes.c_void_p))


# -- dfft/kernels/kernels.h:5-11 --------------------------------------------


def forward_1d_fft(dist: a2aDistribution, data) -> None:
    """Forward 1D transform of every contiguous length-Ng line
    (``a2affts.cu:7-40``)."""
    call("a2a_forward_1d_fft", dist.handle, dist._buf(data))


def inverse_1d_fft(dist: a2aDistribution, data) -> None:
    """Inverse, unnormalised (``a2affts.cu:42-76``)."""
    call("a2a_inverse_1d_fft", dist.handle, dist._buf(data))


def scale_fft(dist: a2aDistribution, out, data) -> None:
    """``out = data / Ng^3`` (``a2affts.cu:78-92``)."""
    call("a2a_scale_fft", dist.handle, dist._buf(out), dist._buf(data))


def fast_copy_fft(dist: a2aDistribution, out, data) -> None:
    """``out = data`` (``a2affts.cu:94-106``)."""
    call("a2a_fast_copy_fft", dist.handle, dist._buf(out), dist._buf(data))


class a2adfft:
    """``a2adfft(a2aDistribution&)`` (``dfft/a2adfft.cpp:7-16``)."""

    def __init__(self, dist: a2aDistribution, method: str = "plain"):
        self.distribution = dist
        self.Ng = dist.Ng
        self.nlocal = dist.nlocal
        self.world_size = dist.world_size
        self.blockSize = dist.blockSize
        h = ctypes.c_void_p()
        call("a2a_dfft_create", dist.handle, ctypes.byref(h))
        self._h = h
        self.plans_made = 0
        self.d_scratch = None
        if method != "plain":
            self.set_method(method)

    def set_method(self, method: str) -> None:
        call("a2a_dfft_set_method", self._h, _METHODS[method])
        self.plans_made = 0

    def set_autotune(self, enable: bool) -> None:
        call("a2a_dfft_set_autotune", self._h, int(bool(enable)))

    def check_device(self) -> None:
        """Raise A2AError(A2A_ERROR_TIMEOUT) if a pass kernel gave up a
        bounded wait since the last check (after async calls: synchronise
        first)."""
        call("a2a_dfft_check_device", self._h)

    def variant_count(self, pass_index: int) -> int:
        n = ctypes.c_int()
        call("a2a_dfft_variant_count", self._h, int(pass_index), ctypes.byref(n))
        return n.value

    def select_variant(self, pass_index: int, variant: int) -> None:
        """Force launch variant `variant` of pass 0 (Z), 1 (X) or 2 (Y)."""
        call("a2a_dfft_select_variant", self._h, int(pass_index), int(variant))

    def plan_report(self) -> str:
        """Every launch variant of each pass, its make_plans timing and the
        chosen one."""
        buf = ctypes.create_string_buffer(1 << 16)
        call("a2a_dfft_plan_report", self._h, buf, len(buf))
        return buf.value.decode()

    def make_plans(self, d_scratch=None) -> None:
        """``a2adfft::make_plans`` (``a2adfft.cpp:18-24``).  The scratch
        buffer is optional because the fused transform runs in place; when it
        is given, every launch variant of each pass is timed on it (its
        contents are clobbered) and the fastest is kept."""
        self.d_scratch = d_scratch
        call("a2a_dfft_make_plans", self._h, None if d_scratch is None else self.distribution._buf(d_scratch))
        self.plans_made = 1

    def forward(self, d_data, stream=None) -> None:
        """``a2adfft::forward`` (``a2adfft.cpp:26-91``).  Synchronous unless a
        stream is given."""
        if stream is None:
            call("a2a_dfft_forward", self._h, self.distribution._buf(d_data))
        else:
            handle = getattr(stream, "cuda_stream", stream)
            call("a2a_dfft_forward_async", self._h, self.distribution._buf(d_data), ctypes.c_void_p(handle))

    def inverse(self, d_data, stream=None) -> None:
        """``a2adfft::inverse`` (``a2adfft.cpp:93-158``), scaled by 1/Ng^3."""
        if stream is None:
            call("a2a_dfft_inverse", self._h, self.distribution._buf(d_data))
        else:
            handle = getattr(stream, "cuda_stream", stream)
            call("a2a_dfft_inverse_async", self._h, self.distribution._buf(d_data), ctypes.c_void_p(handle))

    backward = inverse

    def forward_host(self, host_data, d_buffer) -> None:
        """Host-staged forward (``fft_demo/fft_3d/fft_3d.c:6-96``): host array
        -> ``d_buffer`` -> transform -> back into the host array."""
        call("a2a_dfft_forward_host", self._h, ctypes.c_void_p(_host_ptr(host_data)),
             self.distribution._buf(d_buffer))

    def inverse_host(self, host_data, d_buffer) -> None:
        """Host-staged inverse (``fft_demo/fft_3d/fft_3d.c:98-189``)."""
        call("a2a_dfft_inverse_host", self._h, ctypes.c_void_p(_host_ptr(host_data)),
             self.distribution._buf(d_buffer))

    def execute_pass(self, d_data, pass_index: int, inverse: bool, stream) -> None:
        """Enqueue one of the three fused passes (0 = Z, 1 = X, 2 = Y)."""
        handle = getattr(stream, "cuda_stream", stream)
        call("a2a_dfft_execute_pass_async", self._h, self.distribution._buf(d_data), int(pass_index), int(inverse),
             ctypes.c_void_p(handle))

    def execute_pass_blocks(self, blocks, pass_index: int, inverse: bool, part: int = 0, nparts: int = 1,
                            stream=None) -> None:
        """One fused pass over a virtual buffer split into ``len(blocks)``
        blocks of equal size (block g = virtual ranks ``[g L, (g+1) L)``), each
        a CUDA tensor of this process or a device address (``int``) mapped
        from another process with ``ipc_import``; enqueues tile part ``part``
        of ``nparts``.  The caller orders the passes."""
        vals = [b if isinstance(b, int) else b.data_ptr() for b in blocks]
        arr = (ctypes.c_void_p * len(vals))(*vals)
        handle = 0 if stream is None else getattr(stream, "cuda_stream", stream)
        call("a2a_dfft_execute_pass_blocks", self._h, arr, len(vals), int(pass_index), int(bool(inverse)), int(part),
             int(nparts), ctypes.c_void_p(handle))

    def set_blocks_kernel(self, persistent: bool) -> None:
        """Multi-block pass bodies: persistent CTAs (default, where compiled
        and the tiles fit: TMA-fed X and Y passes, register-pipelined Z pass)
        or one tile per CTA everywhere."""
        call("a2a_dfft_set_blocks_kernel", self._h, int(bool(persistent)))

    @property
    def launches_per_transform(self) -> int:
        n = ctypes.c_int()
        call("a2a_dfft_launches_per_transform", self._h, ctypes.byref(n))
        return n.value

    def destroy(self) -> None:
        if self._h:
            call("a2a_dfft_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


BATCH_EDGES = (32, 48, 64, 96, 128, 192)


def batch_shapes(cubes: int = 96, seed: int = 3, boxes=((128, 256, 512), (128, 256, 512))):
    """Shapes of the measured batch workload: ``cubes`` cubes whose edges are
    drawn uniformly from 32 48 64 96 128 192 with a seeded generator, then
    the fixed anisotropic boxes."""
    import numpy as np

    rng = np.random.default_rng(seed)
    edges = rng.choice(np.array(BATCH_EDGES), size=cubes)
    return [(int(e),) * 3 for e in edges] + [tuple(int(v) for v in b) for b in boxes]


class a2aBatch:
    """Many independent boxes transformed together: one persistent kernel
    launch per direction, replayed from a CUDA graph.  No reference
    counterpart (the reference plans one grid at a time); box ``b`` has the
    layout ``a2aDistribution(world_size, shapes[b])`` gives it and its
    transform equals that distribution's ``a2adfft`` forward / inverse.

    ``shapes``: list of ``(nx, ny, nz)`` (or ints for cubes); every edge one of
    32 48 64 96 128 192 256 512."""

    def __init__(self, shapes, world_size: int = 4, precision: str = "c64"):
        self.shapes = [tuple(int(v) for v in ((s,) * 3 if isinstance(s, int) else s)) for s in shapes]
        self.world_size = int(world_size)
        self.precision = precision
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        self._prec = _PREC[precision]
        flat = [v for s in self.shapes for v in s]
        arr = (ctypes.c_int * len(flat))(*flat)
        h = ctypes.c_void_p()
        call("a2a_batch_create", len(self.shapes), arr, self.world_size, self._prec, ctypes.byref(h))
        self._h = h
        self.elements = []
        for b in range(len(self.shapes)):
            n = ctypes.c_int64()
            call("a2a_batch_box_elements", self._h, b, ctypes.byref(n))
            self.elements.append(n.value)

    @property
    def nboxes(self) -> int:
        return len(self.shapes)

    @property
    def dtype(self):
        return _torch_dtype(self._prec)

    def offsets(self, align_elems: int = 32) -> list[int]:
        """Element offsets of the boxes packed into one flat buffer, each
        rounded up to ``align_elems`` (256 bytes for complex64 at 32)."""
        out, pos = [], 0
        for n in self.elements:
            out.append(pos)
            pos += (n + align_elems - 1) // align_elems * align_elems
        return out + [pos]

    def empty(self, device="cuda"):
        """(flat tensor, per-box views): every box in one allocation."""
        import torch

        offs = self.offsets()
        flat = torch.empty(offs[-1], dtype=self.dtype, device=device)
        views = [flat[offs[b]:offs[b] + self.elements[b]] for b in range(self.nboxes)]
        return flat, views

    def _ptrs(self, bufs):
        if len(bufs) != self.nboxes:
            raise ValueError(f"expected {self.nboxes} buffers, got {len(bufs)}")
        vals = []
        for b, t in enumerate(bufs):
            if isinstance(t, int):
                vals.append(t)
                continue
            if not t.is_cuda or t.dtype != self.dtype or t.numel() < self.elements[b] or not t.is_contiguous():
                raise ValueError(f"box {b}: expected a contiguous CUDA {self.dtype} tensor of >= "
                                 f"{self.elements[b]} elements")
            vals.append(t.data_ptr())
        return (ctypes.c_void_p * self.nboxes)(*vals)

    def make_plans(self, d_scratch=None) -> None:
        call("a2a_batch_make_plans", self._h, None if d_scratch is None else self._ptrs(d_scratch))

    def set_schedule(self, fused: bool = True, claim: int = 16, prefetch: bool = True,
                     grouped: bool = False) -> None:
        """One launch per direction (``fused``) or one per pass; work items
        a CTA takes per queue access; L2 prefetch of each CTA's next tile.
        ``grouped``: instead, the boxes of each shape as one tall grid per
        pass through the single-grid pass kernels, the shapes on parallel
        stream branches (``claim`` and ``prefetch`` then do not apply)."""
        call("a2a_batch_set_schedule", self._h, 2 if grouped else int(bool(fused)), int(claim),
             int(bool(prefetch)))

    def select_variant(self, length: int, batch_mode: bool, variant: int) -> None:
        call("a2a_batch_select_variant", self._h, int(length), int(bool(batch_mode)), int(variant))

    def set_graph(self, enable: bool) -> None:
        call("a2a_batch_set_graph", self._h, int(bool(enable)))

    def inject_stall(self, enable: bool) -> None:
        call("a2a_batch_inject_stall", self._h, int(bool(enable)))

    def plan_report(self) -> str:
        buf = ctypes.create_string_buffer(1 << 16)
        call("a2a_batch_plan_report", self._h, buf, len(buf))
        return buf.value.decode()

    def forward(self, d_data, stream=None) -> None:
        if stream is None:
            call("a2a_batch_forward", self._h, self._ptrs(d_data))
        else:
            handle = getattr(stream, "cuda_stream", stream)
            call("a2a_batch_forward_async", self._h, self._ptrs(d_data), ctypes.c_void_p(handle))

    def inverse(self, d_data, stream=None) -> None:
        if stream is None:
            call("a2a_batch_inverse", self._h, self._ptrs(d_data))
        else:
            handle = getattr(stream, "cuda_stream", stream)
            call("a2a_batch_inverse_async", self._h, self._ptrs(d_data), ctypes.c_void_p(handle))

    def check_device(self) -> None:
        call("a2a_batch_check_device", self._h)

    @property
    def launches_per_transform(self) -> int:
        n = ctypes.c_int()
        call("a2a_batch_launches_per_transform", self._h, ctypes.byref(n))
        return n.value

    def destroy(self) -> None:
        if self._h:
            call("a2a_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

