"""CPU oracle for the a2afft pencil-decomposed 3D FFT -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy, what the reference library
(humz2k/3D-FFTs-MPI, ``src/a2afft``) computes on every MPI rank, with the P
ranks held as a leading array axis ("virtual ranks").  It is the checker for
the CUDA library in ``3d-ffts-mpi_b200/``: only ``tests/``, the smoke check in
``__graft_entry__.py`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  The product path never calls it.

What is restated, and from where:

* decomposition -- ``MPI_Dims_create(P, 3)`` (balanced, non-increasing; the
  MPI standard's rule, which the reference calls at
  ``src/a2afft/distribution/a2adistribution.cpp:59``), ``rank2coords``
  (``a2adistribution.cpp:14-20``), ``topology2localgrid`` (``:25-31``),
  ``get_local_grid_start`` (``:36-42``) and the divisibility asserts
  (``:61-80``);
* the alltoall -- ``MPI_Alltoall`` with ``nsends = nlocal / P`` complexes per
  peer (``a2adistribution.cpp:117-125`` and the five other call sites);
* the six pack/unpack remaps of ``distribution/kernels/a2apencils.cu`` and the
  three fast-axis changes of ``distribution/kernels/a2achangefastaxis.cu``,
  written here from the pencil geometry they implement (sender groups,
  mini-pencils, chunk lines), NOT from their index arithmetic; they are
  pinned bit-exactly against the reference's own CPU copies of those
  functions (``src/pencils_demo/a2a_to_pencils/a2a_to_pencils.c``,
  ``src/pencils_demo/change_fast_axis/change_fast_axis.c``) compiled into
  ``oracle/_ref/`` and against the committed fixtures in ``tests/golden/``;
* the one reference map that is not a permutation on most grids,
  ``d_y_pencils_to_y_a2a`` (``a2apencils.cu:189-208``), is restated twice:
  ``y_pencils_to_y_a2a_ref_map`` reproduces the reference's destination
  formula (so its non-injectivity can be shown), and
  ``y_pencils_to_y_a2a_map`` is the true inverse of the Y unpack, which is
  what the pipeline uses;
* ``a2adfft::forward`` / ``a2adfft::inverse`` (``dfft/a2adfft.cpp:26-158``)
  step for step, including the parity copy (``a2affts.cu:94-106``) and the
  ``1/Ng^3`` scale (``a2affts.cu:78-92``);
* the batched 1D transforms (cuFFT ``Z2Z``/``C2C`` in the reference,
  ``dfft/kernels/a2affts.cu:7-76``; cuFFT is closed and not part of the
  reference tree) as the DFT definition itself: forward kernel
  ``exp(-2 pi i jk/N)``, inverse ``exp(+2 pi i jk/N)``, unnormalised,
  evaluated as a matrix product with twiddles reduced exactly
  (``jk mod N``) and generated in extended precision.  The reference's only
  result check is ``np.allclose(np.fft.fftn(inp), out)``
  (``tests/stitch.py:89``), so ``numpy.fft`` is the cross-check.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------
# Decomposition
# --------------------------------------------------------------------------


def _prime_factors(n: int) -> list[int]:
    out, p = [], 2
    while p * p <= n:
        while n % p == 0:
            out.append(p)
            n //= p
        p += 1
    if n > 1:
        out.append(n)
    return out


def dims_create(nnodes: int, ndims: int = 3) -> list[int]:
    """Balanced non-increasing factorisation of ``nnodes`` into ``ndims``
    factors: the MPI standard's ``MPI_Dims_create`` rule for all-zero input
    dims, as the reference calls it (``a2adistribution.cpp:59``).

    Prime factors are handed out largest first, each to the dimension with
    the smallest running product; the result is sorted non-increasing.  This
    gives [2,2,1] for 4, [3,2,1] for 6, [2,2,2] for 8, [4,2,2] for 16,
    [4,4,4] for 64 and [8,8,4] for 256.
    """
    if nnodes < 1 or ndims < 1:
        raise ValueError("dims_create needs nnodes >= 1 and ndims >= 1")
    dims = [1] * ndims
    for p in sorted(_prime_factors(nnodes), reverse=True):
        i = min(range(ndims), key=lambda k: (dims[k], k))
        dims[i] *= p
    return sorted(dims, reverse=True)


def rank2coords(rank: int, dims) -> tuple[int, int, int]:
    """Row-major rank -> brick coordinates (``a2adistribution.cpp:14-20``)."""
    d1, d2 = dims[1], dims[2]
    return rank // (d1 * d2), (rank // d2) % d1, rank % d2


class DecompositionError(ValueError):
    """A grid the reference would reject with one of its asserts."""


@dataclass
class Decomp:
    """Per-rank brick geometry of ``a2aDistribution``
    (``a2adistribution.cpp:44-80``), generalised to an ``nx x ny x nz`` box
    (the reference itself only takes one ``Ng``)."""

    ng: tuple  # (nx, ny, nz)
    world_size: int
    dims: list = field(default_factory=list)
    local: tuple = ()
    nlocal: int = 0

    def __post_init__(self):
        if isinstance(self.ng, int):
            self.ng = (self.ng, self.ng, self.ng)
        self.ng = tuple(int(v) for v in self.ng)
        P = self.world_size
        if P < 1 or min(self.ng) < 1:
            raise DecompositionError("world_size and grid sizes must be >= 1")
        if not self.dims:
            self.dims = dims_create(P, 3)
        d = self.dims
        for a in range(3):  # a2adistribution.cpp:61-63
            if self.ng[a] % d[a]:
                raise DecompositionError(f"N[{a}]={self.ng[a]} not divisible by dims[{a}]={d[a]}")
        self.local = tuple(self.ng[a] // d[a] for a in range(3))
        lx, ly, lz = self.local
        self.nlocal = lx * ly * lz
        for a in range(3):  # a2adistribution.cpp:74-76
            if P % d[a]:
                raise DecompositionError(f"world_size={P} not divisible by dims[{a}]={d[a]}")
        for pa, pb in ((lx, ly), (lx, lz), (ly, lz)):  # a2adistribution.cpp:78-80
            if (pa * pb) % P:
                raise DecompositionError("a face of the local brick is not divisible by world_size")

    @property
    def chunk(self) -> int:
        """``nsends``: complexes sent to each peer by one alltoall."""
        return self.nlocal // self.world_size

    def coords(self, rank):
        return rank2coords(rank, self.dims)

    def local_start(self, rank):
        c = self.coords(rank)
        return tuple(self.local[a] * c[a] for a in range(3))


# --------------------------------------------------------------------------
# Brick layout <-> global array
# --------------------------------------------------------------------------


def global_to_bricks(g: np.ndarray, d: Decomp) -> np.ndarray:
    """Global ``[x][y][z]`` array -> ``(P, nlocal)`` rank-major bricks, each
    brick ``[x][y][z]`` row-major (the layout ``tests/stitch.py:38-47``
    reassembles)."""
    d0, d1, d2 = d.dims
    lx, ly, lz = d.local
    v = g.reshape(d0, lx, d1, ly, d2, lz).transpose(0, 2, 4, 1, 3, 5)
    return np.ascontiguousarray(v).reshape(d.world_size, d.nlocal)


def bricks_to_global(b: np.ndarray, d: Decomp) -> np.ndarray:
    d0, d1, d2 = d.dims
    lx, ly, lz = d.local
    v = b.reshape(d0, d1, d2, lx, ly, lz).transpose(0, 3, 1, 4, 2, 5)
    return np.ascontiguousarray(v).reshape(d.ng)


def brick_offsets(d: Decomp):
    """Separable element offsets of the rank-major brick layout: global
    ``(x, y, z)`` lives at ``ox[x] + oy[y] + oz[z]``."""
    d0, d1, d2 = d.dims
    lx, ly, lz = d.local
    n = d.nlocal
    x = np.arange(d.ng[0], dtype=np.int64)
    y = np.arange(d.ng[1], dtype=np.int64)
    z = np.arange(d.ng[2], dtype=np.int64)
    ox = (x // lx) * (d1 * d2 * n) + (x % lx) * (ly * lz)
    oy = (y // ly) * (d2 * n) + (y % ly) * lz
    oz = (z // lz) * n + (z % lz)
    return ox, oy, oz


# --------------------------------------------------------------------------
# Alltoall and the remaps
# --------------------------------------------------------------------------


def alltoall(bufs: np.ndarray, d: Decomp) -> np.ndarray:
    """``MPI_Alltoall`` of ``nlocal/P`` complexes per peer over the virtual
    ranks: rank q's slot r receives chunk q of rank r."""
    P, c = d.world_size, d.chunk
    return np.ascontiguousarray(bufs.reshape(P, P, c).transpose(1, 0, 2)).reshape(P, d.nlocal)


_AXIS = {"x": 0, "y": 1, "z": 2}


def _sender_group(axis: str, d: Decomp, r: np.ndarray):
    """For a sender rank r: (group index s of the pencils it contributes to,
    its coordinate along the pencil axis).  Pencils of rank q are ordered by
    s, then by the line inside the alltoall chunk."""
    d0, d1, d2 = d.dims
    c0, c1, c2 = r // (d1 * d2), (r // d2) % d1, r % d2
    if axis == "z":
        return c0 * d1 + c1, c2
    if axis == "x":
        return c1 * d2 + c2, c0
    return c0 * d2 + c2, c1  # "y"


def unpack_map(axis: str, d: Decomp) -> np.ndarray:
    """``new_idx[idx]`` of the ``<axis>_a2a_to_<axis>_pencils`` remap of one
    rank (``a2apencils.cu:5-21`` for z, ``:74-92`` for x, ``:149-168`` for
    y): the received buffer holds, per sender r, ``m`` mini-pencils of length
    ``l_axis``; they are joined into full-length pencils whose element
    ``c_axis(r) * l_axis + e`` comes from sender r."""
    la = d.local[_AXIS[axis]]
    ng = d.ng[_AXIS[axis]]
    c = d.chunk
    m = c // la
    idx = np.arange(d.nlocal, dtype=np.int64)
    r, rem = idx // c, idx % c
    j, e = rem // la, rem % la
    s, ca = _sender_group(axis, d, r)
    return (s * m + j) * ng + ca * la + e


def pack_map(axis: str, d: Decomp) -> np.ndarray:
    """``new_idx[idx]`` of ``<axis>_pencils_to_<axis>_a2a``: the exact inverse
    permutation of ``unpack_map`` (``a2apencils.cu:38-56`` for z,
    ``:111-130`` for x; for y this is the corrected return, see
    ``y_pencils_to_y_a2a_ref_map``)."""
    u = unpack_map(axis, d)
    inv = np.empty_like(u)
    inv[u] = np.arange(u.size, dtype=np.int64)
    return inv


def y_pencils_to_y_a2a_map(d: Decomp) -> np.ndarray:
    return pack_map("y", d)


def y_pencils_to_y_a2a_ref_map(d: Decomp) -> np.ndarray:
    """Destination index the reference's ``d_y_pencils_to_y_a2a`` computes
    (``a2apencils.cu:189-208``).  For pencil element ``idx = p*Ng + n`` with
    pencil group ``s = c0*d2 + c2`` and y-chunk ``c1 = n // ly``, the
    reference takes the destination rank to be ``c1*d2 + s + (s//d2)*d2``
    (``:195-197``); the sender that owns the element is
    ``c0*d1*d2 + c1*d2 + c2``.  Both agree only when ``d1 == 2`` or
    ``d0 == 1``; elsewhere the map is not injective and can leave the
    buffer."""
    d0, d1, d2 = d.dims
    ly = d.local[1]
    ng = d.ng[1]
    c = d.chunk
    m = c // ly
    idx = np.arange(d.nlocal, dtype=np.int64)
    p, n = idx // ng, idx % ng
    s, j = p // m, p % m
    c1, e = n // ly, n % ly
    rank_ref = c1 * d2 + s + (s // d2) * d2
    return rank_ref * c + j * ly + e


def y_return_is_valid(d: Decomp) -> bool:
    """True where the reference's Y pack equals the true inverse."""
    return bool(np.array_equal(y_pencils_to_y_a2a_ref_map(d), pack_map("y", d)))


def scatter(src: np.ndarray, new_idx: np.ndarray) -> np.ndarray:
    """``dest[new_idx[i]] = src[..., i]`` applied per rank (last axis)."""
    out = np.empty_like(src)
    out[..., new_idx] = src
    return out


# fast-axis changes: per-rank local transposes (a2achangefastaxis.cu:4-84)


def fast_z_to_x(b: np.ndarray, d: Decomp) -> np.ndarray:
    """brick ``[x][y][z]`` -> ``[z][y][x]`` (``a2achangefastaxis.cu:4-22``)."""
    lx, ly, lz = d.local
    return np.ascontiguousarray(b.reshape(-1, lx, ly, lz).transpose(0, 3, 2, 1)).reshape(b.shape)


def fast_x_to_y(b: np.ndarray, d: Decomp) -> np.ndarray:
    """``[z][y][x]`` -> ``[x][z][y]`` (``a2achangefastaxis.cu:35-53``)."""
    lx, ly, lz = d.local
    return np.ascontiguousarray(b.reshape(-1, lz, ly, lx).transpose(0, 3, 1, 2)).reshape(b.shape)


def fast_y_to_z(b: np.ndarray, d: Decomp) -> np.ndarray:
    """``[x][z][y]`` -> ``[x][y][z]`` (``a2achangefastaxis.cu:66-84``)."""
    lx, ly, lz = d.local
    return np.ascontiguousarray(b.reshape(-1, lx, lz, ly).transpose(0, 1, 3, 2)).reshape(b.shape)


# --------------------------------------------------------------------------
# The six distribution steps (a2adistribution.cpp:115-215), all ranks at once.
# Each takes and returns (buff1, buff2) with the contents the reference leaves.
# --------------------------------------------------------------------------


def get_z_pencils(b1, b2, d):
    b2 = alltoall(b1, d)
    b1 = scatter(b2, unpack_map("z", d))
    return b1, b2


def return_z_pencils(b1, b2, d):
    b2 = scatter(b1, pack_map("z", d))
    b1 = alltoall(b2, d)
    return b1, b2


def get_x_pencils(b1, b2, d):
    b2 = fast_z_to_x(b1, d)
    b1 = alltoall(b2, d)
    b2 = scatter(b1, unpack_map("x", d))
    return b1, b2


def return_x_pencils(b1, b2, d):
    b1 = scatter(b2, pack_map("x", d))
    b2 = alltoall(b1, d)
    return b1, b2


def get_y_pencils(b1, b2, d):
    b1 = fast_x_to_y(b2, d)
    b2 = alltoall(b1, d)
    b1 = scatter(b2, unpack_map("y", d))
    return b1, b2


def return_y_pencils(b1, b2, d):
    # the Y return packs from Buff2 (a2adistribution.cpp:203): a2adfft puts
    # the transformed pencils there with its parity copy or its scale kernel
    b1 = scatter(b2, pack_map("y", d))  # corrected inverse (see module doc)
    b2 = alltoall(b1, d)
    b1 = fast_y_to_z(b2, d)
    return b1, b2


# --------------------------------------------------------------------------
# 1D transforms (stand-in for the batched cuFFT calls) and the 3D pipeline
# --------------------------------------------------------------------------

_DFT_CACHE: dict = {}


def dft_matrix(n: int, inverse: bool) -> np.ndarray:
    """``F[j, k] = exp(-+ 2 pi i (jk mod n) / n)`` in complex128, generated in
    extended precision with the exponent reduced exactly."""
    key = (n, inverse)
    if key not in _DFT_CACHE:
        jk = np.outer(np.arange(n, dtype=np.int64), np.arange(n, dtype=np.int64)) % n
        ang = np.longdouble(2) * np.pi * jk.astype(np.longdouble) / np.longdouble(n)
        sign = 1.0 if inverse else -1.0
        f = np.cos(ang).astype(np.float64) + 1j * (sign * np.sin(ang)).astype(np.float64)
        _DFT_CACHE[key] = f
    return _DFT_CACHE[key]


def dft_lines(x: np.ndarray, n: int, inverse: bool = False) -> np.ndarray:
    """Unnormalised DFT of every contiguous length-n line of ``x`` (FP64)."""
    shp = x.shape
    v = x.reshape(-1, n).astype(np.complex128)
    return (v @ dft_matrix(n, inverse)).reshape(shp)


def fft_lines(x: np.ndarray, n: int, inverse: bool = False) -> np.ndarray:
    """Same as ``dft_lines`` through numpy's pocketfft (unnormalised)."""
    shp = x.shape
    v = x.reshape(-1, n).astype(np.complex128)
    out = np.fft.ifft(v, axis=1) * n if inverse else np.fft.fft(v, axis=1)
    return out.reshape(shp)


def scipy_lines(workers: int):
    """Batched 1D transforms through scipy's pocketfft with ``workers``
    threads, in the input's own precision (the CPU stand-in for the batched
    cuFFT calls when timing the reference pipeline on host cores)."""
    import scipy.fft as sfft

    def lines(x: np.ndarray, n: int, inverse: bool = False) -> np.ndarray:
        shp = x.shape
        v = x.reshape(-1, n)
        out = sfft.ifft(v, axis=1, norm="forward", workers=workers) if inverse else sfft.fft(
            v, axis=1, workers=workers)
        return out.reshape(shp)

    return lines


def forward(data: np.ndarray, d: Decomp, lines=dft_lines, dtype=np.complex128):
    """``a2adfft::forward`` (``a2adfft.cpp:26-91``) on ``(P, nlocal)`` bricks;
    returns the transformed bricks (``[x][y][z]``, natural order)."""
    if d.ng[0] != d.ng[1] or d.ng[1] != d.ng[2]:
        raise ValueError("the reference pipeline is defined for cubes")
    ng = d.ng[0]
    b1, b2 = np.array(data, dtype=dtype), np.zeros_like(data, dtype=dtype)
    b1, b2 = get_z_pencils(b1, b2, d)
    b1 = lines(b1, ng)
    b1, b2 = return_z_pencils(b1, b2, d)
    b1, b2 = get_x_pencils(b1, b2, d)
    b2 = lines(b2, ng)
    b1, b2 = return_x_pencils(b1, b2, d)
    b1, b2 = get_y_pencils(b1, b2, d)
    b1 = lines(b1, ng)
    b2 = b1.copy()  # launch_fast_copy_fft(d_scratch, d_data) (a2adfft.cpp:79)
    b1, b2 = return_y_pencils(b1, b2, d)
    return b1


def inverse(data: np.ndarray, d: Decomp, lines=dft_lines, dtype=np.complex128):
    """``a2adfft::inverse`` (``a2adfft.cpp:93-158``), including the final
    division by ``Ng^3`` (``a2affts.cu:78-92``)."""
    if d.ng[0] != d.ng[1] or d.ng[1] != d.ng[2]:
        raise ValueError("the reference pipeline is defined for cubes")
    ng = d.ng[0]
    inv = lambda x: lines(x, ng, True)  # noqa: E731
    b1, b2 = np.array(data, dtype=dtype), np.zeros_like(data, dtype=dtype)
    b1, b2 = get_z_pencils(b1, b2, d)
    b1 = inv(b1)
    b1, b2 = return_z_pencils(b1, b2, d)
    b1, b2 = get_x_pencils(b1, b2, d)
    b2 = inv(b2)
    b1, b2 = return_x_pencils(b1, b2, d)
    b1, b2 = get_y_pencils(b1, b2, d)
    b1 = inv(b1)
    b2 = (b1 / float(ng) ** 3).astype(b1.dtype)  # launch_scale_fft(d_scratch, d_data, ...) (a2adfft.cpp:147)
    b1, b2 = return_y_pencils(b1, b2, d)
    return b1


def fft3_global(g: np.ndarray, inverse: bool = False, lines=dft_lines) -> np.ndarray:
    """Separable 3D DFT of a global ``[x][y][z]`` array (any box shape),
    unnormalised forward, ``1/(nx ny nz)`` inverse -- the definition the
    pipeline must reproduce."""
    out = np.asarray(g, dtype=np.complex128)
    for ax in (2, 0, 1):
        n = out.shape[ax]
        moved = np.moveaxis(out, ax, -1)
        out = np.moveaxis(lines(np.ascontiguousarray(moved), n, inverse), -1, ax)
    if inverse:
        out = out / float(np.prod(g.shape))
    return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """``||a - b||_2 / ||b||_2`` in FP64."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = float(np.linalg.norm(b.ravel()))
    return float(np.linalg.norm((a - b).ravel())) / (den if den else 1.0)


def rel_l2_chunked(a: np.ndarray, b: np.ndarray, rows: int = 1 << 22) -> float:
    """``rel_l2`` over flat views in slices of ``rows`` elements, so that
    multi-GiB arrays need no full-size FP64 temporaries."""
    a, b = a.reshape(-1), b.reshape(-1)
    if a.size != b.size:
        raise ValueError("size mismatch")
    num = den = 0.0
    for i in range(0, a.size, rows):
        bb = b[i:i + rows].astype(np.complex128)
        dd = a[i:i + rows].astype(np.complex128) - bb
        num += float(np.vdot(dd, dd).real)
        den += float(np.vdot(bb, bb).real)
    return math.sqrt(num / den) if den else math.sqrt(num)


def fft3_fp64(g: np.ndarray, inverse: bool = False, workers: int | None = None) -> np.ndarray:
    """The reference's own acceptance transform, ``np.fft.fftn(inp)``
    (``src/a2afft/tests/stitch.py:89``), evaluated in complex128 for any box
    through scipy's pocketfft (the same FFT library numpy uses) on
    ``workers`` threads, in place on one complex128 copy of ``g``.  Forward
    unnormalised; the inverse scaled by ``1/(nx ny nz)``.  Used for the
    full-cube checks at sizes where the matrix DFT (``fft3_global``) is too
    slow; ``fft3_global`` and ``dft_points`` cross-check it."""
    import scipy.fft as sfft

    x = np.array(g, dtype=np.complex128)  # always a private copy
    workers = workers or (os.cpu_count() or 1)
    if inverse:
        return sfft.ifftn(x, workers=workers, overwrite_x=True)
    return sfft.fftn(x, workers=workers, overwrite_x=True)


def dft_points(g: np.ndarray, points, inverse: bool = False, slab: int = 32) -> np.ndarray:
    """Exact FP64 3D DFT at a few output points ``[(kx, ky, kz), ...]`` by
    direct summation (spot checks independent of any FFT), accumulated over
    slabs of ``slab`` x planes so that large cubes need no full-size FP64
    copy."""
    nx, ny, nz = g.shape
    sgn = 1.0 if inverse else -1.0
    ws = []
    for kx, ky, kz in points:
        ws.append((np.exp(sgn * 2j * np.pi * ((np.arange(nx) * kx) % nx) / nx),
                   np.exp(sgn * 2j * np.pi * ((np.arange(ny) * ky) % ny) / ny),
                   np.exp(sgn * 2j * np.pi * ((np.arange(nz) * kz) % nz) / nz)))
    out = np.zeros(len(ws), dtype=np.complex128)
    for x0 in range(0, nx, slab):
        blk = np.asarray(g[x0:x0 + slab], dtype=np.complex128)
        for i, (wx, wy, wz) in enumerate(ws):
            out[i] += wx[x0:x0 + slab] @ ((blk @ wz) @ wy)
    return out


# --------------------------------------------------------------------------
# Synthetic inputs (seeded) for the workloads the library is measured on
# --------------------------------------------------------------------------


def make_input(kind: str, shape, seed: int, dtype=np.complex64, tones: int = 0, amp: float = 100.0):
    """Seeded global ``[x][y][z]`` inputs.

    ``kind``: ``"uniform"`` (real and imaginary i.i.d. U[-1,1)),
    ``"normal"`` (i.i.d. N(0,1)), ``"ramp"`` (global-id tracer: the value of
    cell ``(x,y,z)`` is ``x*ny*nz + y*nz + z``, the idea of
    ``fft_demo/initializer/initializer.c:56-80``).  ``tones`` adds that many
    pure tones ``amp * exp(2 pi i k.r / N)`` at random wave vectors."""
    rng = np.random.default_rng(seed)
    shape = tuple(shape)
    rdt = np.float32 if dtype == np.complex64 else np.float64
    if kind == "uniform":
        re = rng.uniform(-1.0, 1.0, size=shape).astype(rdt)
        im = rng.uniform(-1.0, 1.0, size=shape).astype(rdt)
    elif kind == "normal":
        re = rng.standard_normal(size=shape, dtype=np.float64).astype(rdt)
        im = rng.standard_normal(size=shape, dtype=np.float64).astype(rdt)
    elif kind == "ramp":
        re = np.arange(math.prod(shape), dtype=np.float64).reshape(shape).astype(rdt)
        im = np.zeros(shape, dtype=rdt)
    else:
        raise ValueError(kind)
    out = np.empty(shape, dtype=dtype)
    out.real, out.imag = re, im
    if tones:
        nx, ny, nz = shape
        ks = np.stack([rng.integers(0, n, size=tones) for n in shape], axis=1)
        x = np.arange(nx)[:, None, None] / nx
        y = np.arange(ny)[None, :, None] / ny
        z = np.arange(nz)[None, None, :] / nz
        for kx, ky, kz in ks:
            ph = 2 * np.pi * (kx * x + ky * y + kz * z)
            out += (amp * np.exp(1j * ph)).astype(dtype)
    return out


# --------------------------------------------------------------------------
# The reference's host step sequence on all host cores (timed CPU baseline)
# --------------------------------------------------------------------------


class HostPipeline:
    """``a2adfft::forward`` / ``inverse`` (``dfft/a2adfft.cpp:26-158``) over
    all P virtual ranks on the host cores, step for step and pass for pass as
    the reference runs it: every alltoall, pack/unpack remap, fast-axis
    change, batched 1D transform, parity copy and scale is its own pass over
    the rank-major buffer (19 per direction).  Each remap is the permutation
    ``unpack_map`` / ``pack_map`` / ``fast_*`` define, written here as the
    strided copy it is (the sender group and the chunk line are separate
    tensor axes), so torch's CPU copy kernels run it on every thread; the 1D
    transforms are torch.fft on the host (pocketfft), in the buffer's own
    precision, standing in for the reference's batched cuFFT calls.  This is
    the reference arm and CPU baseline of the benchmark, not a checker: it is
    itself pinned against the step functions above (tests/test_oracle.py).
    The Y return uses the true inverse of the Y unpack (see
    ``y_pencils_to_y_a2a_ref_map``)."""

    def __init__(self, d: Decomp, dtype: str = "c64", threads: int | None = None):
        import torch

        if d.ng[0] != d.ng[1] or d.ng[1] != d.ng[2]:
            raise ValueError("the reference pipeline is defined for cubes")
        self.t = torch
        self.d = d
        self.threads = threads or (os.cpu_count() or 1)
        torch.set_num_threads(self.threads)
        self.cdt = torch.complex128 if dtype == "c128" else torch.complex64
        n = d.world_size * d.nlocal
        self.b1 = torch.empty(n, dtype=self.cdt)
        self.b2 = torch.empty(n, dtype=self.cdt)
        self.tmp = torch.empty(n, dtype=self.cdt)  # out-of-place FFT target, swapped in

    # -- passes ---------------------------------------------------------------
    def _alltoall(self, src, dst):
        P, c = self.d.world_size, self.d.chunk
        dst.view(P, P, c).copy_(src.view(P, P, c).transpose(0, 1))

    def _split(self, axis):
        d0, d1, d2 = self.d.dims
        la = self.d.local[_AXIS[axis]]
        return d0, d1, d2, self.d.chunk // la, la

    def _unpack(self, axis, src, dst):
        P = self.d.world_size
        d0, d1, d2, m, la = self._split(axis)
        s = src.view(P, d0, d1, d2, m, la)  # [q][c0][c1][c2][j][e]
        if axis == "z":  # pencil (c0, c1, j, c2, e)
            dst.view(P, d0, d1, m, d2, la).copy_(s.permute(0, 1, 2, 4, 3, 5))
        elif axis == "x":  # pencil (c1, c2, j, c0, e)
            dst.view(P, d1, d2, m, d0, la).copy_(s.permute(0, 2, 3, 4, 1, 5))
        else:  # pencil (c0, c2, j, c1, e)
            dst.view(P, d0, d2, m, d1, la).copy_(s.permute(0, 1, 3, 4, 2, 5))

    def _pack(self, axis, src, dst):
        P = self.d.world_size
        d0, d1, d2, m, la = self._split(axis)
        o = dst.view(P, d0, d1, d2, m, la)
        if axis == "z":
            o.copy_(src.view(P, d0, d1, m, d2, la).permute(0, 1, 2, 4, 3, 5))
        elif axis == "x":
            o.copy_(src.view(P, d1, d2, m, d0, la).permute(0, 4, 1, 2, 3, 5))
        else:
            o.copy_(src.view(P, d0, d2, m, d1, la).permute(0, 1, 4, 2, 3, 5))

    def _fast(self, which, src, dst):
        P = self.d.world_size
        lx, ly, lz = self.d.local
        if which == "z_to_x":  # [x][y][z] -> [z][y][x]
            dst.view(P, lz, ly, lx).copy_(src.view(P, lx, ly, lz).permute(0, 3, 2, 1))
        elif which == "x_to_y":  # [z][y][x] -> [x][z][y]
            dst.view(P, lx, lz, ly).copy_(src.view(P, lz, ly, lx).permute(0, 3, 1, 2))
        else:  # [x][z][y] -> [x][y][z]
            dst.view(P, lx, ly, lz).copy_(src.view(P, lx, lz, ly).permute(0, 1, 3, 2))

    def _lines(self, name, inverse):
        """In-place (by buffer swap) unnormalised 1D transforms of every
        length-Ng line of buffer ``name``."""
        t, ng = self.t, self.d.ng[0]
        src = getattr(self, name)
        if inverse:
            t.fft.ifft(src.view(-1, ng), dim=1, norm="forward", out=self.tmp.view(-1, ng))
        else:
            t.fft.fft(src.view(-1, ng), dim=1, out=self.tmp.view(-1, ng))
        setattr(self, name, self.tmp)
        self.tmp = src

    # -- the six steps (a2adistribution.cpp:115-215) ---------------------------
    def get_z_pencils(self):
        self._alltoall(self.b1, self.b2)
        self._unpack("z", self.b2, self.b1)

    def return_z_pencils(self):
        self._pack("z", self.b1, self.b2)
        self._alltoall(self.b2, self.b1)

    def get_x_pencils(self):
        self._fast("z_to_x", self.b1, self.b2)
        self._alltoall(self.b2, self.b1)
        self._unpack("x", self.b1, self.b2)

    def return_x_pencils(self):
        self._pack("x", self.b2, self.b1)
        self._alltoall(self.b1, self.b2)

    def get_y_pencils(self):
        self._fast("x_to_y", self.b2, self.b1)
        self._alltoall(self.b1, self.b2)
        self._unpack("y", self.b2, self.b1)

    def return_y_pencils(self):
        self._pack("y", self.b2, self.b1)
        self._alltoall(self.b1, self.b2)
        self._fast("y_to_z", self.b2, self.b1)

    # -- a2adfft::forward / inverse --------------------------------------------
    def run(self, inverse: bool = False):
        """One transform of ``self.b1`` in place (``b2`` is the scratch)."""
        ng = self.d.ng[0]
        self.get_z_pencils()
        self._lines("b1", inverse)
        self.return_z_pencils()
        self.get_x_pencils()
        self._lines("b2", inverse)
        self.return_x_pencils()
        self.get_y_pencils()
        self._lines("b1", inverse)
        if inverse:  # launch_scale_fft(d_scratch, d_data) (a2adfft.cpp:147)
            self.t.div(self.b1, float(ng) ** 3, out=self.b2)
        else:  # launch_fast_copy_fft(d_scratch, d_data) (a2adfft.cpp:79)
            self.b2.copy_(self.b1)
        self.return_y_pencils()
