"""Regenerates the committed golden fixtures in this directory.

Runs the reference's own CPU remap code -- the pencils_demo copies of its
pack/unpack and fast-axis kernels, compiled unmodified into
``oracle/_ref/libpencils_ref.so`` by ``oracle/Makefile`` from the reference
tree -- on int32 iota inputs, and records exactly what each call leaves in its
destination buffer (including, for the reference's Y pack on grids where it is
not a permutation, the cells it never writes and the ones it writes twice).
Also records the reference's own test input (``src/a2afft/tests/test.cpp``:
``populate_grid`` fills every rank's brick with ``rand()/RAND_MAX`` real parts
and zero imaginary parts from the unseeded C library generator) for its four
test grids (``src/a2afft/tests/run_tests.py:18-21``), with the result its
checker expects (``np.fft.fftn`` of the stitched cube, ``tests/stitch.py:89``).

Needs the reference tree (``make -C oracle``) and glibc; run from the repo
root:  ``python tests/golden/make_golden.py``.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import a2a_oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libpencils_ref.so")

# (world_size, Ng): the reference's four test grids, then grids that exercise
# every brick-grid shape the measured workloads use (small Ng), including
# grids where the reference's Y pack is not a permutation.
GRIDS = [(8, 8), (8, 32), (6, 12), (4, 4), (4, 16), (16, 32), (64, 32), (2, 16), (3, 12), (12, 24), (32, 32),
         (1, 8), (256, 128)]
REF_TEST_GRIDS = [(8, 8), (8, 32), (6, 12), (4, 4)]
GUARD = 64  # cells past the buffer end, to record out-of-range writes


def ref_remap(lib, name, d):
    IP = ctypes.POINTER(ctypes.c_int)
    n = d.nlocal
    src = np.arange(n, dtype=np.int32)
    loc = (ctypes.c_int * 3)(*d.local)
    dims = (ctypes.c_int * 3)(*d.dims)
    if name.startswith("fast"):
        dst = np.full(n, -1, dtype=np.int32)
        getattr(lib, name)(src.ctypes.data_as(IP), dst.ctypes.data_as(IP), loc)
        return dst
    if name == "y_pencils_to_y_a2a":
        extra = max(GUARD, int(O.y_pencils_to_y_a2a_ref_map(d).max()) + 1 - n + GUARD)
    else:
        extra = GUARD
    dst = np.full(n + extra, -1, dtype=np.int32)
    getattr(lib, name)(src.ctypes.data_as(IP), dst.ctypes.data_as(IP), d.world_size, 0, n, loc, dims)
    return dst


def main():
    lib = ctypes.CDLL(REF_LIB)
    out = {}
    for P, ng in GRIDS:
        d = O.Decomp(ng, P)
        key = f"P{P}_N{ng}"
        for ax in "zxy":
            out[f"{key}_{ax}_a2a_to_{ax}_pencils"] = ref_remap(lib, f"{ax}_a2a_to_{ax}_pencils", d)
            out[f"{key}_{ax}_pencils_to_{ax}_a2a"] = ref_remap(lib, f"{ax}_pencils_to_{ax}_a2a", d)
        for nm in ("fast_z_to_x", "fast_x_to_y", "fast_y_to_z"):
            out[f"{key}_{nm}"] = ref_remap(lib, nm, d)
    np.savez_compressed(os.path.join(HERE, "remaps.npz"), **out)

    libc = ctypes.CDLL(None)
    libc.rand.restype = ctypes.c_int
    RAND_MAX = 2147483647  # glibc
    fft = {}
    for P, ng in REF_TEST_GRIDS:
        d = O.Decomp(ng, P)
        libc.srand(1)  # the unseeded generator starts from seed 1
        vals = np.array([libc.rand() for _ in range(d.nlocal)], dtype=np.float64) / RAND_MAX
        brick = vals.astype(np.complex128)  # every rank generates the same sequence
        bricks = np.tile(brick, (P, 1))
        g = O.bricks_to_global(bricks, d)
        fft[f"P{P}_N{ng}_input"] = bricks
        fft[f"P{P}_N{ng}_forward"] = O.global_to_bricks(np.fft.fftn(g), d)
    np.savez_compressed(os.path.join(HERE, "reference_tests.npz"), **fft)
    print("wrote", len(out), "remap fixtures and", len(fft), "transform fixtures")


if __name__ == "__main__":
    main()
