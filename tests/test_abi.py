"""CPU checks of the C ABI (no GPU): the library loads, exports every entry
point include/a2afft_b200.h declares, and its host-side validation (the
reference's decomposition asserts, argument checks) returns the documented
status codes before any device work."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "a2afft_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:a2a_status|const char\*|int)\s+(a2a_\w+)\s*\(", txt, re.M)))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for n in ["a2a_distribution_create", "a2a_get_z_pencils", "a2a_return_z_pencils", "a2a_get_x_pencils",
              "a2a_return_x_pencils", "a2a_get_y_pencils", "a2a_return_y_pencils", "a2a_distribution_finalize",
              "a2a_forward_1d_fft", "a2a_inverse_1d_fft", "a2a_scale_fft", "a2a_fast_copy_fft", "a2a_dfft_create",
              "a2a_dfft_make_plans", "a2a_dfft_forward", "a2a_dfft_inverse", "a2a_dfft_destroy"]:
        assert n in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.lib()
    raw = ctypes.CDLL(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    from importlib import import_module

    sigs = import_module(pkg.__name__ + "._lib").SIGNATURES
    assert sorted(sigs) == declared_functions()
    assert lib.a2a_version() == 100


def test_status_strings(pkg):
    lib = pkg.lib()
    for code in range(10):
        assert lib.a2a_status_string(code) not in (None, b"", b"unknown status")
    assert lib.a2a_status_string(99) == b"unknown status"


@pytest.mark.parametrize("ng,P", [(8, 6), (10, 4), (64, 256), (12, 8)])
def test_decomposition_errors_without_gpu(pkg, ng, P):
    """Grids the reference rejects with assert (a2adistribution.cpp:61-80)
    return A2A_ERROR_DECOMPOSITION."""
    with pytest.raises(pkg.A2AError) as e:
        pkg.a2aDistribution(P, ng, 64, precision="c64")
    assert e.value.status == 2
    assert "divisible" in e.value.detail


def test_invalid_arguments_without_gpu(pkg):
    lib = pkg.lib()
    h = ctypes.c_void_p()
    assert lib.a2a_distribution_create(0, 4, 64, 0, ctypes.byref(h)) == 1
    assert lib.a2a_distribution_create(8, 0, 64, 0, ctypes.byref(h)) == 1
    assert lib.a2a_distribution_create(8, 4, 0, 0, ctypes.byref(h)) == 1
    assert lib.a2a_distribution_create(8, 4, 2048, 0, ctypes.byref(h)) == 1
    assert lib.a2a_distribution_create(8, 4, 64, 7, ctypes.byref(h)) == 1
    assert lib.a2a_distribution_create(8, 4, 64, 0, None) == 1
    assert b"block_size" in lib.a2a_last_error() or len(lib.a2a_last_error()) > 0
    assert lib.a2a_dfft_forward(None, None) == 1
    assert lib.a2a_dfft_make_plans(None, None) == 1
    assert lib.a2a_distribution_finalize(None) == 0
    assert lib.a2a_dfft_destroy(None) == 0
    # batched form: shape validation happens before any device work
    shapes = (ctypes.c_int * 6)(32, 32, 32, 64, 40, 64)
    assert lib.a2a_batch_create(2, shapes, 4, 1, ctypes.byref(h)) == 3  # edge 40: no batched tile
    assert b"edge 40" in lib.a2a_last_error()
    assert lib.a2a_batch_create(0, shapes, 4, 1, ctypes.byref(h)) == 1
    assert lib.a2a_batch_create(1, None, 4, 1, ctypes.byref(h)) == 1
    assert lib.a2a_batch_create(1, shapes, 4, 5, ctypes.byref(h)) == 1
    assert lib.a2a_batch_create(1, shapes, 3, 1, ctypes.byref(h)) == 2  # 32 over dims [3,1,1]
    assert b"box 0" in lib.a2a_last_error()
    assert lib.a2a_batch_forward(None, None) == 1
    assert lib.a2a_batch_destroy(None) == 0


def test_python_mirror_rejects_bad_precision(pkg):
    with pytest.raises(ValueError):
        pkg.a2aDistribution(4, 8, 64, precision="bf16")


def test_dims_and_rank_dumps_roundtrip_on_cpu(pkg, oracle, tmp_path):
    """The reference's dims / proc<r> files written by the C ABI read back
    with the reference checker's semantics (no GPU: host-only calls)."""
    import importlib

    import numpy as np

    dumps = importlib.import_module(pkg.__name__ + ".dumps")
    for P, ng in [(8, 8), (6, 12), (16, 32)]:
        d = oracle.Decomp(ng, P)
        pkg.write_dims(ng, P, str(tmp_path / "dims"))
        prm = dumps.read_dims(str(tmp_path / "dims"))
        assert prm == {"world_size": P, "Ng": ng, "nlocal": d.nlocal, "dims": d.dims, "local_grid_size": list(d.local)}
        g = oracle.make_input("uniform", (ng,) * 3, seed=1, dtype=np.complex128)
        b = oracle.global_to_bricks(g, d)
        fwd = oracle.global_to_bricks(np.fft.fftn(g), d)
        pkg.write_rank_dumps(ng, P, str(tmp_path), b, fwd, b)
        assert dumps.check(str(tmp_path)) == (True, True)
        raw = dumps.read_rank_dumps(str(tmp_path), prm)
        assert np.array_equal(dumps.stitch(raw[:, 0], prm), g)
    with pytest.raises(pkg.A2AError):
        pkg.write_dims(10, 4, str(tmp_path / "bad"))
