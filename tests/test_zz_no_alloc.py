"""The allocation-free 1D line transform (``a2a_lines_fft_noalloc``) through
the C ABI, against the existing entry points ``a2a_forward_1d_fft`` /
``a2a_inverse_1d_fft`` on the same data.  Two calls in a row with different
lengths and precisions, so the second call rebuilds the tables the first one
left in the shared fixed-size device array.  Tolerance as for every transform
test here: relative L2 <= 1e-6 (complex64), <= 1e-12 (complex128).  The file
name makes pytest collect it last; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-6, "c128": 1e-12}
PREC = {"c64": 1, "c128": 0}


def _rel(a, b):
    a = a.cpu().numpy().astype(np.complex128)
    b = b.cpu().numpy().astype(np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("calls", [[(64, 4, "c64", False), (48, 4, "c128", True)],
                                   [(512, 4, "c64", True), (12, 2, "c64", False)]])
def test_noalloc_lines_match_existing_entry_point(pkg, cuda, calls):
    import torch

    raw = ctypes.CDLL(pkg.LIB_PATH)
    raw.a2a_lines_fft_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p]
    raw.a2a_lines_fft_noalloc.restype = ctypes.c_int
    raw.a2a_last_error.restype = ctypes.c_char_p
    gen = torch.Generator(device=cuda)
    gen.manual_seed(1)
    for ng, P, prec, inverse in calls:
        dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
        real = torch.float64 if prec == "c128" else torch.float32
        n_el = dist.nlocal * P
        x = torch.complex(torch.randn(n_el, generator=gen, device=cuda, dtype=real),
                          torch.randn(n_el, generator=gen, device=cuda, dtype=real))
        ref = x.clone()
        (pkg.inverse_1d_fft if inverse else pkg.forward_1d_fft)(dist, ref)
        nlines = n_el // ng
        st = torch.cuda.current_stream()
        rc = raw.a2a_lines_fft_noalloc(ctypes.c_void_p(x.data_ptr()), ng, nlines, PREC[prec], int(inverse),
                                       ctypes.c_void_p(st.cuda_stream))
        assert rc == 0, raw.a2a_last_error()
        torch.cuda.synchronize()
        e = _rel(x, ref)
        assert e <= TOL[prec], f"Ng={ng} {prec} inverse={inverse}: rel L2 vs existing entry point {e:.3e}"
        dist.finalize()


def test_noalloc_rejects_sizes_beyond_its_array(pkg, cuda):
    import torch

    raw = ctypes.CDLL(pkg.LIB_PATH)
    raw.a2a_lines_fft_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p]
    raw.a2a_lines_fft_noalloc.restype = ctypes.c_int
    raw.a2a_last_error.restype = ctypes.c_char_p
    x = torch.zeros(1024, dtype=torch.complex64, device=cuda)
    # 4 * 2^17 + 4 lines of length 4: the line tables need more than the fixed array
    assert raw.a2a_lines_fft_noalloc(ctypes.c_void_p(x.data_ptr()), 4, 4 * (1 << 17) + 4, 1, 0, None) == 3
    assert b"scratch" in raw.a2a_last_error()
    assert raw.a2a_lines_fft_noalloc(ctypes.c_void_p(x.data_ptr()), 40, 4, 1, 0, None) == 3
    assert raw.a2a_lines_fft_noalloc(ctypes.c_void_p(x.data_ptr()), 8, 6, 1, 0, None) == 3  # 6 lines: no tile
    assert raw.a2a_lines_fft_noalloc(None, 8, 4, 1, 0, None) == 1
