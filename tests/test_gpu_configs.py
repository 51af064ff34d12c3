"""The measured configurations at their full sizes, whole cube against the
FP64 oracle.

The reference's own acceptance check compares the whole stitched cube with
``np.fft.fftn(inp)`` (``src/a2afft/tests/stitch.py:89``).  Here every
configuration the benchmark is quoted on runs through the C ABI on the same
seeded input the benchmark generates (``bench.synth_bricks``, on the GPU),
the input is copied to the host, and the oracle transforms the whole cube in
complex128 (``fft3_fp64``: scipy's pocketfft, the library numpy.fft uses).
Bars (stated per test): relative L2 error <= 1e-6 for complex64 and for both
split-precision tensor-core forms, <= 1e-12 for complex128, and for
complex128 also the reference's elementwise ``allclose``.

* 64^3 complex128, 4 ranks ([2,2,1]), U[-1,1) seed 0
* 256^3 complex64, 16 ranks ([4,2,2]), N(0,1) seed 1
* 512^3 complex64, 64 ranks ([4,4,4]), U[-1,1) + 3 tones x100 seed 2:
  plain, split fp16, split bf16
* 1024^3 complex64, 256 ranks ([8,8,4]), U[-1,1) seed 4: plain, split fp16,
  split bf16
* 768^3 complex128, 64 ranks ([4,4,4]), U[-1,1) seed 4
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-6, "c128": 1e-12}


def gpu_input(torch, cuda, ng, dims, prec, kind, seed, tones):
    real = torch.float64 if prec == "c128" else torch.float32
    return bench.synth_bricks(torch, ng, dims, seed, cuda, real, tones, kind)


def gpu_rel_l2(torch, a, b, chunk=1 << 26):
    """||a - b|| / ||b|| over two device tensors, accumulated in FP64."""
    num = den = 0.0
    for i in range(0, b.numel(), chunk):
        bb = b[i:i + chunk].to(torch.complex128)
        num += float(torch.linalg.vector_norm(a[i:i + chunk].to(torch.complex128) - bb) ** 2)
        den += float(torch.linalg.vector_norm(bb) ** 2)
    return (num / den) ** 0.5


def allclose_chunked(a, b, rows=1 << 22):
    """``np.allclose(b, a)`` with numpy's default rtol/atol (the reference's
    check, ``stitch.py:89``) over flat slices."""
    a, b = a.reshape(-1), b.reshape(-1)
    for i in range(0, a.size, rows):
        if not np.allclose(b[i:i + rows], a[i:i + rows]):
            return False
    return True


def run_config(pkg, O, cuda, ng, P, prec, kind, seed, tones, methods):
    """Forward with each method vs the FP64 oracle (whole cube), then the
    round trip; returns {method: (forward error, round-trip error, allclose)}."""
    import torch

    dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
    d = O.Decomp(ng, P)
    assert dist.dims == d.dims and dist.nlocal == d.nlocal
    x0 = gpu_input(torch, cuda, ng, dist.dims, prec, kind, seed, tones)
    g = O.bricks_to_global(x0.cpu().numpy().reshape(P, -1), d)
    ref = O.fft3_fp64(g)  # complex128, whole cube
    del g
    out = {}
    for m in methods:
        f = pkg.a2adfft(dist, method=m)
        f.make_plans()
        x = x0.clone()
        f.forward(x)
        fwd = O.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
        ef = O.rel_l2_chunked(fwd, ref)
        close = allclose_chunked(fwd, ref) if prec == "c128" else None
        del fwd
        f.inverse(x)
        ei = gpu_rel_l2(torch, x, x0)
        out[m] = (ef, ei, close)
        del x, f
        torch.cuda.empty_cache()
    return out


def test_config1_64_c128(pkg, oracle, cuda):
    r = run_config(pkg, oracle, cuda, 64, 4, "c128", "uniform", 0, 0, ["plain"])
    ef, ei, close = r["plain"]
    assert ef <= TOL["c128"], f"forward rel L2 {ef:.3e}"
    assert ei <= TOL["c128"], f"round trip rel L2 {ei:.3e}"
    assert close


def test_config2_256_c64(pkg, oracle, cuda):
    r = run_config(pkg, oracle, cuda, 256, 16, "c64", "normal", 1, 0, ["plain"])
    ef, ei, _ = r["plain"]
    assert ef <= TOL["c64"], f"forward rel L2 {ef:.3e}"
    assert ei <= TOL["c64"], f"round trip rel L2 {ei:.3e}"


@pytest.mark.parametrize("method", ["plain", "split_fp16", "split_bf16"])
def test_config3_512_c64(pkg, oracle, cuda, method):
    """The headline workload: plain FP32 and both split-precision forms on
    the benchmark's own input, each held to 1e-6 against FP64."""
    r = run_config(pkg, oracle, cuda, 512, 64, "c64", "uniform", 2, 3, [method])
    ef, ei, _ = r[method]
    print(f"512^3 {method}: forward rel L2 {ef:.3e}, round trip {ei:.3e}")
    assert ef <= TOL["c64"], f"{method} forward rel L2 {ef:.3e}"
    assert ei <= 2 * TOL["c64"], f"{method} round trip rel L2 {ei:.3e}"


@pytest.mark.parametrize("method", ["plain", "split_fp16", "split_bf16"])
def test_config5_1024_c64(pkg, oracle, cuda, method):
    """1024^3 complex64 (8 GiB) on 256 virtual ranks, dims [8,8,4]."""
    r = run_config(pkg, oracle, cuda, 1024, 256, "c64", "uniform", 4, 0, [method])
    ef, ei, _ = r[method]
    print(f"1024^3 {method}: forward rel L2 {ef:.3e}, round trip {ei:.3e}")
    assert ef <= TOL["c64"], f"{method} forward rel L2 {ef:.3e}"
    assert ei <= 2 * TOL["c64"], f"{method} round trip rel L2 {ei:.3e}"


def test_config5_768_c128(pkg, oracle, cuda):
    """768^3 complex128 (6.75 GiB), radix 3 x 16 x 16, on 64 virtual ranks."""
    r = run_config(pkg, oracle, cuda, 768, 64, "c128", "uniform", 4, 0, ["plain"])
    ef, ei, close = r["plain"]
    print(f"768^3 c128: forward rel L2 {ef:.3e}, round trip {ei:.3e}")
    assert ef <= TOL["c128"], f"forward rel L2 {ef:.3e}"
    assert ei <= TOL["c128"], f"round trip rel L2 {ei:.3e}"
    assert close
