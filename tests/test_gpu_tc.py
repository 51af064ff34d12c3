"""Split-precision tensor-core form (tcgen05, kind::f16, FP32 accumulate):
every radix-16 stage of the pass kernels runs as a GEMM with split 16-bit
operands.  Accuracy is stated against the FP64 oracle, and both forms are held
to the 1e-6 relative-L2 bar: split fp16 with two parts (hi + lo, 22
significant bits), split bf16 with three (hi + mid + lo, 24 bits; two bf16
parts carry only 16 bits).  The full-size 512^3 and 1024^3 checks are in
test_gpu_configs.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"split_fp16": 1e-6, "split_bf16": 1e-6}


def run(pkg, O, cuda, P, shape, method, kind="uniform", tones=0, seed=0):
    import torch

    shape = (shape,) * 3 if isinstance(shape, int) else tuple(shape)
    dist = pkg.a2aDistribution(P, shape, 64, precision="c64")
    d = O.Decomp(shape, P)
    g = O.make_input(kind, shape, seed=seed, dtype=np.complex64, tones=tones)
    x = torch.from_numpy(O.global_to_bricks(g, d).ravel()).to(cuda)
    f = pkg.a2adfft(dist, method=method)
    f.make_plans()
    f.forward(x)
    fwd = O.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    f.inverse(x)
    inv = O.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    return g, fwd, inv, f


@pytest.mark.parametrize("method", ["split_fp16", "split_bf16"])
@pytest.mark.parametrize("P,shape", [(4, 64), (16, 128), (16, 256), (4, (64, 128, 256)), (4, (64, 1024, 64)),
                                     (4, (1024, 64, 64)), (4, (64, 64, 1024))])
def test_split_vs_fp64_oracle(pkg, oracle, cuda, P, shape, method):
    g, fwd, inv, f = run(pkg, oracle, cuda, P, shape, method)
    ref = oracle.fft3_global(g, lines=oracle.dft_lines if g.size <= 2 ** 22 else oracle.fft_lines)
    ef, ei = oracle.rel_l2(fwd, ref), oracle.rel_l2(inv, g)
    assert ef <= TOL[method], f"forward rel L2 {ef:.3e}"
    assert ei <= 2 * TOL[method], f"round trip rel L2 {ei:.3e}"
    assert "tensor-core" in f.plan_report()


@pytest.mark.parametrize("method", ["split_fp16", "split_bf16"])
def test_split_with_tones(pkg, oracle, cuda, method):
    """U[-1,1) plus three pure tones of amplitude 100: rows span a wide range
    of magnitudes, which the per-row power-of-two scaling must absorb."""
    g, fwd, inv, _ = run(pkg, oracle, cuda, 16, 128, method, tones=3, seed=2)
    ref = oracle.fft3_global(g)
    assert oracle.rel_l2(fwd, ref) <= TOL[method]
    assert oracle.rel_l2(inv, g) <= 2 * TOL[method]


@pytest.mark.parametrize("method", ["split_fp16", "split_bf16"])
@pytest.mark.parametrize("P,shape", [(4, 64), (16, 128), (16, (512, 64, 64)), (4, (64, 64, 512)),
                                     (4, (64, 512, 64)), (4, (64, 1024, 64)), (4, (64, 64, 1024))])
def test_split_every_kernel_form(pkg, oracle, cuda, P, shape, method):
    """Each tensor-core kernel form -- one tile per CTA, the persistent form
    fed by the TMA ring, and the two-stage form (512 = 16 x 32 and 1024 =
    32 x 32: a radix-16 or radix-32 GEMM, one twiddle, a radix-32 GEMM, TMA
    ring; at 1024 with 4- or 8-line tiles; in fp16 also software-pipelined
    over two tensor-memory regions) -- on every pass gives the FP64 oracle's
    transform (relative L2 <= 1e-6)."""
    import torch

    shape = (shape,) * 3 if isinstance(shape, int) else tuple(shape)
    dist = pkg.a2aDistribution(P, shape, 64, precision="c64")
    d = oracle.Decomp(shape, P)
    g = oracle.make_input("uniform", shape, seed=21, dtype=np.complex64, tones=2)
    x0 = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
    ref = oracle.fft3_fp64(g)
    f = pkg.a2adfft(dist, method=method)
    f.make_plans()
    assert f.variant_count(0) == 5
    tested = 0
    applied = [set(), set(), set(), set(), set()]
    for form in (0, 1, 2, 3, 4):
        for p in range(3):
            try:
                f.select_variant(p, form)
                applied[form].add(p)
            except pkg.A2AError:
                assert form >= 1  # the ring and two-stage forms do not fit every pass
                f.select_variant(p, 0)
        x = x0.clone()
        f.forward(x)
        fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
        assert oracle.rel_l2(fwd, ref) <= TOL[method], f"form {form}"
        f.inverse(x)
        assert oracle.rel_l2(x.cpu().numpy(), x0.cpu().numpy()) <= 2 * TOL[method], f"form {form} round trip"
        tested += 1
    assert tested == 5
    assert applied[0] == {0, 1, 2}
    # the two-stage form (512 and 1024) runs on the ring form's tile geometry:
    # it fits exactly the passes of those lengths where the ring form fits
    lengths = (shape[2], shape[0], shape[1])  # Z, X, Y
    assert applied[2] == {p for p in applied[1] if lengths[p] in (512, 1024)}, applied
    assert applied[3] <= {p for p in range(3) if lengths[p] == 1024}, applied  # 8-line tiles of 1024
    # the software-pipelined two-stage form: fp16, on the two-stage form's passes
    assert applied[4] == (applied[2] if method == "split_fp16" else set()), applied


def test_split_rejects_double_and_unsupported_lengths(pkg, cuda):
    with pytest.raises(pkg.A2AError) as e:
        pkg.a2adfft(pkg.a2aDistribution(4, 64, 64, precision="c128"), method="split_fp16")
    assert e.value.status == 9
    with pytest.raises(pkg.A2AError) as e:
        pkg.a2adfft(pkg.a2aDistribution(4, 48, 64, precision="c64"), method="split_fp16")
    assert e.value.status == 9
