"""The six a2aDistribution steps, the 1D calls and the step-by-step
reference sequence through the C ABI, against the oracle.

Permutations are checked bit-exactly per virtual rank: the input is a
global-id tracer (every element of both buffers holds a distinct pair of
exactly representable values derived from its index), so any misplaced element
changes a value.  Both buffers are compared after every step, as the reference leaves
data in both (``src/a2afft/distribution/a2adistribution.cpp:115-215``)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the reference's four test grids, then others; (16, 256) is the 256^3 workload's
# grid at full size, (64, 128) / (256, 128) / (256, 256) the [4,4,4] and
# [8,8,4] grids of the 512^3 and 1024^3 workloads, where the reference's Y
# pack is not a permutation
GRIDS = [(8, 8), (8, 32), (6, 12), (4, 4), (4, 64), (16, 32), (64, 32), (2, 16), (1, 8), (3, 12), (12, 24),
         (32, 32), (24, 48), (16, 64), (16, 256), (64, 128), (256, 128), (256, 256)]

STEPS = ["getZPencils", "returnZPencils", "getXPencils", "returnXPencils", "getYPencils", "returnYPencils"]
ORACLE_STEPS = ["get_z_pencils", "return_z_pencils", "get_x_pencils", "return_x_pencils", "get_y_pencils",
                "return_y_pencils"]


def tracer(O, d, prec, salt):
    """Distinct exact values: element i of the buffer with salt s (0 or 1)
    holds v = 2 i + s split as (v // 4096, -(v % 4096)), exact in float32 for
    every grid here."""
    n = d.world_size * d.nlocal
    v = 2 * np.arange(n, dtype=np.int64) + int(salt)
    out = np.empty(n, dtype=np.complex128 if prec == "c128" else np.complex64)
    out.real = v // 4096
    out.imag = -(v % 4096)
    return out.reshape(d.world_size, d.nlocal)


@pytest.mark.parametrize("prec", ["c64", "c128"])
@pytest.mark.parametrize("P,ng", GRIDS)
def test_steps_bit_exact(pkg, oracle, cuda, P, ng, prec):
    import torch

    dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
    d = oracle.Decomp(ng, P)
    b1 = tracer(oracle, d, prec, 0)
    b2 = tracer(oracle, d, prec, 1)
    t1 = torch.from_numpy(b1.ravel().copy()).to(cuda)
    t2 = torch.from_numpy(b2.ravel().copy()).to(cuda)
    for name, oname in zip(STEPS, ORACLE_STEPS):
        if name == "returnYPencils":
            # the Y return packs from Buff2: a2adfft fills it with its parity
            # copy first (dfft/a2adfft.cpp:79)
            pkg.fast_copy_fft(dist, t2, t1)
            b2 = b1.copy()
        getattr(dist, name)(t1, t2)
        b1, b2 = getattr(oracle, oname)(b1, b2, d)
        g1 = t1.cpu().numpy().reshape(P, -1)
        g2 = t2.cpu().numpy().reshape(P, -1)
        assert np.array_equal(g1, b1.astype(g1.dtype)), f"{name}: buff1 differs"
        assert np.array_equal(g2, b2.astype(g2.dtype)), f"{name}: buff2 differs"
    # the six steps compose to the identity on the data buffer
    assert np.array_equal(t1.cpu().numpy().reshape(P, -1), tracer(oracle, d, prec, 0))


@pytest.mark.parametrize("prec", ["c64", "c128"])
@pytest.mark.parametrize("P,ng", [(8, 8), (6, 12), (4, 64), (64, 32), (16, 32)])
def test_reference_sequence_matches_fused(pkg, oracle, cuda, P, ng, prec):
    """``a2adfft::forward``/``inverse`` spelled out step by step
    (``dfft/a2adfft.cpp:26-158``) through the distribution API and the 1D
    calls gives the fused transform's result."""
    import torch

    dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
    d = oracle.Decomp(ng, P)
    cdt = np.complex64 if prec == "c64" else np.complex128
    g = oracle.make_input("uniform", (ng,) * 3, seed=0, dtype=cdt)
    data = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
    scratch = torch.zeros_like(data)
    fused = data.clone()
    dist.getZPencils(data, scratch)
    pkg.forward_1d_fft(dist, data)
    dist.returnZPencils(data, scratch)
    dist.getXPencils(data, scratch)
    pkg.forward_1d_fft(dist, scratch)
    dist.returnXPencils(data, scratch)
    dist.getYPencils(data, scratch)
    pkg.forward_1d_fft(dist, data)
    pkg.fast_copy_fft(dist, scratch, data)
    dist.returnYPencils(data, scratch)
    f = pkg.a2adfft(dist)
    f.make_plans(torch.zeros_like(fused))
    f.forward(fused)
    tol = 1e-6 if prec == "c64" else 1e-12
    ref = oracle.fft3_global(g)
    step_out = oracle.bricks_to_global(data.cpu().numpy().reshape(P, -1), d)
    fused_out = oracle.bricks_to_global(fused.cpu().numpy().reshape(P, -1), d)
    assert oracle.rel_l2(step_out, ref) <= tol
    assert oracle.rel_l2(fused_out, ref) <= tol
    assert oracle.rel_l2(step_out, fused_out) <= tol
    # inverse sequence with the scale kernel
    dist.getZPencils(data, scratch)
    pkg.inverse_1d_fft(dist, data)
    dist.returnZPencils(data, scratch)
    dist.getXPencils(data, scratch)
    pkg.inverse_1d_fft(dist, scratch)
    dist.returnXPencils(data, scratch)
    dist.getYPencils(data, scratch)
    pkg.inverse_1d_fft(dist, data)
    pkg.scale_fft(dist, scratch, data)
    dist.returnYPencils(data, scratch)
    back = oracle.bricks_to_global(data.cpu().numpy().reshape(P, -1), d)
    assert oracle.rel_l2(back, g) <= tol


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_1d_fft_lines(pkg, oracle, cuda, prec):
    import torch

    for P, ng in [(4, 64), (8, 32), (6, 12), (4, 48)]:
        dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
        cdt = np.complex64 if prec == "c64" else np.complex128
        rng = np.random.default_rng(ng)
        x = (rng.standard_normal(P * dist.nlocal) + 1j * rng.standard_normal(P * dist.nlocal)).astype(cdt)
        t = torch.from_numpy(x.copy()).to(cuda)
        pkg.forward_1d_fft(dist, t)
        ref = oracle.dft_lines(x, ng)
        tol = 1e-6 if prec == "c64" else 1e-12
        assert oracle.rel_l2(t.cpu().numpy(), ref) <= tol
        pkg.inverse_1d_fft(dist, t)
        assert oracle.rel_l2(t.cpu().numpy(), x * ng) <= tol
