"""Fused 3D transform through the C ABI (``a2a_dfft_forward`` /
``a2a_dfft_inverse``) against the FP64 oracle.

The reference's own check is ``np.allclose(np.fft.fftn(inp), out)`` and
``np.allclose(inp, inv)`` on complex64 stitched cubes (``src/a2afft/tests/
stitch.py:89``) for (world_size, Ng) = (8, 8), (8, 32), (6, 12), (4, 4)
(``tests/run_tests.py:18-21``).  Here the bar is the relative L2 error
against an FP64 DFT: <= 1e-6 for complex64, <= 1e-12 for complex128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-6, "c128": 1e-12}
CDT = {"c64": np.complex64, "c128": np.complex128}


def run_fwd_inv(pkg, O, cuda, P, ng, prec, kind="uniform", seed=0, lines=None):
    import torch

    dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
    d = O.Decomp(ng, P)
    assert dist.dims == d.dims and dist.local_grid_size == list(d.local) and dist.nlocal == d.nlocal
    g = O.make_input(kind, (ng, ng, ng), seed=seed, dtype=CDT[prec])
    x = torch.from_numpy(O.global_to_bricks(g, d).ravel()).to(cuda)
    f = pkg.a2adfft(dist)
    f.make_plans()
    f.forward(x)
    fwd = O.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    f.inverse(x)
    inv = O.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    lines = lines or (O.dft_lines if ng <= 128 else O.fft_lines)
    ref = O.fft3_global(g, lines=lines)
    return g, fwd, inv, ref


# the reference's four test grids, then the measured workloads at small sizes
GRIDS = [(8, 8), (8, 32), (6, 12), (4, 4), (4, 64), (16, 64), (64, 32), (16, 32), (4, 48), (4, 96), (2, 16),
         (1, 8), (4, 24), (16, 128), (4, 192)]


@pytest.mark.parametrize("prec", ["c64", "c128"])
@pytest.mark.parametrize("P,ng", GRIDS)
def test_forward_inverse_vs_fp64_oracle(pkg, oracle, cuda, P, ng, prec):
    g, fwd, inv, ref = run_fwd_inv(pkg, oracle, cuda, P, ng, prec)
    ef = oracle.rel_l2(fwd, ref)
    ei = oracle.rel_l2(inv, g)
    assert ef <= TOL[prec], f"forward rel L2 {ef:.3e}"
    assert ei <= TOL[prec], f"round trip rel L2 {ei:.3e}"
    if prec == "c128":
        # the reference's own acceptance test (stitch.py:89, numpy's default
        # rtol/atol), which its FP64 build is held to
        assert np.allclose(np.fft.fftn(g), fwd)
        assert np.allclose(g, inv)


@pytest.mark.parametrize("ng,P", [(256, 16), (512, 4), (1024, 4), (768, 4), (384, 4)])
def test_large_lengths_c64(pkg, oracle, cuda, ng, P):
    """Every long transform length through the 3 passes on a few-rank grid
    (long bricks), whole cube against the oracle's complex128 transform, plus
    exact DFT spot checks and the round trip."""
    import torch

    dist = pkg.a2aDistribution(P, ng, 64, precision="c64")
    d = oracle.Decomp(ng, P)
    gen = torch.Generator(device=cuda).manual_seed(4)
    n = P * dist.nlocal
    x = torch.complex(torch.rand(n, generator=gen, device=cuda) * 2 - 1,
                      torch.rand(n, generator=gen, device=cuda) * 2 - 1)
    x0 = x.clone()
    g = oracle.bricks_to_global(x0.cpu().numpy().reshape(P, -1), d)
    f = pkg.a2adfft(dist)
    f.make_plans()
    f.forward(x)
    fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    rng = np.random.default_rng(0)
    pts = [tuple(int(v) for v in rng.integers(0, ng, 3)) for _ in range(2)] + [(0, 0, 0), (ng - 1, 1, ng // 2)]
    exact = oracle.dft_points(g, pts)
    got = np.array([fwd[p] for p in pts])
    assert np.max(np.abs(got - exact)) / np.sqrt(float(ng) ** 3) <= 1e-5
    ref = oracle.fft3_fp64(g)
    del g
    assert oracle.rel_l2_chunked(fwd, ref) <= 1e-6
    del fwd, ref
    f.inverse(x)
    err = float(torch.linalg.vector_norm((x - x0).to(torch.complex128)) / torch.linalg.vector_norm(
        x0.to(torch.complex128)))
    assert err <= 1e-6


def test_box_transform(pkg, oracle, cuda):
    """Anisotropic box (no reference counterpart): 32 x 64 x 128 on 4 ranks."""
    import torch

    shape = (32, 64, 128)
    for prec in ("c64", "c128"):
        dist = pkg.a2aDistribution(4, shape, 64, precision=prec)
        d = oracle.Decomp(shape, 4)
        g = oracle.make_input("normal", shape, seed=3, dtype=CDT[prec])
        x = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
        f = pkg.a2adfft(dist)
        f.make_plans()
        f.forward(x)
        fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(4, -1), d)
        assert oracle.rel_l2(fwd, oracle.fft3_global(g)) <= TOL[prec]
        f.inverse(x)
        inv = oracle.bricks_to_global(x.cpu().numpy().reshape(4, -1), d)
        assert oracle.rel_l2(inv, g) <= TOL[prec]


VARIANT_CASES = [(4, 64), (16, 128), (4, 96), (16, 192), (16, 256), (64, 512), (4, (1024, 16, 64)),
                 (4, (16, 1024, 64)), (4, (16, 64, 1024)), (4, (768, 16, 32)), (4, (16, 768, 32)),
                 (4, (16, 32, 768)), (4, (384, 32, 32)), (4, (32, 32, 384)),
                 # long X / Y lines inside 256-element bricks (the TMA-ring tiles' single-box case)
                 (64, (1024, 32, 64)), (64, (32, 1024, 64)), (64, (768, 32, 64)), (64, (32, 768, 64))]


@pytest.mark.parametrize("prec", ["c64", "c128"])
@pytest.mark.parametrize("P,shape", VARIANT_CASES)
def test_every_launch_variant(pkg, oracle, cuda, P, shape, prec):
    """Each compiled launch variant of each pass (the autotuner may pick any of
    them) gives the transform the FP64 oracle gives."""
    import torch

    shape = (shape,) * 3 if isinstance(shape, int) else tuple(shape)
    dist = pkg.a2aDistribution(P, shape, 64, precision=prec)
    d = oracle.Decomp(shape, P)
    g = oracle.make_input("normal", shape, seed=11, dtype=CDT[prec])
    x0 = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
    f = pkg.a2adfft(dist)
    f.make_plans()
    n3 = float(np.prod(shape))
    if n3 <= 2 ** 22:
        ref = oracle.fft3_global(g)
    else:
        rng = np.random.default_rng(0)
        pts = [tuple(int(rng.integers(0, n)) for n in shape) for _ in range(4)]
        exact = oracle.dft_points(g, pts)
    tol = 1e-6 if prec == "c64" else 1e-12
    tested = 0
    for p in range(3):
        for v in range(f.variant_count(p)):
            try:
                f.select_variant(p, v)
            except pkg.A2AError:
                continue  # does not fit this geometry
            x = x0.clone()
            f.forward(x)
            fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
            if n3 <= 2 ** 22:
                assert oracle.rel_l2(fwd, ref) <= tol, f"pass {p} variant {v}"
            else:
                got = np.array([fwd[q] for q in pts])
                assert np.max(np.abs(got - exact)) / np.sqrt(n3) <= (1e-5 if prec == "c64" else 1e-12), \
                    f"pass {p} variant {v}"
            f.inverse(x)
            assert oracle.rel_l2(x.cpu().numpy(), x0.cpu().numpy()) <= tol, f"pass {p} variant {v} round trip"
            tested += 1
    assert tested >= 3


def test_autotune_report(pkg, oracle, cuda):
    import torch

    dist = pkg.a2aDistribution(16, 128, 64, precision="c64")
    f = pkg.a2adfft(dist)
    scratch = dist.empty()
    f.make_plans(scratch)
    rep = f.plan_report()
    assert rep.count("<- chosen") == 3
    d = oracle.Decomp(128, 16)
    g = oracle.make_input("uniform", (128,) * 3, seed=1, dtype=np.complex64)
    x = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
    f.forward(x)
    fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(16, -1), d)
    assert oracle.rel_l2(fwd, oracle.fft3_global(g)) <= 1e-6


@pytest.mark.parametrize("inverse_first", [False, True])
@pytest.mark.parametrize("P,shape", [(16, (512, 64, 64)), (16, (64, 512, 64)), (64, (512, 256, 128)),
                                     (16, (64, 64, 512)), (4, (32, 64, 512))])
def test_shuffle_exchange_variant(pkg, oracle, cuda, P, shape, inverse_first):
    """The kernels whose first exchange runs through warp shuffles (the
    batch-mode ring ``tmat2s`` and the line-mode register-pipelined
    ``rpipes``, 512 = 8 x 8 x 8), forced on every pass they fit, against the
    oracle's complex128 transform of the whole box (relative L2 <= 1e-6), in
    both directions."""
    import torch

    dist = pkg.a2aDistribution(P, shape, 64, precision="c64")
    d = oracle.Decomp(shape, P)
    g = oracle.make_input("uniform", shape, seed=23, dtype=np.complex64, tones=2)
    x = torch.from_numpy(oracle.global_to_bricks(g, d).ravel()).to(cuda)
    f = pkg.a2adfft(dist)
    f.make_plans()
    forced = 0
    for p, line in enumerate(_pass_reports(f)):
        idx = [i for i, ln in enumerate(line) if (" tmat2s " in ln or " rpipes " in ln) and "fits=1" in ln]
        if idx:
            f.select_variant(p, idx[0])
            forced += 1
    assert forced >= 1
    if inverse_first:
        f.inverse(x)
        ref = oracle.fft3_fp64(g, inverse=True)
    else:
        f.forward(x)
        ref = oracle.fft3_fp64(g)
    out = oracle.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    assert oracle.rel_l2(out, ref) <= 1e-6


def _pass_reports(f):
    """The plan report's variant lines grouped by pass (Z, X, Y), in variant order."""
    lines = f.plan_report().splitlines()
    return [[ln for ln in lines if ln.startswith(name + " pass")] for name in ("Z", "X", "Y")]
