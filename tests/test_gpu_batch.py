"""Batched form (``a2a_batch_*``: many boxes, one persistent launch per
direction, or the grouped schedule through the single-grid pass kernels)
against the FP64 oracle, against the single-grid plan (``a2a_dfft_*``) box
by box, across its schedules, and its bounded-wait timeout path.
Tolerances as for the single-grid transform: relative L2 error <= 1e-6 for
complex64, <= 1e-12 for complex128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-6, "c128": 1e-12}
CDT = {"c64": np.complex64, "c128": np.complex128}

# every batched length in both access modes, cubes and boxes whose line
# counts force the smaller tile for some lengths
SMALL = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (96, 96, 96), (32, 64, 128), (128, 48, 32), (192, 32, 64),
         (64, 256, 32), (32, 32, 512)]


def fill(pkg, O, cuda, batch, prec, seed=3, kind="normal"):
    import torch

    flat, views = batch.empty(cuda)
    flat.zero_()
    inputs = []
    for i, shp in enumerate(batch.shapes):
        d = O.Decomp(shp, batch.world_size)
        g = O.make_input(kind, shp, seed=seed + i, dtype=CDT[prec])
        views[i].copy_(torch.from_numpy(O.global_to_bricks(g, d).ravel()))
        inputs.append((g, d))
    return flat, views, inputs


def to_global(O, view, d, P):
    return O.bricks_to_global(view.cpu().numpy().reshape(P, -1), d)


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_batch_forward_inverse_vs_oracle(pkg, oracle, cuda, prec):
    P = 4
    b = pkg.a2aBatch(SMALL, P, prec)
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec)
    b.forward(views)
    for i, (g, d) in enumerate(inputs):
        ref = oracle.fft3_global(g, lines=oracle.fft_lines)
        e = oracle.rel_l2(to_global(oracle, views[i], d, P), ref)
        assert e <= TOL[prec], f"box {i} {b.shapes[i]} forward rel L2 {e:.3e}"
    b.inverse(views)
    for i, (g, d) in enumerate(inputs):
        e = oracle.rel_l2(to_global(oracle, views[i], d, P), g)
        assert e <= TOL[prec], f"box {i} {b.shapes[i]} round trip rel L2 {e:.3e}"


def test_batch_matches_single_grid_plan(pkg, oracle, cuda):
    """Each box's batched transform equals what a2a_dfft gives the same box
    on its own distribution (same layout, same definition)."""
    import torch

    P, prec = 4, "c64"
    b = pkg.a2aBatch(SMALL, P, prec)
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec, seed=11)
    singles = [v.clone() for v in views]
    b.forward(views)
    for i, shp in enumerate(b.shapes):
        dist = pkg.a2aDistribution(P, shp, 64, precision=prec)
        f = pkg.a2adfft(dist)
        f.make_plans()
        f.forward(singles[i])
        e = oracle.rel_l2(views[i].cpu().numpy(), singles[i].cpu().numpy())
        assert e <= TOL[prec], f"box {i} {shp}: batched vs single-grid rel diff {e:.3e}"
        f.destroy()
        dist.finalize()
    torch.cuda.synchronize()


@pytest.mark.parametrize("fused,claim,prefetch,graph", [(1, 1, 1, True), (1, 4, 0, True), (0, 2, 1, True),
                                                        (1, 8, 1, False), (0, 1, 0, False)])
def test_batch_schedules_agree_bitwise(pkg, oracle, cuda, fused, claim, prefetch, graph):
    """The schedule only orders the same tiles: results are bit-identical."""
    import torch

    P, prec = 4, "c64"
    ref_b = pkg.a2aBatch(SMALL, P, prec)
    flat, views, _ = fill(pkg, oracle, cuda, ref_b, prec, seed=5)
    flat2 = flat.clone()
    views2 = [flat2[o:o + n] for o, n in zip(ref_b.offsets()[:-1], ref_b.elements)]
    ref_b.forward(views)
    ref_b.inverse(views)
    b = pkg.a2aBatch(SMALL, P, prec)
    b.set_schedule(fused=bool(fused), claim=claim, prefetch=bool(prefetch))
    b.set_graph(graph)
    assert b.launches_per_transform == (1 if fused else 3)
    s = torch.cuda.Stream()
    b.forward(views2, stream=s)
    b.inverse(views2, stream=s)
    s.synchronize()
    b.check_device()
    assert torch.equal(flat, flat2)


# repeated shapes, so that groups hold several boxes
GROUPED = SMALL + [(32, 32, 32), (64, 64, 64), (32, 64, 128), (32, 64, 128), (192, 32, 64)]


@pytest.mark.parametrize("prec,graph", [("c64", True), ("c64", False), ("c128", True)])
def test_batch_grouped_schedule_vs_oracle(pkg, oracle, cuda, prec, graph):
    """The grouped schedule: the boxes of each shape as one tall grid per
    pass through the single-grid pass kernels, the shapes on parallel stream
    branches (one graph branch per shape when captured)."""
    import torch

    P = 4
    b = pkg.a2aBatch(GROUPED, P, prec)
    b.set_schedule(grouped=True)
    b.set_graph(graph)
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec, seed=31)
    assert b.launches_per_transform == 1  # nothing bound yet: no group tables
    s = torch.cuda.Stream()
    b.forward(views, stream=s)
    s.synchronize()
    b.check_device()
    assert b.launches_per_transform == 3 * len(set(GROUPED))
    assert "schedule=grouped " in b.plan_report()
    for i, (g, d) in enumerate(inputs):
        ref = oracle.fft3_global(g, lines=oracle.fft_lines)
        e = oracle.rel_l2(to_global(oracle, views[i], d, P), ref)
        assert e <= TOL[prec], f"box {i} {b.shapes[i]} forward rel L2 {e:.3e}"
    b.inverse(views, stream=s)
    s.synchronize()
    b.check_device()
    for i, (g, d) in enumerate(inputs):
        e = oracle.rel_l2(to_global(oracle, views[i], d, P), g)
        assert e <= TOL[prec], f"box {i} {b.shapes[i]} round trip rel L2 {e:.3e}"


def test_batch_grouped_matches_single_grid_and_rebinds(pkg, oracle, cuda):
    """Grouped results equal each box's own single-grid plan; binding other
    buffers (the groups' base pointers move) rebuilds the line-base tables
    and the captured graph."""
    import torch

    P, prec = 4, "c64"
    b = pkg.a2aBatch(GROUPED, P, prec)
    b.set_schedule(grouped=True)
    for seed in (41, 43):  # two different allocations in turn
        flat, views, _ = fill(pkg, oracle, cuda, b, prec, seed=seed)
        singles = [v.clone() for v in views]
        b.forward(views)
        for i, shp in enumerate(b.shapes):
            dist = pkg.a2aDistribution(P, shp, 64, precision=prec)
            f = pkg.a2adfft(dist)
            f.make_plans()
            f.forward(singles[i])
            e = oracle.rel_l2(views[i].cpu().numpy(), singles[i].cpu().numpy())
            assert e <= TOL[prec], f"seed {seed} box {i} {shp}: grouped vs single-grid rel diff {e:.3e}"
            f.destroy()
            dist.finalize()
        torch.cuda.synchronize()


def test_batch_line_pairs_bit_identical(pkg, oracle, cuda):
    """Variant 2 (batch mode, each thread moving two adjacent lines as one
    16-byte access) computes every line exactly as variant 0 does."""
    import torch

    P, prec = 4, "c64"
    ref_b = pkg.a2aBatch(SMALL, P, prec)
    flat, views, _ = fill(pkg, oracle, cuda, ref_b, prec, seed=23)
    flat2 = flat.clone()
    views2 = [flat2[o:o + n] for o, n in zip(ref_b.offsets()[:-1], ref_b.elements)]
    ref_b.forward(views)
    ref_b.inverse(views)
    b = pkg.a2aBatch(SMALL, P, prec)
    paired = 0
    for n in (32, 48, 64, 96, 128, 192, 256, 512):
        try:
            b.select_variant(n, True, 2)
            paired += 1
        except pkg.A2AError:
            pass  # unused length, or a box whose lines do not pair
    assert paired >= 4, b.plan_report()
    assert "as pairs" in b.plan_report()
    with pytest.raises(pkg.A2AError):
        b.select_variant(64, False, 2)  # line mode has no pairs
    b.forward(views2)
    b.inverse(views2)
    assert torch.equal(flat, flat2)


def test_batch_variants_and_autotune(pkg, oracle, cuda):
    P, prec = 4, "c64"
    b = pkg.a2aBatch(SMALL, P, prec)
    scratch, sviews = b.empty(cuda)
    scratch.normal_()
    b.make_plans(sviews)
    rep = b.plan_report()
    assert "schedule=" in rep and "N=512" in rep
    # a forced tile choice that does not divide every box is refused and the
    # plan stays usable
    with pytest.raises(pkg.A2AError):
        b.select_variant(32, False, 0)  # 48 lines (box 128x48x32, Z pass) do not split into 32-line tiles
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec, seed=21)
    b.forward(views)
    for i, (g, d) in enumerate(inputs):
        ref = oracle.fft3_global(g, lines=oracle.fft_lines)
        e = oracle.rel_l2(to_global(oracle, views[i], d, P), ref)
        assert e <= TOL[prec], f"box {i} forward rel L2 {e:.3e} after tuning"


def test_batch_wait_timeout_is_reported_and_recoverable(pkg, oracle, cuda):
    """A device-side wait that nothing satisfies gives up after about a
    second; the synchronising call reports A2A_ERROR_TIMEOUT, and the
    context stays usable for the next (normal) call."""
    P, prec = 4, "c64"
    shapes = [(32, 32, 32), (64, 64, 64)]
    b = pkg.a2aBatch(shapes, P, prec)
    b.set_schedule(fused=True, claim=1)
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec, seed=7)
    b.inject_stall(True)
    with pytest.raises(pkg.A2AError) as ei:
        b.forward(views)
    assert ei.value.status == 8  # A2A_ERROR_TIMEOUT
    b.check_device()  # the flag was cleared by the failing call
    b.inject_stall(False)
    flat, views, inputs = fill(pkg, oracle, cuda, b, prec, seed=8)
    b.forward(views)
    for i, (g, d) in enumerate(inputs):
        ref = oracle.fft3_global(g, lines=oracle.fft_lines)
        assert oracle.rel_l2(to_global(oracle, views[i], d, P), ref) <= TOL[prec]


@pytest.mark.parametrize("grouped", [False, True])
def test_batch_measured_workload_properties(pkg, oracle, cuda, grouped):
    """The measured batch (96 cubes with edges drawn from 32..192, seed 3,
    plus two 128x256x512 boxes; 4 virtual ranks each, N(0,1) input):
    exact DFT at sample points, Parseval and the round trip, per box, in
    the one-launch and the grouped schedule."""
    import torch

    P, prec = 4, "c64"
    shapes = pkg.batch_shapes()
    assert len(shapes) == 98
    b = pkg.a2aBatch(shapes, P, prec)
    if grouped:
        b.set_schedule(grouped=True)
    flat, views = b.empty(cuda)
    gen = torch.Generator(device=cuda)
    gen.manual_seed(3)
    flat.copy_(torch.complex(torch.randn(flat.numel(), generator=gen, device=cuda),
                             torch.randn(flat.numel(), generator=gen, device=cuda)))
    x0 = flat.clone()
    rng = np.random.default_rng(0)
    check = sorted(set([0, 1, 2, 95, 96, 97] + list(rng.integers(0, 98, 6))))
    before = {i: views[i].cpu().numpy() for i in check}
    b.forward(views)
    for i in check:
        shp = shapes[i]
        d = oracle.Decomp(shp, P)
        g = oracle.bricks_to_global(before[i].reshape(P, -1), d)
        out = to_global(oracle, views[i], d, P)
        pts = [tuple(int(rng.integers(0, n)) for n in shp) for _ in range(4)] + [(0, 0, 0)]
        exact = oracle.dft_points(g, pts)
        got = np.array([out[p] for p in pts])
        scale = np.sqrt(float(np.prod(shp)))
        assert np.max(np.abs(got - exact)) / scale <= 1e-5, f"box {i} {shp}"
        ex = float(np.sum(np.abs(g.astype(np.complex128)) ** 2)) * float(np.prod(shp))
        assert abs(float(np.sum(np.abs(out.astype(np.complex128)) ** 2)) / ex - 1.0) <= 1e-5, f"box {i} Parseval"
    b.inverse(views)
    for i, v in enumerate(views):
        o, n = b.offsets()[i], b.elements[i]
        e = float(torch.linalg.vector_norm((v - x0[o:o + n]).to(torch.complex128)) /
                  torch.linalg.vector_norm(x0[o:o + n].to(torch.complex128)))
        assert e <= 1e-6, f"box {i} {shapes[i]} round trip rel L2 {e:.3e}"
