"""CPU checks of the oracle (no GPU): its decomposition and every remap are
pinned bit-exactly against what the reference's own remap code produces
(committed fixtures from tests/golden/make_golden.py, and the compiled
reference itself when oracle/_ref is built), and its transform against the
reference's own acceptance test on the reference's own test input."""
import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libpencils_ref.so")


@pytest.fixture(scope="module")
def remaps():
    return np.load(os.path.join(GOLDEN, "remaps.npz"))


def grids(remaps):
    keys = sorted({k.split("_")[0] + "_" + k.split("_")[1] for k in remaps.files})
    return [(int(k.split("_")[0][1:]), int(k.split("_")[1][1:])) for k in keys]


def apply_sequential(new_idx, n, size):
    """dest[new_idx[i]] = i for i = 0..n-1 in order (the reference's loop),
    into a -1 filled buffer of `size` cells: later writes win."""
    dest = np.full(size, -1, dtype=np.int64)
    order = np.arange(n)
    # last writer per destination: unique over the reversed sequence
    rev_dst = new_idx[::-1]
    uniq, first = np.unique(rev_dst, return_index=True)
    dest[uniq] = order[::-1][first]
    return dest


def test_dims_create_known_values(oracle):
    expect = {1: [1, 1, 1], 2: [2, 1, 1], 3: [3, 1, 1], 4: [2, 2, 1], 6: [3, 2, 1], 8: [2, 2, 2], 12: [3, 2, 2],
              16: [4, 2, 2], 24: [4, 3, 2], 32: [4, 4, 2], 64: [4, 4, 4], 128: [8, 4, 4], 256: [8, 8, 4],
              512: [8, 8, 8]}
    for n, dims in expect.items():
        assert oracle.dims_create(n, 3) == dims, n


def test_decomposition_rules(oracle):
    d = oracle.Decomp(512, 64)
    assert d.dims == [4, 4, 4] and d.local == (128, 128, 128) and d.nlocal == 128 ** 3 and d.chunk == 32768
    assert d.coords(0) == (0, 0, 0) and d.coords(63) == (3, 3, 3) and d.coords(6) == (0, 1, 2)
    assert d.local_start(6) == (0, 128, 256)
    for ng, P in [(10, 4), (8, 6), (64, 256), (0, 4)]:  # the reference asserts on these
        with pytest.raises(oracle.DecompositionError):
            oracle.Decomp(ng, P)


def test_remaps_match_reference_fixtures(oracle, remaps):
    for P, ng in grids(remaps):
        d = oracle.Decomp(ng, P)
        key = f"P{P}_N{ng}"
        for ax in "zxy":
            ref = remaps[f"{key}_{ax}_a2a_to_{ax}_pencils"]
            mine = apply_sequential(oracle.unpack_map(ax, d), d.nlocal, ref.size)
            assert np.array_equal(mine, ref), f"{key} {ax} unpack"
            ref = remaps[f"{key}_{ax}_pencils_to_{ax}_a2a"]
            m = oracle.y_pencils_to_y_a2a_ref_map(d) if ax == "y" else oracle.pack_map(ax, d)
            mine = apply_sequential(m, d.nlocal, ref.size)
            assert np.array_equal(mine, ref), f"{key} {ax} pack"
        for nm in ("fast_z_to_x", "fast_x_to_y", "fast_y_to_z"):
            mine = getattr(oracle, nm)(np.arange(d.nlocal)[None], d)[0]
            assert np.array_equal(mine, remaps[f"{key}_{nm}"]), f"{key} {nm}"


def test_unpack_maps_are_permutations_and_pack_inverts(oracle, remaps):
    for P, ng in grids(remaps):
        d = oracle.Decomp(ng, P)
        for ax in "zxy":
            u = oracle.unpack_map(ax, d)
            assert np.array_equal(np.sort(u), np.arange(d.nlocal))
            assert np.array_equal(oracle.pack_map(ax, d)[u], np.arange(d.nlocal))


def test_reference_y_pack_bug_is_where_predicted(oracle, remaps):
    """The reference's d_y_pencils_to_y_a2a equals the true inverse of the Y
    unpack exactly when dims[1] == 2 or dims[0] == 1; elsewhere it is not a
    permutation (cells never written, cells written twice, writes past the
    buffer), which the fixtures record."""
    seen_bad = 0
    for P, ng in grids(remaps):
        d = oracle.Decomp(ng, P)
        valid = oracle.y_return_is_valid(d)
        assert valid == (d.dims[1] == 2 or d.dims[0] == 1), (P, ng, d.dims)
        ref = remaps[f"P{P}_N{ng}_y_pencils_to_y_a2a"]
        written = ref[: d.nlocal] >= 0
        if valid:
            assert written.all() and (ref[d.nlocal:] == -1).all()
        else:
            seen_bad += 1
            m = oracle.y_pencils_to_y_a2a_ref_map(d)
            assert len(np.unique(m)) < d.nlocal or m.max() >= d.nlocal
    assert seen_bad >= 3


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built (needs the reference tree)")
def test_remaps_match_live_reference(oracle):
    lib = ctypes.CDLL(REF_LIB)
    IP = ctypes.POINTER(ctypes.c_int)
    for P in (1, 2, 4, 6, 8, 12, 16, 24, 32, 64, 128):
        for ng in (8, 12, 16, 24, 32, 48, 64):
            try:
                d = oracle.Decomp(ng, P)
            except oracle.DecompositionError:
                continue
            loc = (ctypes.c_int * 3)(*d.local)
            dims = (ctypes.c_int * 3)(*d.dims)
            src = np.arange(d.nlocal, dtype=np.int32)
            for ax in "zxy":
                for nm, m in ((f"{ax}_a2a_to_{ax}_pencils", oracle.unpack_map(ax, d)),
                              (f"{ax}_pencils_to_{ax}_a2a",
                               oracle.y_pencils_to_y_a2a_ref_map(d) if ax == "y" else oracle.pack_map(ax, d))):
                    size = max(d.nlocal, int(m.max()) + 1) + 64
                    dst = np.full(size, -1, dtype=np.int32)
                    getattr(lib, nm)(src.ctypes.data_as(IP), dst.ctypes.data_as(IP), P, 0, d.nlocal, loc, dims)
                    assert np.array_equal(apply_sequential(m, d.nlocal, size), dst), (P, ng, nm)


def test_pipeline_on_reference_test_input(oracle):
    """The reference's own check (stitch.py:89) on its own input: every rank's
    brick holds rand()/RAND_MAX (identical bricks), forward must equal
    np.fft.fftn of the stitched cube and inverse must give the input back."""
    fx = np.load(os.path.join(GOLDEN, "reference_tests.npz"))
    for P, ng in [(8, 8), (8, 32), (6, 12), (4, 4)]:
        d = oracle.Decomp(ng, P)
        x = fx[f"P{P}_N{ng}_input"]
        ref = fx[f"P{P}_N{ng}_forward"]
        f = oracle.forward(x, d)
        assert oracle.rel_l2(f, ref) <= 1e-13
        assert np.allclose(f, ref)
        inv = oracle.inverse(f, d)
        assert np.allclose(inv, x) and oracle.rel_l2(inv, x) <= 1e-13


@pytest.mark.parametrize("P,ng", [(4, 64), (16, 32), (64, 32), (2, 16), (6, 12)])
def test_pipeline_matches_fftn_and_separable_dft(oracle, P, ng):
    d = oracle.Decomp(ng, P)
    g = oracle.make_input("uniform", (ng,) * 3, seed=0, dtype=np.complex128)
    b = oracle.global_to_bricks(g, d)
    assert np.array_equal(oracle.bricks_to_global(b, d), g)
    ref = np.fft.fftn(g)
    assert oracle.rel_l2(oracle.bricks_to_global(oracle.forward(b, d), d), ref) <= 1e-13
    assert oracle.rel_l2(oracle.fft3_global(g), ref) <= 1e-13
    assert oracle.rel_l2(oracle.fft3_global(g, lines=oracle.fft_lines), ref) <= 1e-13


def test_brick_offsets_are_separable(oracle):
    for P, ng in [(64, 32), (16, 64), (6, 12), (256, 128)]:
        d = oracle.Decomp(ng, P)
        ox, oy, oz = oracle.brick_offsets(d)
        g = np.arange(ng ** 3).reshape((ng,) * 3)
        flat = oracle.global_to_bricks(g, d).ravel()
        assert np.array_equal(flat[ox[:, None, None] + oy[None, :, None] + oz[None, None, :]], g)


def test_dft_points_and_tones(oracle):
    g = oracle.make_input("uniform", (16, 8, 12), seed=2, dtype=np.complex128, tones=2)
    pts = [(0, 0, 0), (3, 5, 7), (15, 7, 11)]
    full = np.fft.fftn(g)
    assert np.allclose(oracle.dft_points(g, pts), [full[p] for p in pts])


@pytest.mark.parametrize("P,ng", [(4, 16), (8, 8), (6, 12), (64, 32), (16, 32), (256, 128), (1, 8)])
def test_host_pipeline_matches_the_step_functions(oracle, P, ng):
    """The threaded host pipeline (the benchmark's reference arm) takes every
    step to the same buffers, bit for bit, as the oracle's step functions, and
    its transform equals the oracle's."""
    import torch

    d = oracle.Decomp(ng, P)
    hp = oracle.HostPipeline(d, "c128", threads=2)
    g = oracle.make_input("normal", (ng,) * 3, seed=5, dtype=np.complex128)
    b = oracle.global_to_bricks(g, d)
    b1, b2 = b.copy(), np.zeros_like(b)
    hp.b1.copy_(torch.from_numpy(b.ravel()))
    for name in ("get_z_pencils", "return_z_pencils", "get_x_pencils", "return_x_pencils", "get_y_pencils",
                 "return_y_pencils"):
        if name == "return_y_pencils":  # the parity copy fills Buff2 first
            b2 = b1.copy()
            hp.b2.copy_(hp.b1)
        b1, b2 = getattr(oracle, name)(b1, b2, d)
        getattr(hp, name)()
        assert np.array_equal(hp.b1.numpy().reshape(P, -1), b1), name
        assert np.array_equal(hp.b2.numpy().reshape(P, -1), b2), name
    if ng <= 32:
        hp.b1.copy_(torch.from_numpy(b.ravel()))
        hp.run(False)
        assert oracle.rel_l2(hp.b1.numpy().reshape(P, -1), oracle.forward(b, d)) <= 1e-12
        hp.run(True)
        assert oracle.rel_l2(hp.b1.numpy().reshape(P, -1), b) <= 1e-12
