"""The individual remap launchers, the global-id tracer (pencils_demo), the
dump files and the host-staged transforms, on the GPU."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("P,ng", [(8, 8), (6, 12), (16, 32), (64, 32), (12, 24)])
def test_tracer_matches_oracle_steps(pkg, oracle, cuda, P, ng):
    """The sixteen snapshots of all2all_fft_pencils_demo.c through the
    library's launchers equal the oracle's (bit-exact ids), the z/x/y pencil
    snapshots hold whole pencils in natural order, and the last snapshot is
    the start layout again."""
    trace = importlib.import_module(pkg.__name__ + ".trace")
    dist = pkg.a2aDistribution(P, ng, 64, precision="c128")
    snaps = trace.trace_pencils(dist, cuda)
    d = oracle.Decomp(ng, P)
    b1 = snaps[0].copy()
    exp = [b1]
    b2 = oracle.alltoall(b1, d); exp.append(b2)
    b1 = oracle.scatter(b2, oracle.unpack_map("z", d)); exp.append(b1)
    b2 = oracle.scatter(b1, oracle.pack_map("z", d)); exp.append(b2)
    b1 = oracle.alltoall(b2, d); exp.append(b1)
    b2 = oracle.fast_z_to_x(b1, d); exp.append(b2)
    b1 = oracle.alltoall(b2, d); exp.append(b1)
    b2 = oracle.scatter(b1, oracle.unpack_map("x", d)); exp.append(b2)
    b1 = oracle.scatter(b2, oracle.pack_map("x", d)); exp.append(b1)
    b2 = oracle.alltoall(b1, d); exp.append(b2)
    b1 = oracle.fast_x_to_y(b2, d); exp.append(b1)
    b2 = oracle.alltoall(b1, d); exp.append(b2)
    b1 = oracle.scatter(b2, oracle.unpack_map("y", d)); exp.append(b1)
    b2 = oracle.scatter(b1, oracle.pack_map("y", d)); exp.append(b2)
    b1 = oracle.alltoall(b2, d); exp.append(b1)
    b2 = oracle.fast_y_to_z(b1, d); exp.append(b2)
    for k, (got, want) in enumerate(zip(snaps, exp)):
        assert np.array_equal(got, want), f"step {k}"
    for k, axis in ((2, 2), (7, 0), (12, 1)):  # z, x, y pencils
        lines = snaps[k].reshape(-1, ng)
        coord = [lines // (ng * ng), (lines // ng) % ng, lines % ng][axis]
        assert np.array_equal(coord, np.broadcast_to(np.arange(ng), coord.shape))
    assert np.array_equal(snaps[15], snaps[0])


def test_trace_files(pkg, cuda, tmp_path):
    trace = importlib.import_module(pkg.__name__ + ".trace")
    dist = pkg.a2aDistribution(8, 8, 64, precision="c128")
    trace.write_trace_files(dist, str(tmp_path), cuda)
    lines = open(tmp_path / "proc3").read().splitlines()
    assert lines[0] == "Processor 3, coords [0,1,1]" and lines[1] == "step0"
    assert len(lines) == 1 + 16 * (1 + dist.nlocal)


@pytest.mark.parametrize("P,ng", [(8, 8), (8, 32), (6, 12), (4, 4)])
def test_reference_dump_check_on_library_output(pkg, oracle, cuda, tmp_path, P, ng):
    """The reference's own test flow on its own test grids: its input
    (rand()/RAND_MAX on every rank), the library's forward and inverse,
    dumped in its file format and checked with its checker's assertions."""
    import os

    import torch

    dumps = importlib.import_module(pkg.__name__ + ".dumps")
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_tests.npz"))
    x0 = fx[f"P{P}_N{ng}_input"].ravel()
    dist = pkg.a2aDistribution(P, ng, 64, precision="c128")
    f = pkg.a2adfft(dist)
    f.make_plans(dist.empty(cuda))
    x = torch.from_numpy(x0.copy()).to(cuda)
    f.forward(x)
    fwd = x.cpu().numpy()
    assert np.allclose(fwd, fx[f"P{P}_N{ng}_forward"].ravel())
    f.inverse(x)
    dist.write_dims(str(tmp_path / "dims"))
    pkg.write_rank_dumps(ng, P, str(tmp_path), x0, fwd, x.cpu().numpy())
    assert dumps.check(str(tmp_path)) == (True, True)


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_host_staged_transform(pkg, oracle, cuda, prec):
    import torch

    P, ng = 16, 64
    dist = pkg.a2aDistribution(P, ng, 64, precision=prec)
    d = oracle.Decomp(ng, P)
    cdt = np.complex64 if prec == "c64" else np.complex128
    g = oracle.make_input("normal", (ng,) * 3, seed=7, dtype=cdt)
    host = torch.from_numpy(oracle.global_to_bricks(g, d).ravel().copy()).pin_memory()
    dbuf = dist.empty(cuda)
    f = pkg.a2adfft(dist)
    f.make_plans()
    f.forward_host(host, dbuf)
    tol = 1e-6 if prec == "c64" else 1e-12
    assert oracle.rel_l2(oracle.bricks_to_global(host.numpy().reshape(P, -1), d), oracle.fft3_global(g)) <= tol
    f.inverse_host(host.numpy(), dbuf)
    assert oracle.rel_l2(oracle.bricks_to_global(host.numpy().reshape(P, -1), d), g) <= tol


def test_individual_launchers_bit_exact(pkg, oracle, cuda):
    import torch

    for P, ng in [(8, 32), (64, 32), (6, 12)]:
        dist = pkg.a2aDistribution(P, ng, 64, precision="c64")
        d = oracle.Decomp(ng, P)
        src = np.arange(P * d.nlocal, dtype=np.float32).astype(np.complex64).reshape(P, -1)
        ts = torch.from_numpy(src.ravel().copy()).to(cuda)
        td = torch.zeros_like(ts)
        checks = [("d_z_a2a_to_z_pencils", lambda b: oracle.scatter(b, oracle.unpack_map("z", d))),
                  ("d_z_pencils_to_z_a2a", lambda b: oracle.scatter(b, oracle.pack_map("z", d))),
                  ("d_x_a2a_to_x_pencils", lambda b: oracle.scatter(b, oracle.unpack_map("x", d))),
                  ("d_x_pencils_to_x_a2a", lambda b: oracle.scatter(b, oracle.pack_map("x", d))),
                  ("d_y_a2a_to_y_pencils", lambda b: oracle.scatter(b, oracle.unpack_map("y", d))),
                  ("d_y_pencils_to_y_a2a", lambda b: oracle.scatter(b, oracle.pack_map("y", d))),
                  ("d_fast_z_to_x", lambda b: oracle.fast_z_to_x(b, d)),
                  ("d_fast_x_to_y", lambda b: oracle.fast_x_to_y(b, d)),
                  ("d_fast_y_to_z", lambda b: oracle.fast_y_to_z(b, d))]
        for name, ref in checks:
            dist.launch(name, ts, td)
            assert np.array_equal(td.cpu().numpy().reshape(P, -1), ref(src)), name
        dist.alltoall(ts, td)
        assert np.array_equal(td.cpu().numpy().reshape(P, -1), oracle.alltoall(src, d))
