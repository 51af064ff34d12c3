"""The distribution layer across processes (3d-ffts-mpi_b200/distributed.py)
on CPU: world_size 2 and 3 gloo process groups, each process holding a block
of virtual ranks.  The exchange (the alltoall over virtual ranks as one
all_to_all_single between processes plus the local chunk reorders) and the
step composition are checked bit-exactly against the oracle's single-process
steps; the per-rank kernels are the oracle's here (the test's stand-in for
the GPU library, which needs a device), and the full distributed transform
is checked against the FP64 oracle."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleLocal:
    """Per-rank kernels of a block of ranks, by the oracle (test only)."""

    def __init__(self, O, d, L):
        self.O, self.d, self.L = O, d, L

    def _np(self, t):
        return t.numpy().reshape(self.L, self.d.nlocal)

    def launch(self, name, src, dst):
        O, d = self.O, self.d
        x = self._np(src)
        if name.startswith("d_fast"):
            y = getattr(O, name[2:])(x, d)
        else:
            ax = name[2]
            m = O.unpack_map(ax, d) if "a2a_to" in name else O.pack_map(ax, d)
            y = O.scatter(x, m)
        dst.copy_(torch.from_numpy(np.ascontiguousarray(y).ravel()))

    def fft1d(self, data, inverse):
        y = self.O.dft_lines(data.numpy(), self.d.ng[0], inverse)
        data.copy_(torch.from_numpy(y.ravel().astype(np.complex128)))

    def scale(self, out, data):
        out.copy_(data / float(self.d.ng[0]) ** 3)

    def copy(self, out, data):
        out.copy_(data)


def _worker(rank, world, port, P, ng, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as tdist

    import __graft_entry__ as entry

    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        tdist.init_process_group("gloo", rank=rank, world_size=world)
        pkg = entry.load_package()
        O = entry.load_oracle()
        dd = importlib_distributed(pkg)
        d = O.Decomp(ng, P)
        L = P // world
        dist = dd.DistributedDistribution(P, ng, 64, "c128", mode="host", local=OracleLocal(O, d, L))
        assert dist.dims == d.dims and dist.nlocal == d.nlocal and dist.L == L
        # steps on a tracer input, against the oracle's steps on all ranks
        full = (np.arange(P * d.nlocal) + 0.25 * np.arange(P * d.nlocal) % 7).astype(np.complex128).reshape(P, -1)
        blk = slice(rank * L, (rank + 1) * L)
        b1 = torch.from_numpy(full[blk].ravel().copy())
        b2 = torch.zeros_like(b1)
        o1, o2 = full.copy(), np.zeros_like(full)
        for nm, on in [("getZPencils", O.get_z_pencils), ("returnZPencils", O.return_z_pencils),
                       ("getXPencils", O.get_x_pencils), ("returnXPencils", O.return_x_pencils),
                       ("getYPencils", O.get_y_pencils), ("returnYPencils", O.return_y_pencils)]:
            if nm == "returnYPencils":
                b2.copy_(b1)
                o2 = o1.copy()
            getattr(dist, nm)(b1, b2)
            o1, o2 = on(o1, o2, d)
            assert np.array_equal(b1.numpy().reshape(L, -1), o1[blk]), nm
            assert np.array_equal(b2.numpy().reshape(L, -1), o2[blk]), nm
        # the distributed transform
        g = O.make_input("uniform", (ng,) * 3, seed=3, dtype=np.complex128)
        bricks = O.global_to_bricks(g, d)
        data = torch.from_numpy(bricks[blk].ravel().copy())
        f = dd.DistributedDfft(dist)
        f.make_plans(torch.zeros_like(data))
        f.forward(data)
        gathered = [torch.zeros_like(data) for _ in range(world)]
        tdist.all_gather(gathered, data)
        fwd = torch.cat(gathered).numpy().reshape(P, -1)
        f.inverse(data)
        tdist.all_gather(gathered, data)
        inv = torch.cat(gathered).numpy().reshape(P, -1)
        if rank == 0:
            ef = O.rel_l2(O.bricks_to_global(fwd, d), O.fft3_global(g))
            ei = O.rel_l2(inv, bricks)
            q.put(("ok", ef, ei))
        tdist.destroy_process_group()
    except Exception as e:  # report to the parent instead of hanging
        q.put(("error", repr(e), rank))
        raise


def importlib_distributed(pkg):
    import importlib

    return importlib.import_module(pkg.__name__ + ".distributed")


@pytest.mark.parametrize("world,P,ng", [(2, 8, 8), (2, 16, 32), (2, 64, 32), (3, 6, 12), (2, 4, 16)])
def test_distributed_steps_and_transform_gloo(world, P, ng):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, P, ng, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
    assert res[0] == "ok", res
    assert res[1] <= 1e-13 and res[2] <= 1e-13, res
    assert all(p.exitcode == 0 for p in procs)


def test_distributed_rejects_uneven_split():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as entry

    pkg = entry.load_package()
    dd = importlib_distributed(pkg)
    import torch.distributed as tdist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    tdist.init_process_group("gloo", rank=0, world_size=1)
    try:
        # one process may hold every rank; the library must then be asked for them all
        d = dd.DistributedDistribution(4, 8, 64, "c128", local=object())
        assert d.L == 4 and d.first_rank == 0
        with pytest.raises(pkg.A2AError):
            dd.DistributedDistribution(4, 10, 64, "c128", local=object())
    finally:
        tdist.destroy_process_group()
