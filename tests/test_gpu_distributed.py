"""The distribution layer with the library's per-rank kernels on the GPU:
two processes sharing the one GPU, each holding half the virtual ranks, in
the reference's host-staged exchange mode (gloo between processes on host
memory, so no kernel waits on another process); and one process with NCCL in
device mode.  Results against the FP64 oracle."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, P, ng, prec, backend, mode, q):
    sys.path.insert(0, ROOT)
    import importlib

    import torch
    import torch.distributed as tdist

    import __graft_entry__ as entry

    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        torch.cuda.set_device(0)
        tdist.init_process_group(backend, rank=rank, world_size=world)
        pkg = entry.load_package()
        O = entry.load_oracle()
        dd = importlib.import_module(pkg.__name__ + ".distributed")
        dist = dd.DistributedDistribution(P, ng, 64, prec, mode=mode)
        d = O.Decomp(ng, P)
        L = P // world
        cdt = np.complex64 if prec == "c64" else np.complex128
        g = O.make_input("normal", (ng,) * 3, seed=9, dtype=cdt)
        bricks = O.global_to_bricks(g, d)
        data = torch.from_numpy(bricks[rank * L:(rank + 1) * L].ravel().copy()).cuda()
        f = dd.DistributedDfft(dist)
        f.make_plans(torch.zeros_like(data))
        f.forward(data)
        if backend == "nccl":
            gathered = [torch.zeros_like(data) for _ in range(world)]
            tdist.all_gather(gathered, data)
        else:  # gloo gathers host tensors
            gathered = [torch.zeros_like(data, device="cpu") for _ in range(world)]
            tdist.all_gather(gathered, data.cpu())
        fwd = torch.cat([t.cpu() for t in gathered]).numpy().reshape(P, -1)
        f.inverse(data)
        if rank == 0:
            tol = 1e-6 if prec == "c64" else 1e-12
            ef = O.rel_l2(O.bricks_to_global(fwd, d), O.fft3_global(g))
            q.put(("ok", ef, tol))
        torch.cuda.synchronize()
        tdist.destroy_process_group()
    except Exception as e:
        q.put(("error", repr(e), rank))
        raise


@pytest.mark.parametrize("world,backend,mode,P,ng,prec", [
    (2, "gloo", "host", 16, 32, "c128"),
    (2, "gloo", "host", 64, 64, "c64"),
    (1, "nccl", "device", 16, 64, "c128"),
])
def test_distributed_on_gpu(world, backend, mode, P, ng, prec):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, P, ng, prec, backend, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
    assert res[0] == "ok", res
    assert res[1] <= res[2], res
    assert all(p.exitcode == 0 for p in procs)
