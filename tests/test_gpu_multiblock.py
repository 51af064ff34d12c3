"""The fused pass across devices (``a2a_dfft_execute_pass_blocks``): the
virtual rank-major buffer split into G blocks in separate allocations (the
layout of G GPUs, each owning a contiguous range of virtual ranks), every pass
one kernel that gathers its tiles from the owning blocks and scatters them
back.  Checked against the FP64 oracle and against the single-buffer
transform: in one process (G separate allocations on this GPU, the tiles in
one or several parts), and as two processes sharing this GPU whose blocks are
mapped into each other with CUDA IPC (``FusedDistributedDfft``; the processes
order the passes with a host barrier, no kernel waits on another).
Tolerances: relative L2 <= 1e-6 (complex64), <= 1e-12 (complex128)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = {"c64": 1e-6, "c128": 1e-12}
CDT = {"c64": np.complex64, "c128": np.complex128}


def _transform(dfft, blocks, inverse, nparts):
    import torch

    for p in range(3):
        for part in range(nparts):
            dfft.execute_pass_blocks(blocks, p, inverse, part, nparts)
        torch.cuda.synchronize()


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("prec", ["c64", "c128"])
@pytest.mark.parametrize("P,shape,G,nparts", [(4, 64, 2, 1), (16, 128, 4, 3), (64, 256, 8, 2), (8, 32, 2, 5),
                                             (4, (64, 128, 32), 4, 2), (16, (96, 64, 192), 2, 1), (16, (96, 48, 192), 2, 1),
                                             # long lines for the persistent kernels (512, 1024)
                                             (16, (512, 64, 128), 4, 3), (4, (64, 1024, 32), 2, 2),
                                             (4, (32, 64, 512), 2, 3), (4, (32, 64, 1024), 4, 2)])
def test_multiblock_passes_vs_oracle(pkg, oracle, cuda, P, shape, G, nparts, prec, persistent):
    import torch

    shape = (shape,) * 3 if isinstance(shape, int) else tuple(shape)
    dist = pkg.a2aDistribution(P, shape, 64, precision=prec)
    d = oracle.Decomp(shape, P)
    g = oracle.make_input("normal", shape, seed=13, dtype=CDT[prec])
    bricks = oracle.global_to_bricks(g, d)
    L = P // G
    blocks = [torch.from_numpy(bricks[q * L:(q + 1) * L].ravel().copy()).to(cuda) for q in range(G)]
    single = torch.from_numpy(bricks.ravel().copy()).to(cuda)
    f = pkg.a2adfft(dist)
    f.make_plans()
    f.set_blocks_kernel(persistent)
    _transform(f, blocks, False, nparts)
    f.forward(single)
    fwd = torch.cat(blocks).cpu().numpy()
    ref = oracle.fft3_global(g, lines=oracle.fft_lines)
    e = oracle.rel_l2(oracle.bricks_to_global(fwd.reshape(P, -1), d), ref)
    assert e <= TOL[prec], f"forward rel L2 {e:.3e}"
    assert oracle.rel_l2(fwd, single.cpu().numpy()) <= TOL[prec]
    _transform(f, blocks, True, nparts)
    inv = torch.cat(blocks).cpu().numpy()
    assert oracle.rel_l2(inv, bricks.ravel()) <= TOL[prec]


def test_multiblock_argument_checks(pkg, cuda):
    import torch

    dist = pkg.a2aDistribution(4, 64, 64, precision="c64")
    f = pkg.a2adfft(dist)
    f.make_plans()
    x = dist.empty(cuda)
    half = x.numel() // 2
    blocks = [x[:half], x[half:]]
    with pytest.raises(pkg.A2AError):
        f.execute_pass_blocks(blocks * 2 + blocks, 0, False)  # 6 blocks do not divide 4 ranks
    with pytest.raises(pkg.A2AError):
        f.execute_pass_blocks(blocks, 3, False)
    with pytest.raises(pkg.A2AError):
        f.execute_pass_blocks(blocks, 0, False, part=2, nparts=2)
    torch.cuda.synchronize()


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, P, ng, prec, q):
    sys.path.insert(0, ROOT)
    import importlib

    import torch
    import torch.distributed as tdist

    import __graft_entry__ as entry

    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        torch.cuda.set_device(0)
        import datetime

        tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        pkg = entry.load_package()
        O = entry.load_oracle()
        dd = importlib.import_module(pkg.__name__ + ".distributed")
        d = O.Decomp(ng, P)
        L = P // world
        g = O.make_input("normal", (ng,) * 3, seed=17, dtype=CDT[prec])
        bricks = O.global_to_bricks(g, d)
        mine = torch.from_numpy(bricks[rank * L:(rank + 1) * L].ravel().copy()).cuda()
        f = dd.FusedDistributedDfft(P, ng, prec)
        # a block of the wrong element type on one process: every process
        # refuses to bind (nothing is mapped, no process waits alone)
        wrong = torch.zeros(mine.numel(), dtype=torch.complex128 if prec == "c64" else torch.complex64,
                            device="cuda")
        try:
            f.bind(wrong if rank == 0 else mine)
            raise AssertionError("a block of the wrong element type was bound")
        except ValueError as e:
            assert "process 0" in str(e), e
        del wrong
        f.bind(mine)
        f.forward()
        ref = O.global_to_bricks(O.fft3_global(g, lines=O.fft_lines), d)[rank * L:(rank + 1) * L]
        ef = O.rel_l2(mine.cpu().numpy(), ref.ravel())
        f.inverse()
        ei = O.rel_l2(mine.cpu().numpy(), bricks[rank * L:(rank + 1) * L].ravel())
        tdist.barrier()
        f.release()
        q.put(("ok", rank, ef, ei))
        tdist.destroy_process_group()
    except Exception as e:
        q.put(("error", rank, repr(e), 0.0))
        raise


@pytest.mark.parametrize("P,ng,prec", [(8, 64, "c64"), (16, 32, "c128"), (16, 256, "c64")])
def test_fused_distributed_two_processes_one_gpu(cuda, P, ng, prec):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, P, ng, prec, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
    for r in res:
        assert r[0] == "ok", r
        assert r[2] <= TOL[prec] and r[3] <= TOL[prec], r
    assert all(p.exitcode == 0 for p in procs)


def test_ipc_import_twice_shares_one_mapping(pkg, cuda):
    """Two imports of one handle in one process (e.g. two fused objects
    binding the same peer buffer): the same address, the buffer still
    readable through the second import after the first is released, and each
    import released exactly once.  (CUDA refuses imports in the exporting
    process itself, so the handle comes from a child process.)"""
    import torch

    ctx = mp.get_context("spawn")
    q_in, q_out = ctx.Queue(), ctx.Queue()
    p = ctx.Process(target=_exporter, args=(q_in, q_out))
    p.start()
    try:
        h, off = q_out.get(timeout=120)
        a = pkg.ipc_import(h, off)
        b = pkg.ipc_import(h, off)
        assert a == b
        pkg.ipc_release(a)
        # read the 64 floats through the remaining import
        host = torch.empty(64, dtype=torch.float32).pin_memory()
        from cuda.bindings import runtime as cudart

        (err,) = cudart.cudaMemcpy(host.data_ptr(), b, 256, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == cudart.cudaError_t.cudaSuccess
        assert torch.equal(host, torch.arange(64, dtype=torch.float32))
        pkg.ipc_release(b)
        with pytest.raises(pkg.A2AError):
            pkg.ipc_release(b)
    finally:
        q_in.put("done")
        p.join(timeout=60)
    assert p.exitcode == 0


def _exporter(q_in, q_out):
    sys.path.insert(0, ROOT)
    import torch

    import __graft_entry__ as entry

    torch.cuda.set_device(0)
    pkg = entry.load_package()
    x = torch.arange(64, dtype=torch.float32, device="cuda")
    q_out.put(pkg.ipc_export(x))
    q_in.get(timeout=300)
