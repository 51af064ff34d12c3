"""Global-id tracer of the pencil steps -- the reference's pencils_demo
(``src/pencils_demo/all2all_fft_pencils_demo.c:18-133``) run through this
library's kernels.

Every cell starts with its global id ``x*Ng*Ng + y*Ng + z`` and the sixteen
snapshots the demo saves are taken after each of its calls: the alltoalls,
the six pack/unpack remaps and the three fast-axis changes, in the demo's
order.  Ids are carried in the real part of a complex128 buffer (exact below
2^53)."""
from __future__ import annotations

import os

import numpy as np

# (operation, source buffer, destination buffer) per step 1..15 of the demo
_STEPS = [
    ("alltoall", 1, 2), ("d_z_a2a_to_z_pencils", 2, 1), ("d_z_pencils_to_z_a2a", 1, 2), ("alltoall", 2, 1),
    ("d_fast_z_to_x", 1, 2), ("alltoall", 2, 1), ("d_x_a2a_to_x_pencils", 1, 2), ("d_x_pencils_to_x_a2a", 2, 1),
    ("alltoall", 1, 2), ("d_fast_x_to_y", 2, 1), ("alltoall", 1, 2), ("d_y_a2a_to_y_pencils", 2, 1),
    ("d_y_pencils_to_y_a2a", 1, 2), ("alltoall", 2, 1), ("d_fast_y_to_z", 1, 2),
]


def trace_pencils(dist, device="cuda") -> list:
    """Sixteen ``(world_size, nlocal)`` int64 arrays of global ids: the demo's
    snapshots 0..15.  ``dist`` must be a complex128 cube distribution."""
    import torch

    if dist.dtype != torch.complex128:
        raise TypeError("the tracer carries ids in a complex128 distribution")
    ng, P = dist.Ng, dist.world_size
    ids = np.empty(P * dist.nlocal, dtype=np.int64)
    for r in range(P):
        sx, sy, sz = dist.local_coordinates_start(r)
        lx, ly, lz = dist.local_grid_size
        x, y, z = np.meshgrid(np.arange(lx) + sx, np.arange(ly) + sy, np.arange(lz) + sz, indexing="ij")
        ids[r * dist.nlocal:(r + 1) * dist.nlocal] = (x * ng * ng + y * ng + z).ravel()
    bufs = {1: torch.from_numpy(ids.astype(np.complex128)).to(device),
            2: torch.zeros(P * dist.nlocal, dtype=torch.complex128, device=device)}
    snaps = [ids.reshape(P, -1).copy()]
    for op, src, dst in _STEPS:
        if op == "alltoall":
            dist.alltoall(bufs[src], bufs[dst])
        else:
            dist.launch(op, bufs[src], bufs[dst])
        snaps.append(bufs[dst].real.round().to(torch.int64).cpu().numpy().reshape(P, -1))
    return snaps


def write_trace_files(dist, folder: str, device="cuda") -> None:
    """The demo's text dumps: ``<folder>/proc<r>`` with a header line and, per
    step, ``step<k>`` followed by one ``x,y,z`` line per cell."""
    ng = dist.Ng
    snaps = trace_pencils(dist, device)
    os.makedirs(folder, exist_ok=True)
    for r in range(dist.world_size):
        c = dist.coords(r)
        with open(os.path.join(folder, f"proc{r}"), "w") as fh:
            fh.write(f"Processor {r}, coords [{c[0]},{c[1]},{c[2]}]\n")
            for k, s in enumerate(snaps):
                fh.write(f"step{k}\n")
                x, rem = np.divmod(s[r], ng * ng)
                y, z = np.divmod(rem, ng)
                fh.write("".join(f"{a},{b},{e}\n" for a, b, e in zip(x, y, z)))
