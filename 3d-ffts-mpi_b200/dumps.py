"""Readers for the reference's debug dump files, so its own style of check
runs against this library's output.

The reference writes a ``dims`` file (nine int32: world_size, Ng, nlocal,
dims[3], local_grid_size[3]; ``src/a2afft/distribution/a2adistribution.cpp:101-111``)
and one ``proc<r>`` file per rank holding that rank's brick of the input, the
forward result and the inverse result (``src/a2afft/tests/test.cpp:69-125``).
Its checker reassembles the bricks with ``rank2coords`` and asserts
``np.allclose(np.fft.fftn(inp), out)`` and ``np.allclose(inp, inv)``
(``src/a2afft/tests/stitch.py:28-89``).  The writers are
``a2afft_b200.write_dims`` / ``write_rank_dumps`` (C ABI ``a2a_write_dims``,
``a2a_write_rank_dumps``).
"""
from __future__ import annotations

import os

import numpy as np


def read_dims(path: str) -> dict:
    v = np.fromfile(path, dtype=np.int32)
    if v.size != 9:
        raise ValueError(f"{path}: expected 9 int32, found {v.size}")
    return {"world_size": int(v[0]), "Ng": int(v[1]), "nlocal": int(v[2]), "dims": [int(x) for x in v[3:6]],
            "local_grid_size": [int(x) for x in v[6:9]]}


def read_rank_dumps(folder: str, params: dict, dtype=np.complex128) -> np.ndarray:
    """``(world_size, steps, nlocal)`` array of every rank's dumped bricks."""
    rdt = np.float64 if dtype == np.complex128 else np.float32
    out = []
    for r in range(params["world_size"]):
        raw = np.fromfile(os.path.join(folder, f"proc{r}"), dtype=rdt)
        data = raw[0::2] + 1j * raw[1::2]
        out.append(data.reshape(-1, params["nlocal"]))
    return np.array(out)


def stitch(bricks: np.ndarray, params: dict) -> np.ndarray:
    """Rank-major bricks ``(world_size, nlocal)`` -> global ``[x][y][z]`` cube,
    placing rank r's brick at ``local_grid_size * rank2coords(r)``."""
    d0, d1, d2 = params["dims"]
    lx, ly, lz = params["local_grid_size"]
    v = np.asarray(bricks).reshape(d0, d1, d2, lx, ly, lz).transpose(0, 3, 1, 4, 2, 5)
    ng = params["Ng"]
    return np.ascontiguousarray(v).reshape(ng, ng, ng)


def check(folder: str, dtype=np.complex128) -> tuple[bool, bool]:
    """The reference checker's two assertions on a dump folder: forward equals
    ``np.fft.fftn`` of the input, inverse equals the input."""
    params = read_dims(os.path.join(folder, "dims"))
    raw = read_rank_dumps(folder, params, dtype)
    inp, out, inv = (stitch(raw[:, k], params) for k in range(3))
    return bool(np.allclose(np.fft.fftn(inp), out)), bool(np.allclose(inp, inv))
