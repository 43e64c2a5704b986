"""Reader of the solve dumps the oracle binary writes (YZO_DUMP_DIR, see
oracle/backend/oracle_backend.cpp) and of the .npz fixtures made from them.

Dump layout (little endian): 8-byte magic "YZDUMP1\\0"; int32 n, nnz,
precondition, scaling, max_iteration, conc, flavour, ret; int32 iter; float64
epsilon, resid; int32 rowptr[n+1], col[nnz] (storage order), sorted_col[nnz],
sorted_src[nnz], bc[n]; float64 values[nnz] (storage order), rhs[n], x0[n],
x[n] (the oracle's answer).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

KEYS_INT = ("n", "nnz", "precondition", "scaling", "max_iteration", "conc", "flavour", "ret", "iter")


def read_dump(path) -> dict:
    raw = Path(path).read_bytes()
    if raw[:8] != b"YZDUMP1\x00":
        raise ValueError(f"{path}: not a solve dump")
    off = 8
    hdr = np.frombuffer(raw, dtype="<i4", count=9, offset=off)
    off += 36
    eps, resid = np.frombuffer(raw, dtype="<f8", count=2, offset=off)
    off += 16
    d = {k: int(v) for k, v in zip(KEYS_INT, hdr)}
    d["epsilon"], d["resid"] = float(eps), float(resid)
    n, nnz = d["n"], d["nnz"]

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off).copy()
        off += a.nbytes
        return a

    d["rowptr"] = take("<i4", n + 1)
    d["col"] = take("<i4", nnz)
    d["sorted_col"] = take("<i4", nnz)
    d["sorted_src"] = take("<i4", nnz)
    d["bc"] = take("<i4", n)
    d["values"] = take("<f8", nnz)
    d["rhs"] = take("<f8", n)
    d["x0"] = take("<f8", n)
    d["x"] = take("<f8", n)
    return d


def save_npz(path, dumps: list[dict]) -> None:
    arrays = {}
    for j, d in enumerate(dumps):
        for k, v in d.items():
            arrays[f"{j}.{k}"] = np.asarray(v)
    arrays["count"] = np.asarray(len(dumps))
    np.savez_compressed(path, **arrays)


def load_npz(path) -> list[dict]:
    z = np.load(path)
    out = []
    for j in range(int(z["count"])):
        d = {}
        for k in z.files:
            if k.startswith(f"{j}."):
                v = z[k]
                d[k.split(".", 1)[1]] = v.item() if v.ndim == 0 else v
        out.append(d)
    return out
