"""The compact whole-step fixtures at the measured workloads' sizes
(tests/golden/big_<name>.npz, written by tests/golden/make_golden.py --big):
the 224^2 spinodal film and the 512^2 all-physics film.

A fixture keeps what the reference's whole-step probe reported -- its header
values, sha256 hashes of the start fields and of the CRS patterns, and the
film (and concentration) after the reference's own time loop ran the case's
steps -- and rebuilds the start state with the seeded builder of
yuzen_b200.cases, which the hashes pin to the reference's own set-up."""
from __future__ import annotations

import ast
import hashlib
from pathlib import Path

import numpy as np

import stateio
from yuzen_b200 import cases

GOLDEN = Path(__file__).resolve().parent / "golden"
BIG = sorted(GOLDEN.glob("big_*.npz"))


def field_hash(a) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()).hexdigest()


def load(path) -> tuple[dict, dict]:
    """(fixture, state): the fixture's contents and the builder's state of
    the same case (params and start fields, as yuzen_b200.cases gives them)."""
    d = stateio.load_npz(path)
    kw = ast.literal_eval(str(d["builder_kw"]))
    case = getattr(cases, str(d["builder"]))(**kw)
    return d, case.state()
