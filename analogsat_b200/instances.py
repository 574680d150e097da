"""Synthetic CNF instances and initial conditions with the reference generators'
distributions (seeded numpy; used by the tests, bench.py and examples).

* random   -- RandomSatMaker (AnalogSAT/problem/RandomSatMaker.cpp:74-125): each clause
  draws K distinct variables uniformly from 1..N (sorted), signs +-1 with p = 0.5,
  duplicate clauses are redrawn.
* planted  -- PlantedSatMaker (AnalogSAT/problem/PlantedSatMaker.cpp:50-78): as random,
  plus a hidden uniform assignment; clauses it violates are redrawn.
* fast     -- FastSatMaker (AnalogSAT/problem/FastSatMaker.cpp:59-81): no duplicate check.

The reference makers use std::default_random_engine, whose stream is
implementation-defined, so instances are exchanged as literal arrays (or CNF files),
never regenerated from a seed on the other side.
"""
from __future__ import annotations

import numpy as np


def make_instance(kind: str, n: int, m: int, k: int, seed: int):
    """Returns (literals int32[m*k], lengths int32[m], planted bool[n] or None)."""
    rng = np.random.default_rng(seed)
    planted = rng.random(n) < 0.5 if kind == "planted" else None
    unique = kind in ("random", "planted")
    out = np.zeros((0, k), np.int64)
    while out.shape[0] < m:
        need = m - out.shape[0]
        B = max(64, int(need * 1.5) + 16)
        v = np.sort(rng.integers(1, n + 1, size=(B, k)), axis=1)
        ok = np.all(v[:, 1:] != v[:, :-1], axis=1) if k > 1 else np.ones(B, bool)
        v = v[ok]
        sgn = np.where(rng.random(v.shape) < 0.5, 1, -1)
        lits = v * sgn
        if planted is not None:
            truth = planted[v - 1]
            sat = np.any(np.where(lits > 0, truth, ~truth), axis=1)
            lits = lits[sat]
        if unique:
            # keep the first occurrence of every clause, in draw order, across draws
            allc = np.concatenate([out, lits])
            _, first = np.unique(allc, axis=0, return_index=True)
            keep = np.zeros(len(allc), bool)
            keep[first] = True
            lits = allc[len(out):][keep[len(out):]]
        out = np.concatenate([out, lits[:need]])
    return (out.reshape(-1).astype(np.int32), np.full(m, k, np.int32), planted)


def initial_states(n: int, m: int, count: int, seed: int, a0: float = 1.0, dtype=np.float64):
    """count public states [s_1..s_N, a_1..a_M]: s ~ U(-1, 1), a = a0 (counter-based
    Philox keyed by seed, so trajectory t of a seed is reproducible on its own)."""
    g = np.random.Generator(np.random.Philox(key=seed))
    s = g.uniform(-1.0, 1.0, size=(count, n))
    a = np.full((count, m), a0)
    return np.ascontiguousarray(np.concatenate([s, a], axis=1).astype(dtype))


def is_satisfied(literals, lengths, assignment) -> bool:
    """Exact check of a Boolean assignment (assignment[i] = variable i+1 TRUE)."""
    lits = np.asarray(literals)
    v = np.abs(lits) - 1
    t = np.where(lits > 0, assignment[v], ~assignment[v])
    idx = np.repeat(np.arange(len(lengths)), lengths)
    sat = np.zeros(len(lengths), bool)
    np.logical_or.at(sat, idx, t)
    return bool(sat.all())
