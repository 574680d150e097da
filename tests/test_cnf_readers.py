"""The host CNF reader (as_problem_read_cnf) on edge-case DIMACS inputs, against the
reference's own CnfReader (compiled from its sources into oracle/_ref) where it is
built: same clauses on success, a failure where it fails.  The device reader is
checked against this host reader in test_gpu_ingest.py.
"""
import os
import re

import numpy as np
import pytest

from cnf_cases import CASES, formatted_cnf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libanalogsat_ref.so")


def _reference():
    if not os.path.exists(REF_SO):
        return None
    from oracle import Reference
    return Reference()


def read_host(path):
    """(literals, lengths, n) or the failure message."""
    from analogsat_b200 import SatProblem, AnalogSatError
    try:
        p = SatProblem.read_cnf(path)
    except AnalogSatError as e:
        return str(e)
    lits, lens = p.GetAllClauses()
    return lits, lens, p.n


@pytest.mark.parametrize("name,data,expected,ref_agrees", CASES, ids=[c[0] for c in CASES])
def test_host_reader_cases(tmp_path, name, data, expected, ref_agrees):
    f = str(tmp_path / f"{name}.cnf")
    with open(f, "wb") as fh:
        fh.write(data)
    got = read_host(f)
    if expected != "ok":
        assert isinstance(got, str) and re.search(re.escape(expected), got), got
    else:
        assert not isinstance(got, str), got
    R = _reference()
    if R is None or not ref_agrees:
        return
    try:
        rp = R.read_cnf(f)
    except ValueError:
        assert isinstance(got, str)
        return
    assert not isinstance(got, str), got
    rl, rn = rp.export()
    assert np.array_equal(got[0], rl) and np.array_equal(got[1], rn)
    assert got[2] == rp.n


def test_host_reader_deliberate_differences(tmp_path):
    """Where the reference differs by design: a blank preamble line does not swallow
    the declaration after it, and out-of-range literals fail instead of wrapping."""
    got = read_host(_write(tmp_path, b"c a\n\np cnf 3 1\n1 0\n"))
    assert np.array_equal(got[0], [1]) and np.array_equal(got[1], [1])
    assert "out of range" in read_host(_write(tmp_path, b"p cnf 3 1\n1 2147483648 0\n"))


def _write(tmp_path, data, name="d.cnf"):
    f = str(tmp_path / name)
    with open(f, "wb") as fh:
        fh.write(data)
    return f


def test_host_reader_formatted_instance(tmp_path):
    """20,000 clauses with varied formatting: the clauses come back exactly, and the
    reference's reader agrees."""
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance("random", 5000, 20000, 3, seed=3)
    f = _write(tmp_path, formatted_cnf(lits, lens, seed=1))
    got = read_host(f)
    assert np.array_equal(got[0], lits) and np.array_equal(got[1], lens)
    R = _reference()
    if R is not None:
        rl, rn = R.read_cnf(f).export()
        assert np.array_equal(rl, lits) and np.array_equal(rn, lens)


def test_philox_stream_matches_numpy():
    """The documented random-state stream (Philox4x64-10 keyed by (seed, 0), draw d =
    output d%4 of the block with counter d/4 + 1, u = (x >> 11) * 2^-53), restated here
    in Python integers, is numpy's Generator(Philox(key=seed)): the device generator
    is checked against numpy, so this pins what numpy computes to that statement."""
    M0, M1 = 0xD2E7470EE14C6C93, 0xCA5A826395121157
    W0, W1 = 0x9E3779B97F4A7C15, 0xBB67AE8584CAA73B
    mask = (1 << 64) - 1

    def block(c0, k0):
        x, k1 = [c0, 0, 0, 0], 0
        for _ in range(10):
            p0, p1 = M0 * x[0], M1 * x[2]
            x = [(p1 >> 64) ^ x[1] ^ k0, p1 & mask, (p0 >> 64) ^ x[3] ^ k1, p0 & mask]
            k0, k1 = (k0 + W0) & mask, (k1 + W1) & mask
        return x

    for seed in (0, 1, 12345, 2 ** 63 + 7):
        raw = [v for b in range(1, 65) for v in block(b, seed)]
        u = np.array([(x >> 11) * 2.0 ** -53 for x in raw])
        g = np.random.Generator(np.random.Philox(key=seed))
        assert np.array_equal(g.random(256), u)
        g = np.random.Generator(np.random.Philox(key=seed))
        assert np.array_equal(g.uniform(-1.0, 1.0, 256), u * 2.0 - 1.0)


def test_writer_matches_reference_writer_byte_for_byte(tmp_path):
    """as_problem_write_cnf against the reference's CnfWriter: identical files, for a
    3-SAT, a mixed-length and a k = 12 instance (negative literals, unused variables)."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance
    R = _reference()
    if R is None:
        pytest.skip("reference checker not built here")
    for kind, n, m, k, seed in [("random", 300, 1200, 3, 2), ("fast", 50, 40, 12, 1)]:
        lits, lens, _ = make_instance(kind, n, m, k, seed=seed)
        ours, ref = str(tmp_path / "ours.cnf"), str(tmp_path / "ref.cnf")
        SatProblem.from_arrays(lits, lens).write_cnf(ours)
        R.write_cnf(R.problem(lits, lens), ref)
        assert open(ours, "rb").read() == open(ref, "rb").read()
    clauses = [[1], [-2, 3], [4, -5, 6], [-1, 2, -3, 4, 5], [9, -9]]
    lits = np.array([l for c in clauses for l in c], np.int32)
    lens = np.array([len(c) for c in clauses], np.int32)
    ours, ref = str(tmp_path / "ours.cnf"), str(tmp_path / "ref.cnf")
    SatProblem.from_arrays(lits, lens).write_cnf(ours)
    R.write_cnf(R.problem(lits, lens), ref)
    assert open(ours, "rb").read() == open(ref, "rb").read()
