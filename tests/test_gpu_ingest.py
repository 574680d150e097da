"""Device-side ingest: random initial states generated in HBM
(as_solver_set_random_states) and the CNF clause body tokenised on the GPU
(as_problem_read_cnf_device).

Checkers: numpy's Philox generator (instances.initial_states and the same stream
drawn trajectory by trajectory) for the states, bit for bit in FP64 and FP32; the
host CNF reader -- itself checked against the reference's CnfReader on the CPU in
test_cnf_readers.py -- for the device reader: identical clauses, N and messages on
every edge case, on mutated files whose failures fall on 4 KB tile boundaries, and on
a formatted N=1e5, M=1e6 4-SAT file.
"""
import os

import numpy as np
import pytest

from cnf_cases import CASES, formatted_cnf

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _problem(n, m, k=3, seed=1, kind="random"):
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance(kind, n, m, k, seed=seed)
    return SatProblem.from_arrays(lits, lens)


def _numpy_states(problems, pidx, seed, dist, a0, dtype):
    g = np.random.Generator(np.random.Philox(key=seed))
    out = []
    for t in pidx:
        n, m = problems[t].n, problems[t].m
        if dist == "spin_uniform":
            out += [g.uniform(-1.0, 1.0, n), np.full(m, a0)]
        else:
            u = g.random(n + m)
            out += [u[:n] * 2.0 - 1.0, u[n:] + 1.0]
    return np.concatenate(out).astype(dtype)


@pytest.mark.parametrize("precision", [0, 1])
def test_random_states_equal_initial_states(precision):
    """One problem, 37 trajectories: the device states are initial_states(...)."""
    from analogsat_b200 import SatSolver
    from analogsat_b200.instances import initial_states
    p = _problem(300, 1277)
    dt = np.float32 if precision == 0 else np.float64
    s = SatSolver([p], precision=precision)
    s.SetRandomInitialState(np.zeros(37, np.int32), seed=20260, a0=1.25)
    got = s.GetSatStates(dt).reshape(-1)
    ref = initial_states(300, 1277, 37, seed=20260, a0=1.25, dtype=dt).reshape(-1)
    assert got.dtype == ref.dtype and np.array_equal(got, ref)


@pytest.mark.parametrize("dist", ["spin_uniform", "reference"])
@pytest.mark.parametrize("precision", [0, 1])
def test_random_states_mixed_problems(dist, precision):
    """Three problem sizes in one request (draw runs of N or N+M values that do not
    align with Philox's 4-value blocks), both distributions."""
    from analogsat_b200 import SatSolver
    probs = [_problem(50, 213, seed=2), _problem(7, 30, seed=3), _problem(1001, 4250, seed=4)]
    pidx = np.array([0, 1, 2, 1, 1, 0, 2, 2, 1, 0, 1], np.int32)
    dt = np.float32 if precision == 0 else np.float64
    s = SatSolver(probs, precision=precision)
    s.SetRandomInitialState(pidx, seed=7, distribution=dist, a0=1.0)
    got = s.GetSatStates(dt).reshape(-1)
    assert np.array_equal(got, _numpy_states(probs, pidx, 7, dist, 1.0, dt))


def test_random_states_full_batch_and_solve():
    """The 64-instance x 256-trajectory FP32 batch of N=1000, M=4250 (344 MB of
    state): equal to numpy for every trajectory; then a solve from device-generated
    states matches a solve from the same states copied from the host, bit for bit."""
    from analogsat_b200 import SatSolver
    from analogsat_b200.instances import initial_states
    probs = [_problem(1000, 4250, seed=100 + i, kind="planted") for i in range(64)]
    pidx = np.repeat(np.arange(64, dtype=np.int32), 256)
    s = SatSolver(probs, precision=0)
    s.SetRandomInitialState(pidx, seed=99)
    got = s.GetSatStates(np.float32).reshape(64 * 256, 5250)
    ref = initial_states(1000, 4250, 64 * 256, seed=99, dtype=np.float32)
    assert np.array_equal(got, ref)
    sub = pidx[:512]
    for use_device in (True, False):
        t = SatSolver(probs, precision=0)
        t.SetEpsilon(1e-6); t.SetBatchSize(50); t.SetMaxSteps(400)
        if use_device:
            t.SetRandomInitialState(sub, seed=99)
        else:
            t.SetSatStates(sub, ref[:512])
        t.Solve()
        r = (t.results(), t.GetSatStates(np.float32))
        if use_device:
            first = r
    for key in first[0]:
        assert np.array_equal(first[0][key], r[0][key]), key
    assert np.array_equal(first[1], r[1])


def test_random_states_errors():
    from analogsat_b200 import SatSolver, AnalogSatError
    s = SatSolver([_problem(20, 80)], precision=1)
    with pytest.raises(AnalogSatError):
        s.SetRandomInitialState([0, 1], seed=1)        # problem index out of range
    with pytest.raises(AnalogSatError):
        s.SetRandomInitialState([0], seed=1, a0=0.0)   # a must start positive
    with pytest.raises(KeyError):
        s.SetRandomInitialState([0], seed=1, distribution="gaussian")


def _read(path, device):
    from analogsat_b200 import SatProblem, AnalogSatError
    try:
        p = SatProblem.read_cnf(path, device=device)
    except AnalogSatError as e:
        return f"{e.code} {str(e).split(': ')[-1]}"
    lits, lens = p.GetAllClauses()
    return lits, lens, p.n, p.m, p.k


def _same(a, b):
    if isinstance(a, str) or isinstance(b, str):
        assert a == b, (a, b)
        return
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def _write(tmp_path, data, name="x.cnf"):
    f = str(tmp_path / name)
    with open(f, "wb") as fh:
        fh.write(data)
    return f


@pytest.mark.parametrize("name,data,expected,ref_agrees", CASES, ids=[c[0] for c in CASES])
def test_device_reader_cases(tmp_path, name, data, expected, ref_agrees):
    f = _write(tmp_path, data)
    host, dev = _read(f, None), _read(f, 0)
    _same(host, dev)
    assert isinstance(dev, str) == (expected != "ok")


def test_device_reader_golden_file(golden):
    got = _read(os.path.join(ROOT, "tests", "golden", "p50.cnf"), 0)
    assert np.array_equal(got[0], golden["p50/literals"])
    assert np.array_equal(got[1], golden["p50/lengths"])


def test_device_reader_mutations(tmp_path):
    """300 mutated copies of a formatted 3,000-clause file (bytes replaced, inserted
    or cut, some of them on 4 KB tile boundaries of the body): device and host readers
    agree on every one, success or failure."""
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance("random", 800, 3000, 3, seed=6)
    base = formatted_cnf(lits, lens, seed=2)
    start = base.index(b"\n", base.index(b"p cnf"))  # the device body starts right after M
    body0 = start + 1
    alphabet = b"0123456789-+ \n\t\r\x0bx%c\x00"
    rng = np.random.default_rng(11)
    outcomes = set()
    for i in range(300):
        data = bytearray(base)
        for _ in range(int(rng.integers(1, 4))):
            if i % 3 == 0:  # on a tile boundary of the body
                pos = start + 4096 * int(rng.integers(1, (len(data) - start) // 4096 + 1)) + int(rng.integers(-2, 2))
            else:
                pos = int(rng.integers(body0, len(data)))
            pos = min(max(pos, body0), len(data) - 1)
            op = rng.integers(3)
            ch = alphabet[int(rng.integers(len(alphabet)))]
            if op == 0:
                data[pos] = ch
            elif op == 1:
                data.insert(pos, ch)
            else:
                del data[pos:pos + int(rng.integers(1, 6))]
        if i % 50 == 49:
            data = data[: int(rng.integers(body0, len(data)))]  # truncated file
        f = _write(tmp_path, bytes(data), f"m{i}.cnf")
        host, dev = _read(f, None), _read(f, 0)
        _same(host, dev)
        outcomes.add(host.split(" ", 1)[1] if isinstance(host, str) else "ok")
    assert {"ok", "expected more literals in file"} <= outcomes


def test_device_reader_large_formatted_instance(tmp_path):
    """FastSatMaker-style 4-SAT, N=1e5, M=1e6, written with varied formatting
    (about 30 MB): the clauses come back exactly."""
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance("fast", 100000, 1000000, 4, seed=5)
    f = _write(tmp_path, formatted_cnf(lits, lens, seed=3))
    got = _read(f, 0)
    assert np.array_equal(got[0], lits) and np.array_equal(got[1], lens)
    assert (got[2], got[3], got[4]) == (int(np.abs(lits).max()), 1000000, 4)
