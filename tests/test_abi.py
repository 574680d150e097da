"""C-ABI boundary checks that need no GPU: the library loads, exports exactly what
include/analogsat_b200.h declares, and its host-side logic (SatProblem semantics,
DIMACS IO, argument validation) matches the reference."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "analogsat_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(as_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_loads():
    from analogsat_b200 import build, load
    build.build()
    assert load() is not None


def test_exports_every_declared_symbol():
    from analogsat_b200 import _abi
    lib = _abi.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (as_[a-z0-9_]+)", out))
    decl = set(declared_functions())
    assert decl, "no declarations parsed"
    assert decl <= exported, sorted(decl - exported)
    assert decl == {name for name, _, _ in _abi.SIGNATURES}


def test_problem_semantics_match_satproblem(golden):
    from analogsat_b200 import SatProblem
    # zero literals filtered, empty clauses dropped, N = max |lit|, K = max length
    p = SatProblem.from_arrays([1, 0, -3, 0, 0, 2, -7, 4, 5], [3, 1, 1, 4])
    assert (p.n, p.m, p.k) == (7, 2, 4)
    lits, lens = p.GetAllClauses()
    assert list(lens) == [2, 4]
    assert list(lits) == [1, -3, 2, -7, 4, 5]
    for tag in ["p50", "mix", "k12", "p1000"]:
        q = SatProblem.from_arrays(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
        assert (q.n, q.m, q.k) == tuple(golden[f"{tag}/nmk"])
        l2, n2 = q.GetAllClauses()
        assert np.array_equal(l2, golden[f"{tag}/literals"])
        assert np.array_equal(n2, golden[f"{tag}/lengths"])


def test_cnf_read_reference_file_and_roundtrip(tmp_path, golden):
    from analogsat_b200 import SatProblem
    p = SatProblem.read_cnf(os.path.join(ROOT, "tests", "golden", "p50.cnf"))
    lits, lens = p.GetAllClauses()
    assert np.array_equal(lits, golden["p50/literals"])
    assert np.array_equal(lens, golden["p50/lengths"])
    f = str(tmp_path / "rt.cnf")
    p.write_cnf(f)
    assert open(f).read() == open(os.path.join(ROOT, "tests", "golden", "p50.cnf")).read()
    q = SatProblem.read_cnf(f)
    assert np.array_equal(q.GetAllClauses()[0], lits)


def test_cnf_reader_errors(tmp_path):
    from analogsat_b200 import SatProblem, AnalogSatError
    bad = tmp_path / "bad.cnf"
    bad.write_text("c comment\np cnf 3 2\n1 -2 0\n")
    with pytest.raises(AnalogSatError, match="expected more literals"):
        SatProblem.read_cnf(str(bad))
    nohdr = tmp_path / "nohdr.cnf"
    nohdr.write_text("c nothing here\n")
    with pytest.raises(AnalogSatError, match="SAT declaration"):
        SatProblem.read_cnf(str(nohdr))
    with pytest.raises(AnalogSatError, match="file open failed"):
        SatProblem.read_cnf(str(tmp_path / "missing.cnf"))
    empty = tmp_path / "empty.cnf"
    empty.write_text("p cnf 0 0\n")
    e = SatProblem.read_cnf(str(empty))
    assert (e.n, e.m, e.k) == (0, 0, 0)


def test_bad_arguments_return_codes():
    from analogsat_b200 import _abi
    lib = _abi.load()
    h = C.c_void_p()
    assert lib.as_problem_create(None, None, 3, C.byref(h)) == _abi.AS_ERR_BAD_INPUT
    assert "null" in _abi.last_error()
    lens = (C.c_int32 * 1)(-1)
    lits = (C.c_int32 * 1)(1)
    assert lib.as_problem_create(lits, lens, 1, C.byref(h)) == _abi.AS_ERR_BAD_INPUT
    assert lib.as_solver_create(None, 0, 0, -1, C.byref(h)) == _abi.AS_ERR_BAD_INPUT
    assert lib.as_solver_set_max_time(None, 1.0) == _abi.AS_ERR_BAD_INPUT
    assert lib.as_rhs_f32(None, None, None, 1, 0, None) == _abi.AS_ERR_BAD_INPUT


def test_empty_problem_rejected_like_reference():
    """CpuSat throws runtime_error("SAT problem has not been set") for K == 0."""
    from analogsat_b200 import SatProblem, SatSolver, AnalogSatError, _abi
    p = SatProblem.from_arrays([], [])
    with pytest.raises(AnalogSatError) as e:
        SatSolver([p])
    assert e.value.code == _abi.AS_ERR_NO_PROBLEM


def test_instances_follow_reference_distributions():
    from analogsat_b200.instances import make_instance, is_satisfied
    lits, lens, planted = make_instance("planted", 300, 1275, 3, seed=1)
    c = lits.reshape(-1, 3)
    v = np.abs(c)
    assert np.all(v[:, 0] < v[:, 1]) and np.all(v[:, 1] < v[:, 2])  # distinct, sorted
    assert len({tuple(r) for r in c}) == len(c)                      # no duplicate clauses
    assert is_satisfied(lits, lens, planted)
    l2, _, _ = make_instance("random", 300, 1275, 3, seed=1)
    assert abs((l2 > 0).mean() - 0.5) < 0.03
    l3, _, _ = make_instance("fast", 100, 4000, 4, seed=2)
    assert l3.size == 16000 and np.abs(l3).max() <= 100


def test_packing_layout_quality():
    """Degree-sorted SELL slots carry little padding and the bank-aware clause grouping
    cuts the shared-memory wavefronts of a spin-gather pass well below the natural
    order (the ideal is k * ceil(M/32))."""
    from analogsat_b200 import SatProblem, AS_PREC_F32_LOGA, AS_PREC_F64
    from analogsat_b200.instances import make_instance
    n, m, k = 1000, 4250, 3
    lits, lens, _ = make_instance("planted", n, m, k, seed=2000)
    p = SatProblem.from_arrays(lits, lens)
    ideal = k * ((m + 31) // 32)
    s32 = p.layout_stats(AS_PREC_F32_LOGA)
    s64 = p.layout_stats(AS_PREC_F64)
    assert s32["compact"] and s64["compact"]
    assert m * k <= s32["nslots"] <= 1.1 * m * k
    assert s32["bank_wavefronts"] <= 1.6 * ideal   # literal reordering allowed (FP32)
    assert s64["bank_wavefronts"] <= 2.2 * ideal   # clause regrouping only (FP64)
    from analogsat_b200._abi import AS_LAYOUT_F32_PAIR
    sp = p.layout_stats(AS_LAYOUT_F32_PAIR)      # 16-lane groups + public-clause banks
    assert sp["nslots"] == s32["nslots"]
    assert sp["bank_wavefronts"] <= 1.4 * k * ((m + 15) // 16)
    big = SatProblem.from_arrays(*make_instance("fast", 40000, 200000, 4, seed=1)[:2])
    assert not big.layout_stats()["compact"]


def test_result_messages():
    """GetSatResultMessage's strings (AnalogSAT/solver/SatResult.cpp)."""
    from analogsat_b200 import load
    lib = load()
    msgs = {0: b"solution found", 1: b"underflow", 2: b"user interrupt", 3: b"maximum time reached",
            4: b"maximum steps reached", 5: b"unknown result", 99: b"unknown result"}
    for code, msg in msgs.items():
        assert lib.as_result_message(code) == msg


def test_stream_arguments_accept_handles_and_stream_objects():
    """Stream arguments of the Python API take a raw cudaStream_t handle or any object
    with a .cuda_stream handle (a torch.cuda.Stream); both reach the C ABI as the same
    pointer value."""
    from analogsat_b200 import _stream_ptr

    class FakeStream:
        cuda_stream = 0x1234

    assert _stream_ptr(0x1234).value == 0x1234
    assert _stream_ptr(FakeStream()).value == 0x1234
