"""ctypes binding of the C ABI declared in ``include/analogsat_b200.h``.

The shared library is built in-tree (``analogsat_b200/libanalogsat_b200.so``).
There is no fallback: if the library is missing or fails to load, every call
raises, so a CPU path can never stand in for the CUDA one.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libanalogsat_b200.so")

AS_OK = 0
AS_ERR_BAD_INPUT = -1
AS_ERR_CUDA = -2
AS_ERR_NO_PROBLEM = -3
AS_ERR_UNSUPPORTED = -4
AS_ERR_IO = -5
AS_ERR_TIMEOUT = -6
AS_PREC_F32_LOGA = 0
AS_PREC_F64 = 1
AS_LAYOUT_F32_PAIR = 2  # layout_stats only
AS_KERNEL_AUTO = 0
AS_KERNEL_GENERIC = 1
AS_MODEL_CTDS = 0
AS_MODEL_TANH = 1

_vp = C.c_void_p
_i32 = C.c_int32
_pi32 = C.POINTER(C.c_int32)
_pf64 = C.POINTER(C.c_double)

# (name, restype, argtypes) for every exported symbol; tests check this list
# against the header and the library's dynamic symbol table.
SIGNATURES = [
    ("as_last_error", _i32, [C.c_char_p, _i32]),
    ("as_device_sm_count", _i32, [_i32]),
    ("as_problem_create", _i32, [_pi32, _pi32, _i32, C.POINTER(_vp)]),
    ("as_problem_read_cnf", _i32, [C.c_char_p, C.POINTER(_vp), C.c_char_p, _i32]),
    ("as_problem_read_cnf_device", _i32, [C.c_char_p, _i32, C.POINTER(_vp), C.c_char_p, _i32]),
    ("as_problem_write_cnf", _i32, [_vp, C.c_char_p]),
    ("as_problem_get_nmk", _i32, [_vp, _pi32, _pi32, _pi32]),
    ("as_problem_num_literals", _i32, [_vp]),
    ("as_problem_get_clauses", _i32, [_vp, _pi32, _pi32]),
    ("as_problem_layout_stats", _i32, [_vp, _i32, _pi32, _pi32, C.POINTER(C.c_int64), _pi32]),
    ("as_problem_set_model", _i32, [_vp, _i32, C.c_double]),
    ("as_result_message", C.c_char_p, [_i32]),
    ("as_solver_write_result", _i32, [_vp, _i32, C.c_char_p]),
    ("as_solver_append_perf", _i32, [_vp, _i32, C.c_char_p, C.c_char_p, C.c_char_p]),
    ("as_problem_set_bias", _i32, [_vp, C.c_double]),
    ("as_problem_get_model", _i32, [_vp, _pi32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("as_problem_free", None, [_vp]),
    ("as_rhs_f32", _i32, [_vp, _vp, _vp, _i32, _i32, _vp]),
    ("as_rhs_f64", _i32, [_vp, _vp, _vp, _i32, _vp]),
    ("as_rhs_check", _i32, [_vp, _vp]),
    ("as_violations_f32", _i32, [_vp, _vp, _vp, _i32, _vp]),
    ("as_violations_f64", _i32, [_vp, _vp, _vp, _i32, _vp]),
    ("as_solver_create", _i32, [C.POINTER(_vp), _i32, _i32, _i32, C.POINTER(_vp)]),
    ("as_solver_free", None, [_vp]),
    ("as_solver_set_max_time", _i32, [_vp, C.c_double]),
    ("as_solver_set_max_steps", _i32, [_vp, _i32]),
    ("as_solver_set_batch_size", _i32, [_vp, _i32]),
    ("as_solver_set_epsilon", _i32, [_vp, C.c_double]),
    ("as_solver_set_wall_budget", _i32, [_vp, C.c_double]),
    ("as_solver_set_stop_on_first", _i32, [_vp, _i32]),
    ("as_solver_set_track_best", _i32, [_vp, _i32]),
    ("as_solver_set_states_f64", _i32, [_vp, _pi32, _i32, _vp]),
    ("as_solver_set_states_f32", _i32, [_vp, _pi32, _i32, _vp]),
    ("as_solver_set_states_device", _i32, [_vp, _pi32, _i32, _vp, _vp]),
    ("as_solver_set_random_states", _i32, [_vp, _pi32, _i32, C.c_uint64, _i32, C.c_double]),
    ("as_solver_solve", _i32, [_vp]),
    ("as_solver_solve_async", _i32, [_vp, _vp]),
    ("as_solver_sync", _i32, [_vp]),
    ("as_solver_get_results", _i32, [_vp, _pi32, _pf64, _pi32, _pi32, _pi32, _pi32, _pi32, _pf64]),
    ("as_solver_get_states_f64", _i32, [_vp, _vp]),
    ("as_solver_get_states_f32", _i32, [_vp, _vp]),
    ("as_solver_get_state_f64", _i32, [_vp, _i32, _vp]),
    ("as_solver_get_state_f32", _i32, [_vp, _i32, _vp]),
    ("as_solver_states_device", _vp, [_vp]),
    ("as_solver_get_best_assignment", _i32, [_vp, _i32, _vp]),
    ("as_solver_get_launch_shape", _i32, [_vp, _pi32, _pi32, _pi32, _pi32]),
    ("as_solver_force_threads", _i32, [_vp, _i32]),
    ("as_solver_set_kernel", _i32, [_vp, _i32]),
    ("as_solver_kernel_name", C.c_char_p, [_vp]),
    ("as_solver_set_storage_mode", _i32, [_vp, _i32]),
    ("as_solver_set_cluster_size", _i32, [_vp, _i32]),
    ("as_solver_set_stream_parts", _i32, [_vp, _i32]),
    ("as_solver_solve_noalloc", _i32, [_vp, _i32, _i32, _vp, _vp, _vp]),
    ("as_solver_adjoint", _i32, [_vp, C.c_double, _i32, _vp, _vp, _vp, _vp, _vp, _vp]),
]

_lib = None


class AnalogSatError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m analogsat_b200.build` "
            "(the solver has no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().as_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(code: int) -> int:
    if code is not None and code < 0:
        raise AnalogSatError(code, last_error())
    return code
