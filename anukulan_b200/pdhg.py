"""Host-side mirror of the reference's PDHG interface over the CUDA engine.

``solve_pdhg(lp, options)`` is ``anukulan::solve_pdhg``
(src/anukulan/pdhg.hpp:543): same options (``PdhgOptions`` field names, see
:func:`anukulan_b200.abi.make_options`), same result fields, same status
values. Every call goes through ``libanu_pdhg.so``; there is no CPU path, and
a missing library or device raises instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from .abi import (OPTIMAL, PRIMAL_INFEASIBLE, CLp, PdhgResult, Residual, anu_csr, anu_lp,
                  anu_pdhg_options, anu_pdhg_residual, anu_pdhg_result, f64_ptr, make_options)
from .model import StandardLp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libanu_pdhg.so")

_P = C.POINTER
_lib = None

# Every function the C ABI declares (include/anu_pdhg.h).
EXPORTS = (
    "anu_pdhg_version", "anu_pdhg_default_options", "anu_last_error", "anu_device_count",
    "anu_release_cached_memory",
    "anu_pdhg_solve", "anu_pdhg_create", "anu_pdhg_run", "anu_pdhg_set_case", "anu_pdhg_destroy",
    "anu_evaluate_residual", "anu_estimate_matrix_norm", "anu_locality_relabel",
    "anu_backend_allocate", "anu_backend_deallocate", "anu_backend_upload",
    "anu_backend_download", "anu_backend_fill", "anu_backend_copy", "anu_backend_prepare",
    "anu_backend_release", "anu_backend_multiply", "anu_backend_dot", "anu_backend_two_norm",
    "anu_backend_inf_norm", "anu_backend_primal_update", "anu_backend_dual_update",
    "anu_backend_accumulate", "anu_backend_scale_into", "anu_backend_weighted_norm_squared",
    "anu_backend_step_size_terms", "anu_backend_convergence_terms",
    "anu_backend_convergence_terms_noalloc", "anu_backend_set_profiling",
    "anu_backend_profile_report",
    "anu_pdhg_batch_create", "anu_pdhg_batch_solve", "anu_pdhg_batch_solve_warm",
    "anu_pdhg_batch_destroy", "anu_pdhg_batch_stream",
    "anu_pdhg_packed_create", "anu_pdhg_packed_solve", "anu_pdhg_packed_workers",
    "anu_pdhg_packed_destroy",
    "anu_pdhg_unrolled_create", "anu_pdhg_unrolled_step_sizes", "anu_pdhg_forward_unrolled",
    "anu_pdhg_backward", "anu_pdhg_unrolled_destroy",
)


class EngineError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"anu_pdhg error {code}: {message}")
        self.code = code


def lib():
    """Loads libanu_pdhg.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `python -m anukulan_b200.build`")
    L = C.CDLL(LIB_PATH)

    def d(name, res, args):
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args

    d("anu_pdhg_version", C.c_char_p, [])
    d("anu_pdhg_default_options", None, [_P(anu_pdhg_options)])
    d("anu_last_error", C.c_int, [C.c_char_p, C.c_int32])
    d("anu_device_count", C.c_int32, [])
    d("anu_release_cached_memory", C.c_int64, [])
    d("anu_pdhg_solve", C.c_int, [_P(anu_lp), _P(anu_pdhg_options), _P(C.c_double),
                                  _P(C.c_double), _P(C.c_double), _P(C.c_double),
                                  _P(anu_pdhg_result)])
    d("anu_pdhg_create", C.c_int, [_P(anu_lp), _P(anu_pdhg_options), _P(C.c_void_p)])
    d("anu_pdhg_run", C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double), _P(C.c_double),
                                _P(C.c_double), _P(anu_pdhg_result)])
    d("anu_pdhg_set_case", C.c_int, [C.c_void_p] + [_P(C.c_double)] * 4)
    d("anu_pdhg_destroy", None, [C.c_void_p])
    d("anu_evaluate_residual", C.c_int, [_P(anu_lp), _P(C.c_double), _P(C.c_double),
                                         _P(anu_pdhg_residual)])
    d("anu_estimate_matrix_norm", C.c_int, [_P(anu_lp), C.c_int32, C.c_double,
                                            _P(C.c_double)])
    d("anu_pdhg_batch_create", C.c_int, [_P(anu_lp), C.c_int32, _P(C.c_double),
                                         _P(C.c_double), _P(C.c_double), _P(C.c_double),
                                         _P(anu_pdhg_options), _P(C.c_void_p)])
    d("anu_pdhg_batch_solve", C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double),
                                        _P(anu_pdhg_result)])
    d("anu_pdhg_batch_solve_warm", C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double),
                                             _P(C.c_double), _P(C.c_double),
                                             _P(anu_pdhg_result)])
    d("anu_pdhg_batch_destroy", None, [C.c_void_p])
    d("anu_locality_relabel", C.c_int, [_P(anu_lp), _P(C.c_int32), _P(C.c_int32)])
    d("anu_pdhg_batch_stream", C.c_int, [C.c_void_p, C.c_int32, CASE_SOURCE, CASE_SINK,
                                         C.c_void_p])
    d("anu_pdhg_packed_create", C.c_int, [C.c_int32, _P(anu_lp), _P(anu_pdhg_options),
                                          C.c_int32, _P(C.c_void_p)])
    d("anu_pdhg_packed_solve", C.c_int, [C.c_void_p, _P(_P(C.c_double)), _P(_P(C.c_double)),
                                         _P(anu_pdhg_result)])
    d("anu_pdhg_packed_workers", C.c_int32, [C.c_void_p])
    d("anu_pdhg_packed_destroy", None, [C.c_void_p])
    d("anu_pdhg_unrolled_create", C.c_int, [_P(anu_lp), C.c_int32] + [_P(C.c_double)] * 4
      + [_P(anu_pdhg_options), C.c_int32, C.c_int32, _P(C.c_void_p)])
    d("anu_pdhg_unrolled_step_sizes", C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double)])
    d("anu_pdhg_forward_unrolled", C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double)])
    d("anu_pdhg_backward", C.c_int, [C.c_void_p] + [_P(C.c_double)] * 4)
    d("anu_pdhg_unrolled_destroy", None, [C.c_void_p])
    vp = C.c_void_p
    i64 = C.c_int64
    dbl = C.c_double
    d("anu_backend_allocate", C.c_int, [i64, _P(vp)])
    d("anu_backend_deallocate", C.c_int, [vp])
    d("anu_backend_upload", C.c_int, [_P(dbl), vp, i64])
    d("anu_backend_download", C.c_int, [vp, _P(dbl), i64])
    d("anu_backend_fill", C.c_int, [vp, i64, dbl])
    d("anu_backend_copy", C.c_int, [vp, vp, i64])
    d("anu_backend_prepare", C.c_int, [C.c_uint64, _P(anu_csr)])
    d("anu_backend_release", C.c_int, [])
    d("anu_backend_multiply", C.c_int, [C.c_uint64, vp, vp])
    d("anu_backend_dot", C.c_int, [vp, vp, i64, _P(dbl)])
    d("anu_backend_two_norm", C.c_int, [vp, i64, _P(dbl)])
    d("anu_backend_inf_norm", C.c_int, [vp, i64, _P(dbl)])
    d("anu_backend_primal_update", C.c_int, [i64, dbl, dbl, dbl] + [vp] * 9)
    d("anu_backend_dual_update", C.c_int, [i64, i64, dbl, dbl, dbl] + [vp] * 10)
    d("anu_backend_accumulate", C.c_int, [i64, dbl, vp, vp])
    d("anu_backend_scale_into", C.c_int, [i64, dbl, vp, vp])
    d("anu_backend_weighted_norm_squared", C.c_int, [i64, i64, vp, vp, dbl, _P(dbl)])
    d("anu_backend_step_size_terms", C.c_int, [i64, i64, vp, vp, vp, dbl, _P(dbl), _P(dbl)])
    d("anu_backend_convergence_terms", C.c_int, [i64, i64] + [vp] * 6 + [i64] + [vp] * 4
      + [_P(dbl)])
    d("anu_backend_convergence_terms_noalloc", C.c_int,
      [i64, i64] + [vp] * 6 + [i64] + [vp] * 4 + [_P(dbl)])
    d("anu_backend_set_profiling", C.c_int, [C.c_int32])
    d("anu_backend_profile_report", C.c_int, [C.c_char_p, C.c_int32, _P(C.c_int32)])
    _lib = L
    return L


def backend_set_profiling(on: bool) -> None:
    """LinAlgBackend::set_profiling on the seam (backend.hpp:213)."""
    check(lib().anu_backend_set_profiling(1 if on else 0))


def backend_profile_report() -> str:
    """LinAlgBackend::profile_report of the seam (backend.hpp:214)."""
    n = C.c_int32(0)
    check(lib().anu_backend_profile_report(None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(lib().anu_backend_profile_report(buf, n.value + 1, C.byref(n)))
    return buf.value.decode()


def check(rc: int) -> None:
    if rc != 0:
        buf = C.create_string_buffer(512)
        lib().anu_last_error(buf, 512)
        raise EngineError(rc, buf.value.decode(errors="replace"))


def version() -> str:
    return lib().anu_pdhg_version().decode()


def device_count() -> int:
    return int(lib().anu_device_count())


def release_cached_memory() -> int:
    """Frees the blocks destroyed solvers left cached for reuse; the bytes
    freed."""
    return int(lib().anu_release_cached_memory())


def default_options() -> anu_pdhg_options:
    o = anu_pdhg_options()
    lib().anu_pdhg_default_options(C.byref(o))
    return o


def _options(options: Optional[anu_pdhg_options], kw) -> anu_pdhg_options:
    if options is None:
        return make_options(**kw)
    if kw:
        o = anu_pdhg_options()
        C.memmove(C.byref(o), C.byref(options), C.sizeof(o))
        for k, v in kw.items():
            setattr(o, k, int(v) if isinstance(v, bool) else v)
        return o
    return options


def locality_relabel(lp: StandardLp):
    """``anu_locality_relabel``: (row_old, col_old), the relabelling that
    options.locality_order applies (new -> original). Host only."""
    cl = CLp(lp)
    row_old = np.zeros(max(cl.m, 1), np.int32)
    col_old = np.zeros(max(cl.n, 1), np.int32)
    check(lib().anu_locality_relabel(cl.ref(), row_old.ctypes.data_as(C.POINTER(C.c_int32)),
                                     col_old.ctypes.data_as(C.POINTER(C.c_int32))))
    return row_old[:cl.m].copy(), col_old[:cl.n].copy()


def solve_pdhg(lp: StandardLp, options: Optional[anu_pdhg_options] = None,
               warm_x=None, warm_y=None, **kw) -> PdhgResult:
    """``solve_pdhg`` on the B200 engine (pdhg.hpp:543)."""
    cl = CLp(lp)
    o = _options(options, kw)
    x = np.zeros(cl.n)
    y = np.zeros(cl.m)
    r = anu_pdhg_result()
    wx = None if warm_x is None else np.ascontiguousarray(warm_x, np.float64)
    wy = None if warm_y is None else np.ascontiguousarray(warm_y, np.float64)
    check(lib().anu_pdhg_solve(cl.ref(), C.byref(o), f64_ptr(wx), f64_ptr(wy), f64_ptr(x),
                               f64_ptr(y), C.byref(r)))
    return PdhgResult.from_c(r, x, y)


class PdhgHandle:
    """A prepared LP (scaled, uploaded, ||K|| measured) that can be solved
    repeatedly: ``anu_pdhg_create`` / ``anu_pdhg_run``."""

    def __init__(self, lp: StandardLp, options: Optional[anu_pdhg_options] = None, **kw):
        self._cl = CLp(lp)
        self.options = _options(options, kw)
        self._h = C.c_void_p()
        check(lib().anu_pdhg_create(self._cl.ref(), C.byref(self.options), C.byref(self._h)))

    def run(self, warm_x=None, warm_y=None, x=None, y=None) -> PdhgResult:
        x = np.zeros(self._cl.n) if x is None else x
        y = np.zeros(self._cl.m) if y is None else y
        r = anu_pdhg_result()
        wx = None if warm_x is None else np.ascontiguousarray(warm_x, np.float64)
        wy = None if warm_y is None else np.ascontiguousarray(warm_y, np.float64)
        check(lib().anu_pdhg_run(self._h, f64_ptr(wx), f64_ptr(wy), f64_ptr(x), f64_ptr(y),
                                 C.byref(r)))
        return PdhgResult.from_c(r, x, y)

    def set_case(self, c=None, q=None, lower=None, upper=None) -> None:
        """``anu_pdhg_set_case``: another LP with the same matrix (None keeps
        a vector); the scaled matrix and ||K|| are kept."""
        keep = [None if v is None else np.ascontiguousarray(v, np.float64)
                for v in (c, q, lower, upper)]
        for v, size in zip(keep, (self._cl.n, self._cl.m, self._cl.n, self._cl.n)):
            if v is not None and v.shape != (size,):
                raise ValueError("case vector of the wrong length")
        check(lib().anu_pdhg_set_case(self._h, *[f64_ptr(v) for v in keep]))

    def close(self):
        if self._h:
            lib().anu_pdhg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def evaluate_residual(lp: StandardLp, x, y) -> Residual:
    """``evaluate_residual`` (pdhg.hpp:548) computed on the device."""
    cl = CLp(lp)
    out = anu_pdhg_residual()
    check(lib().anu_evaluate_residual(cl.ref(), f64_ptr(np.ascontiguousarray(x, np.float64)),
                                      f64_ptr(np.ascontiguousarray(y, np.float64)),
                                      C.byref(out)))
    return Residual.from_c(out)


def estimate_matrix_norm(lp: StandardLp, iterations: int = 200, tolerance: float = 1e-8) -> float:
    """``estimate_matrix_norm`` (pdhg.hpp:580) on the device."""
    out = C.c_double(0.0)
    check(lib().anu_estimate_matrix_norm(CLp(lp).ref(), iterations, tolerance, C.byref(out)))
    return out.value


# anu_pdhg_case_source / anu_pdhg_case_sink.
CASE_SOURCE = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double))
CASE_SINK = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                        C.POINTER(C.c_double), C.POINTER(anu_pdhg_result))


class CaseStackSolver:
    """A case stack sharing one matrix (``anu_pdhg_batch_*``)."""

    def __init__(self, base: StandardLp, c=None, q=None, lower=None, upper=None,
                 options: Optional[anu_pdhg_options] = None, **kw):
        arrays = [c, q, lower, upper]
        counts = {np.asarray(a).shape[0] for a in arrays if a is not None}
        if len(counts) != 1:
            raise ValueError("case arrays must share their first dimension")
        self.num_cases = counts.pop()
        self._keep = [None if a is None else np.ascontiguousarray(a, np.float64) for a in arrays]
        self._cl = CLp(base)
        self.options = _options(options, kw)
        self._h = C.c_void_p()
        check(lib().anu_pdhg_batch_create(self._cl.ref(), self.num_cases,
                                          *[f64_ptr(a) for a in self._keep],
                                          C.byref(self.options), C.byref(self._h)))

    def solve(self, warm_x=None, warm_y=None):
        """Returns a list of PdhgResult, one per case. warm_x (K x n) and
        warm_y (K x m) warm start every case, as solve_pdhg's warm start."""
        K, n, m = self.num_cases, self._cl.n, self._cl.m
        x = np.zeros((K, n))
        y = np.zeros((K, m))
        res = (anu_pdhg_result * K)()
        if warm_x is None or warm_y is None:
            check(lib().anu_pdhg_batch_solve(self._h, f64_ptr(x), f64_ptr(y), res))
        else:
            wx = np.ascontiguousarray(warm_x, np.float64).reshape(K, n)
            wy = np.ascontiguousarray(warm_y, np.float64).reshape(K, m)
            check(lib().anu_pdhg_batch_solve_warm(self._h, f64_ptr(wx), f64_ptr(wy), f64_ptr(x),
                                                  f64_ptr(y), res))
        return [PdhgResult.from_c(res[k], x[k], y[k]) for k in range(K)]

    def stream(self, source, sink, slots: int = 64):
        """A streaming stack (``anu_pdhg_batch_stream``). `source(case)`
        fills the next case and returns its id, or returns None when it has
        none now; `case` has writable arrays c, q, lower and upper holding the
        base LP's vectors. `sink(case_id, result)` receives each result as its
        case retires, before the freed slot is refilled."""
        n, m = self._cl.n, self._cl.m
        failure = []

        class Case:
            pass

        def src(_user, case_id, c, q, lower, upper):
            try:
                case = Case()
                case.c = np.ctypeslib.as_array(c, shape=(n,))
                case.q = np.ctypeslib.as_array(q, shape=(m,))
                case.lower = np.ctypeslib.as_array(lower, shape=(n,))
                case.upper = np.ctypeslib.as_array(upper, shape=(n,))
                k = source(case)
                if k is None:
                    return 0
                case_id[0] = int(k)
                return 1
            except BaseException as e:  # no exception may cross the C boundary
                failure.append(e)
                return 0

        def snk(_user, case_id, x, y, res):
            try:
                sink(int(case_id), PdhgResult.from_c(
                    res.contents, np.ctypeslib.as_array(x, shape=(n,)).copy(),
                    np.ctypeslib.as_array(y, shape=(m,)).copy()))
            except BaseException as e:
                failure.append(e)

        cb_src, cb_snk = CASE_SOURCE(src), CASE_SINK(snk)
        check(lib().anu_pdhg_batch_stream(self._h, int(slots), cb_src, cb_snk, None))
        if failure:
            raise failure[0]

    def close(self):
        if self._h:
            lib().anu_pdhg_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NodeRelaxation:
    """One branch-and-bound node's first-order relaxation, judged as
    branch_and_bound.cpp:532-565 judges it.

    A first-order point is only nearly optimal, so its objective is no bound.
    The dual objective is one by weak duality, as long as y is dual feasible.
    The node therefore counts as solved (`optimal`) when PDHG reports optimal
    and dual_residual_inf <= 1e-7 * max(1, |dual objective|). `bound` is then
    that dual objective (standard form, a minimisation), and NaN otherwise.
    `proved_infeasible` is a primal infeasibility certificate."""

    __slots__ = ("result", "optimal", "proved_infeasible", "bound")

    def __init__(self, result: PdhgResult):
        d = result.residual.dual_objective
        enough = 1e-7 * max(1.0, abs(d))
        self.result = result
        self.optimal = result.status == OPTIMAL and result.residual.dual_residual_inf <= enough
        self.proved_infeasible = result.status == PRIMAL_INFEASIBLE
        self.bound = d if self.optimal else float("nan")


def solve_node_relaxations(lp: StandardLp, lower, upper,
                           options: Optional[anu_pdhg_options] = None, **kw):
    """Relaxations of branch-and-bound nodes as one case stack.

    The nodes differ from `lp` only in column bounds: `lower` and `upper`
    are (nodes x n). The reference solves each node with solve_pdhg
    (branch_and_bound.cpp:532-537). That call passes the parent's x alone as
    warm_x, and solve_pdhg takes a warm start only when both x and y are
    given (pdhg.cpp:481-484), so every node starts from the origin, as here.
    Returns one :class:`NodeRelaxation` per node."""
    lower = np.atleast_2d(np.asarray(lower, np.float64))
    upper = np.atleast_2d(np.asarray(upper, np.float64))
    if lower.shape != upper.shape or lower.shape[1] != lp.num_cols:
        raise ValueError("node bounds must be (nodes x columns), the same for lower and upper")
    solver = CaseStackSolver(lp, lower=lower, upper=upper, options=options, **kw)
    try:
        return [NodeRelaxation(r) for r in solver.solve()]
    finally:
        solver.close()


def solve_case_stack(stack, options: Optional[anu_pdhg_options] = None, **kw):
    """Solves an :class:`anukulan_b200.lpgen.CaseStack` on the engine."""
    s = CaseStackSolver(stack.base, stack.c, stack.q, stack.lower, stack.upper, options, **kw)
    try:
        return s.solve()
    finally:
        s.close()


class PackedBatchSolver:
    """Independent LPs of different shapes solved together
    (``anu_pdhg_packed_*``). `workers` = 0 lets the engine autotune the
    number of LPs in flight."""

    def __init__(self, lps, options: Optional[anu_pdhg_options] = None, workers: int = 0, **kw):
        self._cls = [CLp(lp) for lp in lps]
        arr = (anu_lp * len(self._cls))(*[c.struct for c in self._cls])
        self._arr = arr
        self.options = _options(options, kw)
        self._h = C.c_void_p()
        check(lib().anu_pdhg_packed_create(len(self._cls), arr, C.byref(self.options),
                                           int(workers), C.byref(self._h)))

    @property
    def workers(self) -> int:
        return int(lib().anu_pdhg_packed_workers(self._h))

    def solve(self):
        """Returns a list of PdhgResult, one per LP, in input order."""
        N = len(self._cls)
        xs = [np.zeros(c.n) for c in self._cls]
        ys = [np.zeros(c.m) for c in self._cls]
        px = (C.POINTER(C.c_double) * N)(*[f64_ptr(v) for v in xs])
        py = (C.POINTER(C.c_double) * N)(*[f64_ptr(v) for v in ys])
        res = (anu_pdhg_result * N)()
        check(lib().anu_pdhg_packed_solve(self._h, px, py, res))
        return [PdhgResult.from_c(res[i], xs[i], ys[i]) for i in range(N)]

    def close(self):
        if self._h:
            lib().anu_pdhg_packed_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_packed(lps, options: Optional[anu_pdhg_options] = None, workers: int = 0, **kw):
    """Solves independent LPs as one packed batch; one PdhgResult per LP."""
    s = PackedBatchSolver(lps, options, workers, **kw)
    try:
        return s.solve()
    finally:
        s.close()


class UnrolledPdhg:
    """Truncated, unrolled PDHG over a case stack and its adjoint
    (``anu_pdhg_unrolled_*``): forward() gives x_T, y_T; backward(dL/dx_T,
    dL/dy_T) gives dL/dc, dL/dq, all unscaled and case-major."""

    def __init__(self, base: StandardLp, c=None, q=None, lower=None, upper=None,
                 iterations: int = 2000, checkpoint_every: int = 100,
                 options: Optional[anu_pdhg_options] = None, **kw):
        arrays = [c, q, lower, upper]
        counts = {np.atleast_2d(a).shape[0] for a in arrays if a is not None}
        if len(counts) > 1:
            raise ValueError("case arrays must share their first dimension")
        self.num_cases = counts.pop() if counts else 1
        self._keep = [None if a is None else np.ascontiguousarray(np.atleast_2d(a), np.float64)
                      for a in arrays]
        self._cl = CLp(base)
        self.options = _options(options, kw)
        self._h = C.c_void_p()
        check(lib().anu_pdhg_unrolled_create(self._cl.ref(), self.num_cases,
                                             *[f64_ptr(a) for a in self._keep],
                                             C.byref(self.options), int(iterations),
                                             int(checkpoint_every), C.byref(self._h)))

    def step_sizes(self):
        tau = np.zeros(self.num_cases)
        sigma = np.zeros(self.num_cases)
        check(lib().anu_pdhg_unrolled_step_sizes(self._h, f64_ptr(tau), f64_ptr(sigma)))
        return tau, sigma

    def forward(self):
        K, n, m = self.num_cases, self._cl.n, self._cl.m
        x = np.zeros((K, n))
        y = np.zeros((K, m))
        check(lib().anu_pdhg_forward_unrolled(self._h, f64_ptr(x), f64_ptr(y)))
        return x, y

    def backward(self, dloss_dx, dloss_dy=None):
        K, n, m = self.num_cases, self._cl.n, self._cl.m
        dx = np.ascontiguousarray(np.broadcast_to(dloss_dx, (K, n)), np.float64)
        dy = None if dloss_dy is None else np.ascontiguousarray(
            np.broadcast_to(dloss_dy, (K, m)), np.float64)
        gc = np.zeros((K, n))
        gq = np.zeros((K, m))
        check(lib().anu_pdhg_backward(self._h, f64_ptr(dx), f64_ptr(dy), f64_ptr(gc),
                                      f64_ptr(gq)))
        return gc, gq

    def close(self):
        if self._h:
            lib().anu_pdhg_unrolled_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
