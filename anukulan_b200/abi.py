"""ctypes mirror of include/anu_pdhg.h: the option, result and problem structs
of the C ABI, and the conversion of a :class:`StandardLp` into an ``anu_lp``.

The same structs drive the CUDA engine (``libanu_pdhg.so``) and the CPU
checkers, so one options object means the same solve everywhere.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields
from typing import Any, List

import numpy as np

from .model import StandardLp

i32 = C.c_int32
f64 = C.c_double

ANU_OK = 0
STATUS_NAMES = {0: "optimal", 1: "primal infeasible", 2: "iteration limit",
                3: "time limit", 4: "numerical error"}
OPTIMAL, PRIMAL_INFEASIBLE, ITERATION_LIMIT, TIME_LIMIT, NUMERICAL_ERROR = range(5)
TERMINATION_FULL, TERMINATION_PRIMAL, TERMINATION_DUAL = range(3)
PRECISION_FP64, PRECISION_FP32 = 0, 1


class anu_csr(C.Structure):
    _fields_ = [("rows", i32), ("cols", i32), ("nnz", i32),
                ("start", C.POINTER(i32)), ("index", C.POINTER(i32)),
                ("value", C.POINTER(f64))]


class anu_lp(C.Structure):
    _fields_ = [("k", anu_csr), ("c", C.POINTER(f64)), ("q", C.POINTER(f64)),
                ("lower", C.POINTER(f64)), ("upper", C.POINTER(f64)),
                ("num_equalities", i32), ("objective_scale", f64),
                ("objective_offset", f64)]


class anu_pdhg_options(C.Structure):
    _fields_ = [
        ("tolerance", f64), ("gap_tolerance", f64), ("max_iterations", i32),
        ("time_limit_seconds", f64), ("termination_check_frequency", i32),
        ("absolute_tolerance", f64), ("require_inf_norm_termination", i32),
        ("adaptive_step_size", i32), ("primal_weight_updates", i32),
        ("restarts", i32), ("halpern", i32), ("halpern_restart", i32),
        ("halpern_minimum_epoch", i32), ("polish_feasibility", i32),
        ("polish_first_iteration", i32), ("polish_iteration_factor", f64),
        ("polish_minimum_iterations", i32), ("polish_maximum_iterations", i32),
        ("polish_on_exit", i32), ("reflection", f64), ("constant_step_size", i32),
        ("constant_step_scale", f64), ("restart_on_fixed_point", i32),
        ("pid_primal_weight", i32), ("primal_weight_kp", f64),
        ("primal_weight_ki", f64), ("primal_weight_kd", f64),
        ("ruiz_iterations", i32), ("pock_chambolle", i32), ("reuse_products", i32),
        ("detect_infeasibility", i32), ("infeasibility_tolerance", f64),
        ("termination", i32), ("known_matrix_norm", f64), ("initial_step_size", f64),
        ("initial_primal_weight", f64), ("verbose", i32), ("log_frequency", i32),
        ("stop", C.POINTER(C.c_uint8)),
        ("precision", i32), ("refinement", i32), ("device", i32), ("use_graphs", i32),
        ("profile", i32), ("split_stacks", i32), ("persistent_chunks", i32),
        ("locality_order", i32), ("scaling_on_device", i32), ("tile_threads", i32),
        ("cluster_chunks", i32),
    ]


class anu_pdhg_residual(C.Structure):
    _fields_ = [(name, f64) for name in (
        "primal_residual", "dual_residual", "primal_residual_inf", "dual_residual_inf",
        "primal_objective", "dual_objective", "absolute_gap", "relative_primal",
        "relative_dual", "relative_gap", "relative_primal_inf", "relative_dual_inf")]


class anu_pdhg_phases(C.Structure):
    _fields_ = [(name, f64) for name in (
        "scaling", "matrix_norm", "setup", "iterating", "checks", "polishing")]


class anu_pdhg_result(C.Structure):
    _fields_ = [
        ("status", i32), ("objective", f64), ("iterations", i32), ("restarts", i32),
        ("polish_attempts", i32), ("polish_iterations", i32), ("polished", i32),
        ("solve_seconds", f64), ("matrix_norm_estimate", f64),
        ("final_step_size", f64), ("final_primal_weight", f64),
        ("phases", anu_pdhg_phases), ("residual", anu_pdhg_residual),
        ("row_spread_before", f64), ("row_spread_after", f64),
        ("col_spread_before", f64), ("col_spread_after", f64),
        ("refinement_rounds", i32), ("kernel_launches", i32),
        ("device_iteration_seconds", f64), ("device_iterations", C.c_int64),
        ("row_product_threads", i32), ("column_product_threads", i32),
        ("tile_trial_seconds", f64),
        ("message", C.c_char * 160),
    ]


# PdhgOptions{} defaults, src/anukulan/pdhg.hpp:19-415.
DEFAULTS = dict(
    tolerance=1e-6, gap_tolerance=0.0, max_iterations=200000,
    time_limit_seconds=300.0, termination_check_frequency=40,
    absolute_tolerance=0.0, require_inf_norm_termination=1, adaptive_step_size=1,
    primal_weight_updates=1, restarts=1, halpern=1, halpern_restart=0,
    halpern_minimum_epoch=16, polish_feasibility=1, polish_first_iteration=100,
    polish_iteration_factor=0.125, polish_minimum_iterations=40,
    polish_maximum_iterations=20000, polish_on_exit=1, reflection=1.0,
    constant_step_size=1, constant_step_scale=0.90, restart_on_fixed_point=1,
    pid_primal_weight=1, primal_weight_kp=0.5, primal_weight_ki=0.0,
    primal_weight_kd=0.3, ruiz_iterations=10, pock_chambolle=1, reuse_products=1,
    detect_infeasibility=1, infeasibility_tolerance=1e-8, termination=0,
    known_matrix_norm=0.0, initial_step_size=0.0, initial_primal_weight=0.0,
    verbose=0, log_frequency=5000, precision=0, refinement=1,
    device=0, use_graphs=1, profile=0, split_stacks=1,
    persistent_chunks=0, locality_order=0, scaling_on_device=1, tile_threads=0,
    cluster_chunks=0,
)


def make_options(**overrides: Any) -> anu_pdhg_options:
    """An ``anu_pdhg_options`` with the reference defaults and `overrides`
    applied (bools accepted)."""
    o = anu_pdhg_options()
    vals = dict(DEFAULTS)
    for k, v in overrides.items():
        if k not in vals and k != "stop":
            raise KeyError(f"unknown PDHG option {k!r}")
        vals[k] = v
    for k, v in vals.items():
        if k == "stop":
            o.stop = v
            continue
        setattr(o, k, int(v) if isinstance(v, bool) else v)
    return o


def options_dict(o: anu_pdhg_options) -> dict:
    return {name: getattr(o, name) for name, _ in anu_pdhg_options._fields_ if name != "stop"}


@dataclass
class Residual:
    primal_residual: float = 0.0
    dual_residual: float = 0.0
    primal_residual_inf: float = 0.0
    dual_residual_inf: float = 0.0
    primal_objective: float = 0.0
    dual_objective: float = 0.0
    absolute_gap: float = 0.0
    relative_primal: float = 0.0
    relative_dual: float = 0.0
    relative_gap: float = 0.0
    relative_primal_inf: float = 0.0
    relative_dual_inf: float = 0.0

    @staticmethod
    def from_c(r: anu_pdhg_residual) -> "Residual":
        return Residual(**{f.name: getattr(r, f.name) for f in fields(Residual)})

    def primal_ok(self, tol, abs_tol=0.0, inf=True):
        ok = self.relative_primal <= tol
        if inf:
            ok = ok and self.relative_primal_inf <= tol
        if abs_tol > 0:
            ok = ok and self.primal_residual_inf <= abs_tol
        return ok

    def dual_ok(self, tol, abs_tol=0.0, inf=True):
        ok = self.relative_dual <= tol
        if inf:
            ok = ok and self.relative_dual_inf <= tol
        if abs_tol > 0:
            ok = ok and self.dual_residual_inf <= abs_tol
        return ok

    def converged(self, tol, abs_tol=0.0, inf=True, gap_tol=0.0):
        """``PdhgResidual::converged`` (pdhg.hpp:476-481)."""
        return (self.primal_ok(tol, abs_tol, inf) and self.dual_ok(tol, abs_tol, inf)
                and self.relative_gap <= (gap_tol if gap_tol > 0 else tol))

    def worst_relative(self, inf=True):
        w = max(self.relative_primal, self.relative_dual, self.relative_gap)
        if inf:
            w = max(w, self.relative_primal_inf, self.relative_dual_inf)
        return w


@dataclass
class PdhgResult:
    """``PdhgResult`` (pdhg.hpp:498-541)."""

    status: int
    x: np.ndarray
    y: np.ndarray
    objective: float
    iterations: int
    restarts: int
    polish_attempts: int
    polish_iterations: int
    polished: bool
    solve_seconds: float
    matrix_norm_estimate: float
    final_step_size: float
    final_primal_weight: float
    phases: dict
    residual: Residual
    spreads: tuple
    refinement_rounds: int
    kernel_launches: int
    device_iteration_seconds: float
    device_iterations: int
    message: str
    # Single-LP product tiles (CTA sizes) of K~ x and K~' y, and the time of
    # the trial solves that chose them (0 when the option fixed them).
    row_product_threads: int = 128
    column_product_threads: int = 128
    tile_trial_seconds: float = 0.0

    @property
    def status_name(self) -> str:
        return STATUS_NAMES.get(self.status, "unknown")

    @staticmethod
    def from_c(r: anu_pdhg_result, x: np.ndarray, y: np.ndarray) -> "PdhgResult":
        return PdhgResult(
            r.status, x, y, r.objective, r.iterations, r.restarts, r.polish_attempts,
            r.polish_iterations, bool(r.polished), r.solve_seconds,
            r.matrix_norm_estimate, r.final_step_size, r.final_primal_weight,
            {name: getattr(r.phases, name) for name, _ in anu_pdhg_phases._fields_},
            Residual.from_c(r.residual),
            (r.row_spread_before, r.row_spread_after, r.col_spread_before,
             r.col_spread_after),
            r.refinement_rounds, r.kernel_launches, r.device_iteration_seconds,
            r.device_iterations, r.message.decode(errors="replace"),
            r.row_product_threads, r.column_product_threads, r.tile_trial_seconds)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class CLp:
    """An ``anu_lp`` view of a StandardLp; keeps the numpy buffers alive."""

    def __init__(self, lp: StandardLp, c=None, q=None, lower=None, upper=None):
        k = lp.k
        self._keep: List[np.ndarray] = []

        def hold(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        start = hold(k.start, np.int32)
        index = hold(k.index, np.int32)
        value = hold(k.value, np.float64)
        cc = hold(lp.c if c is None else c, np.float64)
        qq = hold(lp.q if q is None else q, np.float64)
        lo = hold(lp.lower if lower is None else lower, np.float64)
        hi = hold(lp.upper if upper is None else upper, np.float64)
        self.struct = anu_lp()
        self.struct.k = anu_csr(k.rows, k.cols, k.nnz, _ptr(start, i32), _ptr(index, i32),
                                _ptr(value, f64))
        self.struct.c = _ptr(cc, f64)
        self.struct.q = _ptr(qq, f64)
        self.struct.lower = _ptr(lo, f64)
        self.struct.upper = _ptr(hi, f64)
        self.struct.num_equalities = lp.num_equalities
        self.struct.objective_scale = lp.objective_scale
        self.struct.objective_offset = lp.objective_offset
        self.m = k.rows
        self.n = k.cols

    def ref(self):
        return C.byref(self.struct)


def f64_ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(f64))
