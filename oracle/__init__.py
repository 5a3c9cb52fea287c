"""Test infrastructure: ctypes loaders of the CPU checkers.

* :func:`oracle_lib` - ``liboracle.so``, the C restatement of the reference
  PDHG path (pdhg_oracle.c). Always present once built.
* :func:`ref_cuda_lib` - ``_ref/libanuref_cuda.so``, the same with the
  reference's own CUDA backend (the plain FP64 single-case GPU PDHG).
* :func:`ref_lib` - ``_ref/libanuref.so``, the reference's own sources compiled
  by oracle/Makefile, present where the reference tree was available at build
  time (the built file travels with the working tree).
* :func:`ref_b200_lib` - ``_ref/libanuref_b200.so``, the reference's solver
  with its CUDA backend replaced by the adapter over the engine; with it the
  reference's own ``test_backend`` and ``test_pdhg`` binaries
  (``_ref/test_*_b200``), built from its unmodified test sources.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package. The engine never does.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from typing import Optional

import numpy as np

from anukulan_b200.abi import (CLp, PdhgResult, Residual, anu_pdhg_options,
                               anu_pdhg_residual, anu_pdhg_result, f64_ptr,
                               make_options)
from anukulan_b200.model import StandardLp

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libanuref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libanuref_cuda.so")
REF_B200_SO = os.path.join(HERE, "_ref", "libanuref_b200.so")
REF_B200_TEST_BACKEND = os.path.join(HERE, "_ref", "test_backend_b200")
REF_B200_TEST_PDHG = os.path.join(HERE, "_ref", "test_pdhg_b200")
# The reference checkout is named by the caller of build() or by the
# ANUKULAN_REFERENCE environment variable; nothing here assumes where it is.
REF_ENV = "ANUKULAN_REFERENCE"

_oracle = None
_ref = None
_ref_cuda = None
_ref_b200 = None

_P = C.POINTER


def reference_root(root: Optional[str] = None) -> Optional[str]:
    """The reference checkout to build from: `root`, else $ANUKULAN_REFERENCE,
    kept only when it holds the reference's sources (src/anukulan/pdhg.cpp)."""
    root = root or os.environ.get(REF_ENV) or None
    if root and os.path.exists(os.path.join(root, "src", "anukulan", "pdhg.cpp")):
        return os.path.abspath(root)
    return None


def build(with_reference: Optional[bool] = None, root: Optional[str] = None) -> None:
    """Builds liboracle.so, and the reference builds under _ref/ when a
    reference checkout is given (`root` or $ANUKULAN_REFERENCE) and holds the
    sources. `with_reference=False` skips them; True requires them."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if with_reference is False:
        return
    ref = reference_root(root)
    if ref is None:
        if with_reference:
            raise RuntimeError(f"no reference checkout: pass root= or set {REF_ENV}")
        return
    subprocess.run(["make", "-s", "-j8", "-C", HERE, f"REF={ref}", "ref", "ref_cuda", "ref_b200"],
                   check=True)


def _declare(lib, name, restype, argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = argtypes
    return fn


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_reference=False)
        lib = C.CDLL(ORACLE_SO)
        _declare(lib, "oracle_pdhg_solve", C.c_int,
                 [C.c_void_p, _P(anu_pdhg_options), _P(C.c_double), _P(C.c_double),
                  _P(C.c_double), _P(C.c_double), _P(anu_pdhg_result)])
        _declare(lib, "oracle_evaluate_residual", None,
                 [C.c_void_p, _P(C.c_double), _P(C.c_double), _P(anu_pdhg_residual)])
        _declare(lib, "oracle_estimate_matrix_norm", C.c_double,
                 [C.c_void_p, C.c_int, C.c_double, C.c_int])
        _declare(lib, "oracle_scale_lp", C.c_int,
                 [C.c_void_p, C.c_int, C.c_int] + [_P(C.c_double)] * 8)
        _declare(lib, "oracle_pdhg_solve_many", C.c_int,
                 [C.c_int, C.c_void_p, _P(anu_pdhg_options), C.c_int,
                  _P(_P(C.c_double)), _P(_P(C.c_double)), _P(anu_pdhg_result)])
        _oracle = lib
    return _oracle


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("oracle/_ref/libanuref.so is not built")
        lib = C.CDLL(REF_SO)
        _declare(lib, "ref_pdhg_solve", C.c_int,
                 [C.c_void_p, _P(anu_pdhg_options), C.c_int, _P(C.c_double),
                  _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(anu_pdhg_result)])
        _declare(lib, "ref_evaluate_residual", C.c_int,
                 [C.c_void_p, _P(C.c_double), _P(C.c_double), _P(anu_pdhg_residual)])
        _declare(lib, "ref_estimate_matrix_norm", C.c_double,
                 [C.c_void_p, C.c_int, C.c_double, C.c_int])
        _declare(lib, "ref_scale_lp", C.c_int,
                 [C.c_void_p, C.c_int, C.c_int] + [_P(C.c_double)] * 8)
        _declare(lib, "ref_simplex_solve", C.c_int,
                 [C.c_void_p, C.c_double, _P(C.c_double), _P(C.c_double),
                  _P(C.c_double), _P(C.c_int)])
        _declare(lib, "ref_default_thread_count", C.c_int, [])
        _declare(lib, "ref_default_options", None, [_P(anu_pdhg_options)])
        _declare(lib, "ref_to_standard_form", C.c_int,
                 [C.c_int32, C.c_int32, C.c_int32, _P(C.c_int32), _P(C.c_int32),
                  _P(C.c_double)] + [_P(C.c_double)] * 5 + [C.c_int, C.c_double,
                  _P(C.c_int32), _P(C.c_int32), _P(C.c_double), _P(C.c_double),
                  _P(C.c_double), _P(C.c_int32), _P(C.c_double), _P(C.c_double),
                  _P(C.c_int32)])
        _ref = lib
    return _ref


def _opts(options=None, **kw) -> anu_pdhg_options:
    if options is not None:
        return options
    return make_options(**kw)


def oracle_solve(lp: StandardLp, options=None, warm_x=None, warm_y=None, **kw) -> PdhgResult:
    """The restated solve_pdhg on the host."""
    cl = CLp(lp)
    o = _opts(options, **kw)
    x = np.zeros(cl.n)
    y = np.zeros(cl.m)
    r = anu_pdhg_result()
    wx = None if warm_x is None else np.ascontiguousarray(warm_x, np.float64)
    wy = None if warm_y is None else np.ascontiguousarray(warm_y, np.float64)
    oracle_lib().oracle_pdhg_solve(cl.ref(), C.byref(o), f64_ptr(wx), f64_ptr(wy),
                                   f64_ptr(x), f64_ptr(y), C.byref(r))
    return PdhgResult.from_c(r, x, y)


def have_reference_cuda() -> bool:
    return os.path.exists(REF_CUDA_SO)


def ref_cuda_lib():
    """_ref/libanuref_cuda.so: the reference with its own CUDA backend."""
    global _ref_cuda
    if _ref_cuda is None:
        if not os.path.exists(REF_CUDA_SO):
            raise FileNotFoundError("oracle/_ref/libanuref_cuda.so is not built")
        lib = C.CDLL(REF_CUDA_SO)
        _declare(lib, "ref_pdhg_solve", C.c_int,
                 [C.c_void_p, _P(anu_pdhg_options), C.c_int, _P(C.c_double),
                  _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(anu_pdhg_result)])
        _ref_cuda = lib
    return _ref_cuda


def ref_cuda_solve(lp: StandardLp, options=None, lib=None, **kw) -> PdhgResult:
    """The reference's own solve_pdhg on its CUDA backend (cuda_backend.cu,
    FP64, one LP per call), or on whatever `lib`'s cuda_backend() is."""
    cl = CLp(lp)
    o = _opts(options, **kw)
    x = np.zeros(cl.n)
    y = np.zeros(cl.m)
    r = anu_pdhg_result()
    lib = lib if lib is not None else ref_cuda_lib()
    rc = lib.ref_pdhg_solve(cl.ref(), C.byref(o), -2, None, None, f64_ptr(x),
                            f64_ptr(y), C.byref(r))
    if rc != 0:
        raise RuntimeError(r.message.decode())
    return PdhgResult.from_c(r, x, y)


def have_reference_b200() -> bool:
    return all(os.path.exists(p) for p in (REF_B200_SO, REF_B200_TEST_BACKEND,
                                            REF_B200_TEST_PDHG))


def ref_b200_lib():
    """_ref/libanuref_b200.so: the reference's unmodified solver with
    anukulan::cuda_backend() resolved to the LinAlgBackend adapter over the
    engine (include/anu_b200_backend.hpp). It loads the engine library."""
    global _ref_b200
    if _ref_b200 is None:
        if not os.path.exists(REF_B200_SO):
            raise FileNotFoundError("oracle/_ref/libanuref_b200.so is not built")
        lib = C.CDLL(REF_B200_SO)
        _declare(lib, "ref_pdhg_solve", C.c_int,
                 [C.c_void_p, _P(anu_pdhg_options), C.c_int, _P(C.c_double),
                  _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(anu_pdhg_result)])
        _declare(lib, "ref_default_backend_name", C.c_int, [C.c_char_p, C.c_int])
        _declare(lib, "ref_finish_simplex", C.c_int,
                 [C.c_void_p, _P(C.c_double), _P(C.c_double), C.c_int, _P(C.c_double),
                  _P(C.c_double), _P(C.c_double), _P(C.c_int32), _P(C.c_int32),
                  _P(C.c_int32), _P(C.c_int32)])
        _declare(lib, "ref_simplex_basis", C.c_int,
                 [C.c_void_p, _P(C.c_int32), C.c_int32, _P(C.c_int32), C.c_int32,
                  _P(C.c_int32), _P(C.c_int32), _P(C.c_int32), _P(C.c_int32), _P(C.c_double)])
        _ref_b200 = lib
    return _ref_b200


def ref_b200_backend_name() -> str:
    buf = C.create_string_buffer(64)
    ref_b200_lib().ref_default_backend_name(buf, 64)
    return buf.value.decode()


def ref_pipeline(model, options=None, use_presolve: bool = True, engine: bool = True, **kw):
    """anu_b200::solve_model_pdhg (include/anu_b200_pipeline.hpp): the
    reference's presolve -> standard form -> solve_pdhg -> postsolve on a
    :class:`Model`, with the PDHG step on the engine (`engine`) or on the
    reference's cpu_backend(). Returns (rc, result, x, y, info) with info =
    worst violation, relative row violation, dual exact, presolve status."""
    lib = ref_b200_lib()
    fn = getattr(lib, "ref_pipeline_solve")
    fn.restype = C.c_int
    a = model.constraints
    m, n = a.rows, a.cols
    i32 = lambda arr: np.ascontiguousarray(arr, np.int32)
    f64 = lambda arr: np.ascontiguousarray(arr, np.float64)
    keep = [i32(a.start), i32(a.index), f64(a.value), f64(model.objective),
            f64(model.row_lower), f64(model.row_upper), f64(model.col_lower),
            f64(model.col_upper)]
    ip = lambda arr: arr.ctypes.data_as(_P(C.c_int32))
    o = _opts(options, **kw)
    x = np.zeros(max(n, 1))
    y = np.zeros(max(m, 1))
    info = np.zeros(4)
    r = anu_pdhg_result()
    rc = fn(C.c_int32(m), C.c_int32(n), C.c_int32(a.nnz), ip(keep[0]), ip(keep[1]),
            f64_ptr(keep[2]), f64_ptr(keep[3]), f64_ptr(keep[4]), f64_ptr(keep[5]),
            f64_ptr(keep[6]), f64_ptr(keep[7]), C.c_int(int(model.maximize)),
            C.c_double(float(model.objective_offset)), C.byref(o), C.c_int(int(use_presolve)),
            C.c_int(0 if engine else 1), f64_ptr(x), f64_ptr(y), C.byref(r), f64_ptr(info))
    return rc, PdhgResult.from_c(r, x[:n].copy(), y[:m].copy()), x[:n].copy(), y[:m].copy(), info


SIMPLEX_STATUS_NAMES = {0: "optimal"}


def ref_pipeline_crossover(model, options=None, use_presolve: bool = True, engine: bool = True,
                           crossover_tolerance: float = 1e-4, **kw):
    """anu_b200::solve_model_crossover (include/anu_b200_pipeline.hpp): the
    CLI's `simplex --crossover` (app/anukulan_cli.cpp:574-636) on a
    :class:`Model`, the PDHG seed on the engine (`engine`) or on cpu_backend().
    Returns (rc, x, info) with info a dict: simplex status (0 optimal),
    pivots, seeded, fell_back, seeded_pivots, seed_iterations, seed_status,
    row_violation, objective, candidates, pushed, presolve_status."""
    lib = ref_b200_lib()
    fn = getattr(lib, "ref_pipeline_crossover")
    fn.restype = C.c_int
    a = model.constraints
    m, n = a.rows, a.cols
    i32 = lambda arr: np.ascontiguousarray(arr, np.int32)
    f64 = lambda arr: np.ascontiguousarray(arr, np.float64)
    keep = [i32(a.start), i32(a.index), f64(a.value), f64(model.objective),
            f64(model.row_lower), f64(model.row_upper), f64(model.col_lower),
            f64(model.col_upper)]
    ip = lambda arr: arr.ctypes.data_as(_P(C.c_int32))
    o = _opts(options, **kw)
    x = np.zeros(max(n, 1))
    info = np.zeros(12)
    rc = fn(C.c_int32(m), C.c_int32(n), C.c_int32(a.nnz), ip(keep[0]), ip(keep[1]),
            f64_ptr(keep[2]), f64_ptr(keep[3]), f64_ptr(keep[4]), f64_ptr(keep[5]),
            f64_ptr(keep[6]), f64_ptr(keep[7]), C.c_int(int(model.maximize)),
            C.c_double(float(model.objective_offset)), C.byref(o), C.c_int(int(use_presolve)),
            C.c_int(0 if engine else 1), C.c_double(crossover_tolerance), f64_ptr(x),
            f64_ptr(info))
    names = ("status", "pivots", "seeded", "fell_back", "seeded_pivots", "seed_iterations",
             "seed_status", "row_violation", "objective", "candidates", "pushed",
             "presolve_status")
    d = dict(zip(names, info.tolist()))
    for k in names:
        if k not in ("row_violation", "objective"):
            d[k] = int(d[k])
    return rc, x[:n].copy(), d


def ref_finish_simplex(lp: StandardLp, x, y, dual: bool = False):
    """anu_b200::finish_with_simplex: crossover_basis at (x, y), the simplex
    from its basis (the dual simplex when `dual`), the cold solve after a
    miss. Returns a dict: status (0 optimal), pivots, seeded, fell_back,
    seeded_pivots, objective, seconds, candidates, pushed, x, y and basis (the
    simplex's final (basic, status), for ref_simplex_basis)."""
    cl = CLp(lp)
    xi = np.ascontiguousarray(x, np.float64)
    yi = np.ascontiguousarray(y, np.float64)
    xo = np.zeros(max(cl.n, 1))
    yo = np.zeros(max(cl.m, 1))
    info = np.zeros(9)
    cap_b, cap_s = max(cl.m, 1) + 8, cl.n + cl.m + 8
    bo = np.zeros(cap_b, np.int32)
    so = np.zeros(cap_s, np.int32)
    nb, ns = C.c_int32(cap_b), C.c_int32(cap_s)
    ip = lambda arr: arr.ctypes.data_as(_P(C.c_int32))
    rc = ref_b200_lib().ref_finish_simplex(cl.ref(), f64_ptr(xi), f64_ptr(yi), int(dual),
                                           f64_ptr(xo), f64_ptr(yo), f64_ptr(info), ip(bo),
                                           C.byref(nb), ip(so), C.byref(ns))
    if rc != 0:
        raise RuntimeError(f"ref_finish_simplex returned {rc}")
    d = dict(zip(("status", "pivots", "seeded", "fell_back", "seeded_pivots", "objective",
                  "seconds", "candidates", "pushed"), info.tolist()))
    for k in ("status", "pivots", "seeded", "fell_back", "seeded_pivots", "candidates", "pushed"):
        d[k] = int(d[k])
    d["x"] = xo[:cl.n].copy()
    d["y"] = yo[:cl.m].copy()
    d["basis"] = (bo[:nb.value].copy(), so[:ns.value].copy())
    return d


def ref_finish_model(model, x, y, use_presolve: bool = False, dual: bool = False,
                     seeded_pivot_limit: int = 0):
    """anu_b200::finish_model_with_simplex: a :class:`Model` finished exactly
    from a first-order point of its unpresolved standard form (x: columns, y:
    standard-form rows). Returns (rc, x_model, info) with info a dict: status
    (0 optimal), pivots, seeded, fell_back, seeded_pivots, objective (model),
    seconds, candidates, pushed, row_violation, presolve_status."""
    lib = ref_b200_lib()
    fn = getattr(lib, "ref_finish_model")
    fn.restype = C.c_int
    a = model.constraints
    m, n = a.rows, a.cols
    i32 = lambda arr: np.ascontiguousarray(arr, np.int32)
    f64 = lambda arr: np.ascontiguousarray(arr, np.float64)
    keep = [i32(a.start), i32(a.index), f64(a.value), f64(model.objective),
            f64(model.row_lower), f64(model.row_upper), f64(model.col_lower),
            f64(model.col_upper), f64(x), f64(y)]
    ip = lambda arr: arr.ctypes.data_as(_P(C.c_int32))
    xo = np.zeros(max(n, 1))
    info = np.zeros(11)
    rc = fn(C.c_int32(m), C.c_int32(n), C.c_int32(a.nnz), ip(keep[0]), ip(keep[1]),
            f64_ptr(keep[2]), f64_ptr(keep[3]), f64_ptr(keep[4]), f64_ptr(keep[5]),
            f64_ptr(keep[6]), f64_ptr(keep[7]), C.c_int(int(model.maximize)),
            C.c_double(float(model.objective_offset)), f64_ptr(keep[8]), f64_ptr(keep[9]),
            C.c_int32(len(keep[9])), C.c_int(int(use_presolve)), C.c_int(int(dual)),
            C.c_int32(int(seeded_pivot_limit)), f64_ptr(xo), f64_ptr(info))
    names = ("status", "pivots", "seeded", "fell_back", "seeded_pivots", "objective",
             "seconds", "candidates", "pushed", "row_violation", "presolve_status")
    d = dict(zip(names, info.tolist()))
    for k in ("status", "pivots", "seeded", "fell_back", "seeded_pivots", "candidates",
              "pushed", "presolve_status"):
        d[k] = int(d[k])
    return rc, xo[:n].copy(), d


def ref_simplex_basis(lp: StandardLp, basis=None):
    """One member of the reference's `family --from-first` (dual simplex,
    app/anukulan_cli.cpp:1065-1230): solve_lp from `basis` = (basic, status),
    or cold when None. Returns (info, final basis) with info a dict: status
    (0 optimal), pivots, objective, seconds."""
    cl = CLp(lp)
    cap_b = max(cl.m, 1) + 8
    cap_s = cl.n + cl.m + 8
    bo = np.zeros(cap_b, np.int32)
    so = np.zeros(cap_s, np.int32)
    nb = C.c_int32(cap_b)
    ns = C.c_int32(cap_s)
    info = np.zeros(4)
    ip = lambda arr: None if arr is None else arr.ctypes.data_as(_P(C.c_int32))
    if basis is None:
        bi = si = None
        lb = ls = 0
    else:
        bi = np.ascontiguousarray(basis[0], np.int32)
        si = np.ascontiguousarray(basis[1], np.int32)
        lb, ls = len(bi), len(si)
    rc = ref_b200_lib().ref_simplex_basis(cl.ref(), ip(bi), lb, ip(si), ls, ip(bo),
                                          C.byref(nb), ip(so), C.byref(ns), f64_ptr(info))
    if rc != 0:
        raise RuntimeError(f"ref_simplex_basis returned {rc}")
    d = dict(zip(("status", "pivots", "objective", "seconds"), info.tolist()))
    d["status"] = int(d["status"])
    d["pivots"] = int(d["pivots"])
    return d, (bo[:nb.value].copy(), so[:ns.value].copy())


def ref_b200_solve(lp: StandardLp, options=None, **kw) -> PdhgResult:
    """The reference's own solve_pdhg, unchanged, with the engine's kernels
    under its LinAlgBackend seam (FP64, one seam call per launch)."""
    return ref_cuda_solve(lp, options, lib=ref_b200_lib(), **kw)


def ref_solve(lp: StandardLp, options=None, threads: int = 1, warm_x=None, warm_y=None,
              **kw) -> PdhgResult:
    """The reference's own solve_pdhg (cpu_backend, or threaded_cpu_backend
    when threads > 1; threads < 0 is the reference's default count)."""
    cl = CLp(lp)
    o = _opts(options, **kw)
    x = np.zeros(cl.n)
    y = np.zeros(cl.m)
    r = anu_pdhg_result()
    wx = None if warm_x is None else np.ascontiguousarray(warm_x, np.float64)
    wy = None if warm_y is None else np.ascontiguousarray(warm_y, np.float64)
    rc = ref_lib().ref_pdhg_solve(cl.ref(), C.byref(o), threads, f64_ptr(wx), f64_ptr(wy),
                                  f64_ptr(x), f64_ptr(y), C.byref(r))
    if rc != 0:
        raise RuntimeError(r.message.decode())
    return PdhgResult.from_c(r, x, y)


def oracle_residual(lp: StandardLp, x, y) -> Residual:
    cl = CLp(lp)
    out = anu_pdhg_residual()
    oracle_lib().oracle_evaluate_residual(cl.ref(), f64_ptr(np.ascontiguousarray(x, np.float64)),
                                          f64_ptr(np.ascontiguousarray(y, np.float64)),
                                          C.byref(out))
    return Residual.from_c(out)


def ref_residual(lp: StandardLp, x, y) -> Residual:
    cl = CLp(lp)
    out = anu_pdhg_residual()
    ref_lib().ref_evaluate_residual(cl.ref(), f64_ptr(np.ascontiguousarray(x, np.float64)),
                                    f64_ptr(np.ascontiguousarray(y, np.float64)),
                                    C.byref(out))
    return Residual.from_c(out)


def oracle_matrix_norm(lp: StandardLp, iterations=200, tolerance=1e-8, scaled=False) -> float:
    return oracle_lib().oracle_estimate_matrix_norm(CLp(lp).ref(), iterations, tolerance,
                                                    int(scaled))


def ref_matrix_norm(lp: StandardLp, iterations=200, tolerance=1e-8, scaled=False) -> float:
    return ref_lib().ref_estimate_matrix_norm(CLp(lp).ref(), iterations, tolerance, int(scaled))


def _scale(fn, lp: StandardLp, ruiz=10, pc=True):
    cl = CLp(lp)
    n, m, nnz = lp.num_cols, lp.num_rows, lp.k.nnz
    out = dict(k_value=np.zeros(nnz), c=np.zeros(n), q=np.zeros(m), lower=np.zeros(n),
               upper=np.zeros(n), row_scale=np.zeros(m), col_scale=np.zeros(n),
               spreads=np.zeros(4))
    fn(cl.ref(), ruiz, int(pc), *[f64_ptr(out[k]) for k in
                                 ("k_value", "c", "q", "lower", "upper", "row_scale",
                                  "col_scale", "spreads")])
    return out


def oracle_scale(lp: StandardLp, ruiz=10, pc=True) -> dict:
    return _scale(oracle_lib().oracle_scale_lp, lp, ruiz, pc)


def ref_scale(lp: StandardLp, ruiz=10, pc=True) -> dict:
    return _scale(ref_lib().ref_scale_lp, lp, ruiz, pc)


def ref_simplex(lp: StandardLp, time_limit: float = 300.0):
    """The reference dual simplex (through solve_lp). Returns
    (status, objective, iterations, x, y); status 0 is optimal."""
    cl = CLp(lp)
    x = np.zeros(cl.n)
    y = np.zeros(cl.m)
    obj = C.c_double(0.0)
    its = C.c_int(0)
    st = ref_lib().ref_simplex_solve(cl.ref(), time_limit, f64_ptr(x), f64_ptr(y),
                                     C.byref(obj), C.byref(its))
    return st, obj.value, its.value, x, y


def ref_default_options() -> anu_pdhg_options:
    o = anu_pdhg_options()
    ref_lib().ref_default_options(C.byref(o))
    return o


def ref_to_standard_form(model) -> Optional[StandardLp]:
    """The reference's to_standard_form of a :class:`Model`."""
    from anukulan_b200.model import Csr
    a = model.constraints
    m, n, nnz = a.rows, a.cols, a.nnz
    i32 = lambda arr: np.ascontiguousarray(arr, np.int32)
    f64 = lambda arr: np.ascontiguousarray(arr, np.float64)
    keep = [i32(a.start), i32(a.index), f64(a.value), f64(model.objective),
            f64(model.row_lower), f64(model.row_upper), f64(model.col_lower),
            f64(model.col_upper)]
    o_start = np.zeros(2 * m + 1, np.int32)
    o_index = np.zeros(max(2 * nnz, 1), np.int32)
    o_value = np.zeros(max(2 * nnz, 1))
    o_c = np.zeros(max(n, 1))
    o_q = np.zeros(max(2 * m, 1))
    o_row = np.zeros(max(2 * m, 1), np.int32)
    o_sign = np.zeros(max(2 * m, 1))
    so = np.zeros(2)
    sizes = np.zeros(2, np.int32)
    ip = lambda arr: arr.ctypes.data_as(_P(C.c_int32))
    rows = ref_lib().ref_to_standard_form(
        m, n, nnz, ip(keep[0]), ip(keep[1]), f64_ptr(keep[2]), f64_ptr(keep[3]),
        f64_ptr(keep[4]), f64_ptr(keep[5]), f64_ptr(keep[6]), f64_ptr(keep[7]),
        int(model.maximize), float(model.objective_offset), ip(o_start), ip(o_index),
        f64_ptr(o_value), f64_ptr(o_c), f64_ptr(o_q), ip(o_row), f64_ptr(o_sign), f64_ptr(so),
        ip(sizes))
    if rows < 0:
        return None
    k = Csr(rows, n, o_start[:rows + 1].copy(), o_index[:sizes[1]].copy(),
            o_value[:sizes[1]].copy())
    return StandardLp(k, o_c[:n].copy(), o_q[:rows].copy(), f64(model.col_lower).copy(),
                      f64(model.col_upper).copy(), int(sizes[0]), float(so[0]), float(so[1]),
                      o_row[:rows].copy(), o_sign[:rows].copy())


def oracle_solve_many(lps, options=None, threads: int = 1, **kw):
    """Solves independent LPs on `threads` host threads; returns
    (results, seconds)."""
    o = _opts(options, **kw)
    cls = [CLp(lp) for lp in lps]
    arr = (type(cls[0].struct) * len(cls))(*[c.struct for c in cls])
    xs = [np.zeros(c.n) for c in cls]
    ys = [np.zeros(c.m) for c in cls]
    xp = (_P(C.c_double) * len(cls))(*[f64_ptr(a) for a in xs])
    yp = (_P(C.c_double) * len(cls))(*[f64_ptr(a) for a in ys])
    res = (anu_pdhg_result * len(cls))()
    t0 = time.perf_counter()
    oracle_lib().oracle_pdhg_solve_many(len(cls), C.cast(arr, C.c_void_p), C.byref(o), threads,
                                        xp, yp, res)
    dt = time.perf_counter() - t0
    return [PdhgResult.from_c(res[i], xs[i], ys[i]) for i in range(len(cls))], dt
