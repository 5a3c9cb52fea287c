"""The convergence-terms reduction without device allocation.

``anu_backend_convergence_terms_noalloc`` serves hosts that may not call
cudaMalloc. Examples are a plugin inside an application that owns the device
memory pool, and code that runs while such an application holds a stream
capture. The entry point keeps its partial sums in a fixed array in the
library's device image instead of allocating them.

This file is named to run last, so the entry point is tested both in a fresh
process (run it alone) and after every other test has used the library.

Each case calls the regular entry point and the no-alloc one on the same
device vectors. They must agree to 1e-12 relative. Both must agree with a
float64 numpy restatement of the terms to 1e-10 relative, because numpy sums in
another order. Two cases run back to back with
different sizes, so a stale partial left in the shared array by the first
call would show in the second.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12
NAMES = ("primal_sq", "primal_inf", "q_dot_y", "dual_sq", "dual_inf", "bound_term", "c_dot_x")


def _problem(n, m, num_eq, seed):
    rng = np.random.default_rng(seed)
    p = {
        "c": rng.standard_normal(n),
        "lower": np.where(rng.random(n) < 0.3, -np.inf, rng.uniform(-2, 0, n)),
        "upper": np.where(rng.random(n) < 0.3, np.inf, rng.uniform(0, 2, n)),
        "q": rng.standard_normal(m),
        "row_scale": rng.uniform(0.5, 2.0, m),
        "col_scale": rng.uniform(0.5, 2.0, n),
        "x": rng.uniform(-1, 1, n),
        "k_x": rng.standard_normal(m),
        "y": rng.standard_normal(m),
        "kt_y": rng.standard_normal(n),
    }
    p["y"][num_eq:] = np.abs(p["y"][num_eq:]) * (rng.random(m - num_eq) < 0.8)
    return p


def _numpy_terms(p, num_eq):
    """The seven terms in float64, restated from
    LinAlgBackend::convergence_terms (backend.cpp:143-201)."""
    rs, cs = p["row_scale"], p["col_scale"]
    row = np.where(rs != 0.0, p["k_x"] / np.where(rs != 0.0, rs, 1.0), p["k_x"])
    viol = row - p["q"]
    viol[num_eq:] = np.minimum(viol[num_eq:], 0.0)
    prod = np.where(cs != 0.0, p["kt_y"] / np.where(cs != 0.0, cs, 1.0), p["kt_y"])
    lam = p["c"] - prod
    has_lo, has_hi = p["lower"] > -np.inf, p["upper"] < np.inf
    left = np.where(has_lo & has_hi, 0.0,
                    np.where(has_lo, np.minimum(lam, 0.0),
                             np.where(has_hi, np.maximum(lam, 0.0), lam)))
    absorbed = lam - left
    with np.errstate(invalid="ignore"):
        bound = np.where(absorbed > 0.0, absorbed * p["lower"],
                         np.where(absorbed < 0.0, absorbed * p["upper"], 0.0))
    return np.array([np.sum(viol ** 2), np.max(np.abs(viol), initial=0.0),
                     np.dot(p["q"], rs * p["y"]), np.sum(left ** 2),
                     np.max(np.abs(left), initial=0.0), np.sum(bound),
                     np.dot(p["c"], cs * p["x"])])


class _Device:
    def __init__(self, engine):
        self.engine = engine
        self.lib = engine.lib()
        self.held = []

    def put(self, v):
        p = C.c_void_p()
        self.engine.check(self.lib.anu_backend_allocate(len(v), C.byref(p)))
        self.held.append(p)
        a = np.ascontiguousarray(v, np.float64)
        self.engine.check(self.lib.anu_backend_upload(a.ctypes.data_as(C.POINTER(C.c_double)),
                                                      p, len(v)))
        return p

    def free(self):
        for p in self.held:
            self.engine.check(self.lib.anu_backend_deallocate(p))
        self.held = []


def _call(lib, fn, n, m, num_eq, d):
    out = np.full(7, np.nan)
    rc = getattr(lib, fn)(n, m, d["c"], d["lower"], d["upper"], d["q"], d["row_scale"],
                          d["col_scale"], num_eq, d["x"], d["k_x"], d["y"], d["kt_y"],
                          out.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, out


def _close(a, b):
    return np.all(np.abs(a - b) <= RTOL * np.maximum(1.0, np.abs(b)))


def test_noalloc_matches_regular_entry_point_twice(engine):
    dev = _Device(engine)
    lib = dev.lib
    try:
        # The first call is the larger, so its partials fill more of the
        # shared array than the second call writes.
        for (n, m, num_eq, seed) in ((200_003, 150_001, 40_000, 1), (733, 501, 120, 2)):
            p = _problem(n, m, num_eq, seed)
            d = {k: dev.put(v) for k, v in p.items()}
            rc_ref, ref = _call(lib, "anu_backend_convergence_terms", n, m, num_eq, d)
            engine.check(rc_ref)
            rc, got = _call(lib, "anu_backend_convergence_terms_noalloc", n, m, num_eq, d)
            engine.check(rc)
            assert _close(got, ref), dict(zip(NAMES, zip(got, ref)))
            want = _numpy_terms(p, num_eq)
            assert np.all(np.abs(got - want) <= 1e-10 * np.maximum(1.0, np.abs(want))), \
                dict(zip(NAMES, zip(got, want)))
            dev.free()
    finally:
        dev.free()


def test_noalloc_rejects_lengths_beyond_its_limit(engine):
    lib = engine.lib()
    out = np.zeros(7)
    null = None
    rc = lib.anu_backend_convergence_terms_noalloc(
        2 ** 31, 4, null, null, null, null, null, null, 0, null, null, null, null,
        out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 1  # ANU_ERR_INVALID, before any device work
    msg = C.create_string_buffer(256)
    lib.anu_last_error(msg, 256)
    assert b"2147483647" in msg.value
