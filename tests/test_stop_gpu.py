"""Cancellation through the C ABI, on the B200.

PdhgOptions::stop (pdhg.hpp:414) is a std::atomic<bool> that another thread
sets; the engine race sets it when the simplex wins (ipm.cpp:1306-1317).
Here a one-byte flag, as anu_pdhg_options.stop takes it, is set by the test's
main thread while the solve runs on another thread (ctypes releases the GIL
for the call). The solve, and every case of a case stack, must end at the
next termination check with ANU_PDHG_TIME_LIMIT, the reference's status for
a stop request, well before its iteration limit and soon after the flag.
"""
import ctypes as C
import threading
import time

import pytest

from anukulan_b200 import lpgen
from anukulan_b200.abi import TIME_LIMIT

pytestmark = pytest.mark.gpu

# A tolerance FP64 iterates cannot reach on the refinery LP, so only the flag
# ends the run. (FP32 iterates with re-centring refinement can: their FP64
# base point reaches machine precision there, so these tests run in FP64.)
RUN = dict(tolerance=1e-15, gap_tolerance=1e-15, max_iterations=50_000_000,
           time_limit_seconds=120.0, polish_feasibility=False)


def _run_and_stop(call, delay=1.0):
    flag = (C.c_uint8 * 1)(0)
    box = {}

    def worker():
        t0 = time.perf_counter()
        box["result"] = call(C.cast(flag, C.POINTER(C.c_uint8)))
        box["seconds"] = time.perf_counter() - t0

    th = threading.Thread(target=worker)
    th.start()
    time.sleep(delay)
    assert th.is_alive(), "the solve ended before the stop request"
    flag[0] = 1
    th.join(timeout=60)
    assert not th.is_alive(), "the solve did not stop"
    return box["result"], box["seconds"]


def test_stop_flag_ends_a_single_solve(engine):
    lp = lpgen.refinery_stack().base
    r, seconds = _run_and_stop(lambda stop: engine.solve_pdhg(lp, stop=stop, **RUN))
    assert r.status == TIME_LIMIT, r.message
    assert 0 < r.iterations < RUN["max_iterations"]
    assert seconds < 10.0


def test_stop_flag_ends_a_case_stack(engine):
    st = lpgen.refinery_stack()
    sub = lpgen.CaseStack(st.base, st.names[:8], st.c[:8], st.q[:8], st.lower[:8], st.upper[:8])
    res, seconds = _run_and_stop(
        lambda stop: engine.solve_case_stack(sub, stop=stop, **RUN))
    assert len(res) == 8
    for r in res:
        assert r.status == TIME_LIMIT, r.message
        assert 0 < r.iterations < RUN["max_iterations"]
    assert seconds < 10.0
