"""Failure paths of a solve, made on the host (needs a B200).

* A stop requested from another thread while a long solve runs
  (Solver::requestStop, solver.cpp:175-184): the solve returns AXISIM_E_STOPPED
  at an iteration boundary (solver.cpp:1111-1114 checks at the top of each
  iteration), the fields read back are exactly the state after the iterations it
  reports (the oracle after that many iterations, bit for bit), and continuing
  from there gives the same fields as one uninterrupted solve.
* A non-finite boundary value built on the host: the residual turns NaN, which
  never counts as converged (solver.cpp:53-60); the solve ends early with
  AXISIM_E_DIVERGED instead of running out its budget, and the handle stays
  usable.

No GPU fault is involved: the stop is a host flag the first kernel of each
iteration reads, and divergence is a residual check on the device.
"""
import math
import threading
import time

import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi
import oracle

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "mDot")


def _case(max_iter):
    c = cases.expansion(scale=1 / 16, max_iter=max_iter, tol=1e-30)
    return c, abi.multiblock(c.blocks)


def test_request_stop_from_another_thread_returns_consistent_fields():
    case, mesh = _case(200000)
    s = abi.Solver(mesh, case.bc_fields(), case.settings)
    result = {}

    def run():
        result["r"] = s.solve(allow=(abi.OK, abi.E_STOPPED))

    t = threading.Thread(target=run)
    t.start()
    time.sleep(0.5)  # set-up, graph capture and the first iterations
    assert t.is_alive(), "the solve ended before the stop was requested"
    assert s.request_stop() == abi.OK
    t.join(timeout=60)
    assert not t.is_alive(), "the solve did not stop"
    r = result["r"]
    assert r["status"] == abi.E_STOPPED, r
    k = r["iterations"]
    assert 0 < k < 200000, r
    stopped = {f: s.get(f) for f in FIELDS}
    # the stopped state is exactly the state after k complete iterations
    st = dict(case.settings, maxIter=k)
    o = oracle.Oracle(oracle.multiblock(case.blocks), case.bc_fields(), st)
    it, _ = o.run()
    assert it == k
    for f in FIELDS:
        assert np.array_equal(stopped[f], o.get(f)), f
    o.close()
    # continue for 7 more iterations == one solve of k + 7 iterations
    ok, why = s.can_continue()
    assert ok, why
    s.set_max_iter(7)
    r2 = s.solve(cont=True)
    assert r2["status"] == abi.OK and r2["iterations"] == 7, r2
    cont = {f: s.get(f) for f in FIELDS}
    s.close()
    g = abi.Solver(mesh, case.bc_fields(), dict(case.settings, maxIter=k + 7))
    r3 = g.solve()
    assert r3["iterations"] == k + 7
    for f in FIELDS:
        assert np.array_equal(cont[f], g.get(f)), f
    g.close()


def test_nan_boundary_value_reports_diverged_and_the_handle_recovers():
    case, mesh = _case(500)
    bcs = case.bc_fields()
    bad = {k: {kk: (np.array(vv, copy=True) if vv is not None else None) for kk, vv in v.items()}
           for k, v in bcs.items()}
    inlet = 0  # group 0 is the velocity inlet
    bad["u"]["value"][inlet] = math.nan
    s = abi.Solver(mesh, bad, case.settings)
    t0 = time.perf_counter()
    r = s.solve(allow=(abi.E_DIVERGED,))
    assert time.perf_counter() - t0 < 60
    assert r["status"] == abi.E_DIVERGED, r
    assert r["iterations"] < 500, r
    assert not all(math.isfinite(x) for x in r["residual"]), r
    # the same handle, given the finite value back, solves normally from rest
    b, keep = abi.bc_struct(bcs["u"])
    s._check(abi.lib().axisim_set_bc(s.h, abi.VAR_U, abi.C.byref(b)))
    s.set_max_iter(5)
    r = s.solve()
    assert r["status"] == abi.OK and r["iterations"] == 5, r
    assert all(np.isfinite(s.get(f)).all() for f in FIELDS)
    s.close()
