"""The CPU oracle against golden vectors produced by the REFERENCE's own solver.

tests/golden/*.npz come from tests/golden/make_golden.py, which runs the
reference's solver translation units compiled unchanged from their sources
(oracle/ref_build) on a B200. The reference sums its multigrid Galerkin and
restriction with atomicAdd and contracts a*b+c into FMA, so agreement is to
rounding: 1e-10 relative L2 on u, v, p and the gradients, and the same
iteration count (also to convergence at 1e-6). The scalar-transport fixtures
add temperature and concentration with their gradients; the reference's Hill
and inhibition laws call CUDA's pow where the oracle calls the C library's,
so those agree to rounding as well.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
import sys  # noqa: E402
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

CASES = make_golden.fixture_cases()
ORACLE_NAMES = {"u": "u", "v": "v", "p": "p", "gradPZ": "gradPZ", "gradPR": "gradPR", "gradUZ": "gradUZ",
                "gradUR": "gradUR", "gradVZ": "gradVZ", "gradVR": "gradVR", "T": "T", "gradTZ": "gradTZ",
                "gradTR": "gradTR", "C": "C", "gradCZ": "gradCZ", "gradCR": "gradCR"}
TOL = 1e-10


@pytest.mark.parametrize("name,case", CASES, ids=[n for n, _ in CASES])
def test_oracle_matches_reference_solver(name, case):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    mesh = case.packed(oracle.multiblock)
    o = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, conv = o.run()
    assert it == int(g["iterations"])
    assert conv == bool(g["converged"])
    for k, on in ORACLE_NAMES.items():
        if k in g:
            assert rel_l2(o.get(on), g[k]) <= TOL, (name, k, rel_l2(o.get(on), g[k]))
    if "continuity" in g:
        # per-cell mass imbalance after the last iteration (Solver::getMassImbalance)
        scale = np.abs(o.get("mDot")).max()
        assert np.max(np.abs(o.get("res_Continuity") - g["continuity"])) <= 1e-9 * scale
    # the monitored residual history (U, V, Continuity[, Temperature, Concentration]) of the reference
    hist = g["residual_history"]
    assert hist.shape[0] == it
    np.testing.assert_allclose(o.residuals(), hist[-1, 1:4], rtol=1e-6)
    if hist.shape[1] == 6:
        s = case.settings
        solved = (s["solveEnergy"], s["solveConcentration"])
        for e in range(2):
            if s["scalarResEnabled"][e] and solved[e]:
                # scaled residuals at rounding level (1e-16) carry no digits to compare
                np.testing.assert_allclose(o.scalar_residuals()[e], hist[-1, 4 + e], rtol=1e-6, atol=1e-12)


FULLSIZE = make_golden.fullsize_fixture_cases()


@pytest.mark.parametrize("name,case", FULLSIZE, ids=[n for n, _ in FULLSIZE])
def test_oracle_matches_reference_solver_at_full_size(name, case):
    """874,496 cells, 5 iterations: strided samples, block sums and norms of u,
    v, p and grad p (compact fixture) to 1e-10, the same iteration count."""
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    mesh = oracle.multiblock(case.blocks)
    assert mesh["nCells"] == int(g["nCells"])
    o = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, conv = o.run()
    assert it == int(g["iterations"]) and conv == bool(g["converged"])
    worst = make_golden.compact_mismatch({k: o.get(k) for k in make_golden.COMPACT_FIELDS}, g)
    assert max(worst.values()) <= TOL, worst
    np.testing.assert_allclose(o.residuals(), g["residual_history"][-1, 1:4], rtol=1e-6)
    o.close()


def test_fixture_cases_are_small():
    for name, _ in CASES + FULLSIZE:
        assert os.path.getsize(os.path.join(HERE, "golden", name + ".npz")) < 400_000
