"""Parity at the workloads' own sizes (needs a B200).

The FP64 CUDA path and the oracle run the same few SIMPLE iterations on each
workload at full size, and every intermediate array is compared bit for bit
(the same lists as the small-case parity tests):

* the sudden expansion, 256 x 4096 band cells (874,496 cells), SOU + LSQ;
* the jittered bullet triangle mesh (485,868 cells), LSQ + non-orthogonal corrector;
* the pulsatile expansion at 1,998,855 cells, two BDF2 time steps;
* the first 16 cases of the seed-0 batch draw solved as one batch, each case
  against the oracle solving it alone.

The expansion is also matched to the reference's own solver at full size (a
compact fixture: strided samples, block sums, norms; 1e-10), and the mixed
precision path is held to 1e-6 relative L2 of the FP64 fields on the bullet.
"""
import os

import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi
import oracle
from helpers import FIELDS, GEOM, rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _bitexact(name, case, mesh, fields=FIELDS):
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it_o, _ = orc.run()
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    r = gpu.solve()
    assert r["iterations"] == it_o, (r, it_o)
    for g in GEOM:
        np.testing.assert_array_equal(gpu.get(g), orc.get(g), err_msg=f"{name}: {g}")
    for f in fields:
        a, b = gpu.get(f), orc.get(f)
        assert a.shape == b.shape, f
        np.testing.assert_array_equal(a, b, err_msg=f"{name}: {f}")
    np.testing.assert_allclose(r["residual"], orc.residuals(), rtol=1e-12, atol=0)
    gpu.close()
    orc.close()


def test_expansion_874k_bitexact():
    case = cases.expansion(scale=1.0, max_iter=3, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    assert mesh["nCells"] == 874496
    _bitexact("expansion_874496", case, mesh)


def test_bullet_485k_bitexact():
    case = cases.bullet(scale=1.0, max_iter=3, tol=1e-30)
    assert case.mesh["nCells"] == 485868
    _bitexact("bullet_485868", case, case.mesh)


def test_pulsatile_2m_two_bdf2_steps_bitexact():
    case = cases.pulsatile_expansion(scale=1.512, dt=1e-4, steps=2, max_iter=3, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    assert mesh["nCells"] == 1998855
    _bitexact("pulsatile_1998855", case, mesh, fields=["u", "v", "p", "pp", "mDot", "DU", "DV", "gradPZ", "gradPR",
                                                       "AC_u", "b_u", "AF_u", "AC_pp", "b_pp", "res_U", "res_V",
                                                       "res_Continuity"])


def test_batch_of_16_cases_bitexact_per_case():
    """The first 16 cases of the seed-0 batch draw (1,163,304 cells), solved
    as one batch, against the oracle solving each case alone."""
    cs = batch.random_cases(16, seed=0, max_iter=3, tol=1e-30)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    assert union["nCells"] > 1_000_000
    gpu = abi.Solver(union, bcs, cs[0].settings)
    gpu.set_batch(start)
    r = gpu.solve()
    assert r["iterations"] == 3
    got = {f: batch.split_fields(gpu.get(f), start) for f in ("u", "v", "p", "pp", "DU", "gradPZ", "res_U")}
    gpu.close()
    for i, c in enumerate(cs):
        orc = oracle.Oracle(meshes[i], c.bc_fields(), c.settings)
        assert orc.run()[0] == 3
        for f, parts in got.items():
            np.testing.assert_array_equal(parts[i], orc.get(f), err_msg=f"case {i}: {f}")
        orc.close()


def test_expansion_874k_matches_reference_solver():
    """The CUDA path against the reference's own solver at full size (5 iterations)."""
    import make_golden
    name, case = make_golden.fullsize_fixture_cases()[0]
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    r = gpu.solve()
    assert r["iterations"] == int(g["iterations"]) and r["converged"] == bool(g["converged"])
    worst = make_golden.compact_mismatch({k: gpu.get(k) for k in make_golden.COMPACT_FIELDS}, g)
    assert max(worst.values()) <= 1e-10, worst
    np.testing.assert_allclose(r["residual"], g["residual_history"][-1, 1:4], rtol=1e-6)
    gpu.close()


def test_bullet_485k_mixed_precision_within_1e6_of_fp64():
    """FP32 inner solves inside FP64 refinement: after 30 SIMPLE iterations of
    the full bullet mesh, u, v and p stay within 1e-6 relative L2 of the
    all-FP64 oracle run of the same iterations."""
    case = cases.bullet(scale=1.0, max_iter=30, tol=1e-30)
    orc = oracle.Oracle(case.mesh, case.bc_fields(), case.settings)
    orc.run()
    gpu = abi.Solver(case.mesh, case.bc_fields(), case.settings, precision=abi.PREC_MIXED)
    r = gpu.solve()
    assert r["iterations"] == 30
    for f in ("u", "v", "p"):
        e = rel_l2(gpu.get(f), orc.get(f))
        assert e <= 1e-6, (f, e)
    gpu.close()
    orc.close()
