"""Several momentum Jacobi sweeps per launch from shared-memory tiles (needs a B200).

The tile kernel repeats the per-sweep kernel's arithmetic on a tile and its
halo, so a solve with S sweeps per launch must equal the solve with one launch
per sweep (the default) bit for bit: FP64 (and so the oracle), the FP32
correction sweeps of mixed precision, every S from 2 to 8, every CTA size, the
triangle mesh (three faces per cell) and a batch whose tile curve runs case by
case.
"""
import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi
import oracle

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "pp", "mDot")


def _run(mesh, bcs, settings, sweeps, threads=0, precision=abi.PREC_FP64, start=None):
    s = abi.Solver(mesh, bcs, settings, precision=precision)
    if start is not None:
        s.set_batch(start)
    s.set_momentum_sweeps(sweeps, threads)
    r = s.solve()
    out = {f: s.get(f) for f in FIELDS}
    tiles = s.sweep_tiles()
    names = {k["name"] for k in s.profile(1)}
    s.close()
    return r, out, tiles, names


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("sweeps,threads", [(2, 0), (3, 512), (4, 0), (4, 256), (8, 1024)])
def test_tiled_sweeps_equal_one_launch_per_sweep(precision, sweeps, threads):
    case = cases.expansion(scale=1 / 4, max_iter=4, tol=1e-30)  # 54k cells, four faces per cell
    mesh = abi.multiblock(case.blocks)
    r1, ref, t1, n1 = _run(mesh, case.bc_fields(), case.settings, 1, precision=precision)
    r2, got, t2, n2 = _run(mesh, case.bc_fields(), case.settings, sweeps, threads, precision=precision)
    assert t1 == 0 and t2 > 1
    tile_name = "jacobi_uv32_tiles" if precision == abi.PREC_MIXED else "jacobi_uv_tiles"
    assert tile_name in n2 and tile_name not in n1
    assert r1["iterations"] == r2["iterations"] == 4
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)


def test_tiled_sweeps_on_triangles_match_the_oracle():
    case = cases.bullet(scale=0.1, max_iter=3, tol=1e-30)  # three faces per cell
    orc = oracle.Oracle(case.mesh, case.bc_fields(), case.settings)
    assert orc.run()[0] == 3
    r, got, tiles, names = _run(case.mesh, case.bc_fields(), case.settings, 4)
    assert tiles > 1 and "jacobi_uv_tiles" in names
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], orc.get(f), err_msg=f)
    orc.close()


def test_tiled_sweeps_in_a_batch_equal_one_launch_per_sweep():
    cs = batch.random_cases(6, seed=4, scale=0.05, max_iter=4, tol=1e-30)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    _, ref, _, _ = _run(union, bcs, cs[0].settings, 1, start=start)
    _, got, tiles, _ = _run(union, bcs, cs[0].settings, 4, start=start)
    assert tiles > 1
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)


def test_launch_counts_and_gauss_seidel_keeps_its_launches():
    case = cases.expansion(scale=1 / 8, max_iter=2, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    s = abi.Solver(mesh, case.bc_fields(), case.settings)
    s.solve()
    assert s.sweep_tiles() == 0  # default: one launch per sweep
    assert {k["name"]: k for k in s.profile(1)}["jacobi_uv"]["launches"] == 20
    s.set_momentum_sweeps(4)
    s.solve()
    assert s.sweep_tiles() > 0
    prof = {k["name"]: k for k in s.profile(1)}
    assert prof["jacobi_uv_tiles"]["launches"] == 5  # 20 sweeps, four per launch
    s.close()
    gs = dict(case.settings, linearType=1)
    g = abi.Solver(mesh, case.bc_fields(), gs)
    g.set_momentum_sweeps(4)
    g.solve()
    assert g.sweep_tiles() == 0
    g.close()
    with pytest.raises(abi.AxisimError):
        abi.Solver(mesh, case.bc_fields(), case.settings).set_momentum_sweeps(9)
