"""axisim_residual_static: the allocation-free residual entry point.

Its inputs are the momentum systems, fields and face mass fluxes that a solve
left behind (read back through axisim_get_field); its per-cell outputs must
equal the residual arrays that the solve's own residual step wrote, and its
sums the sums of those arrays, on two calls in a row (the second one reusing
the static scratch the first left behind).
"""
import ctypes as C

import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _solved_case():
    case = cases.expansion(scale=1 / 8, max_iter=30, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    s = abi.Solver(mesh, case.bc_fields(), case.settings)
    s.solve()
    names = ("AF_u", "AC_u", "AC_v", "b_u", "b_v", "u", "v", "mDot", "res_U", "res_V", "res_Continuity")
    got = {n: s.get(n) for n in names}
    s.close()
    return mesh, got


def _call(mesh, dev, out, normU, normV, n_cells=None):
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = abi.lib().axisim_residual_static(
        int(mesh["nCells"]) if n_cells is None else n_cells, int(mesh["nFaces"]), len(mesh["cellFaceIDs"]),
        dev["cellFaceStart"].data_ptr(), dev["cellFaceIDs"].data_ptr(), dev["faceOwner"].data_ptr(),
        dev["faceNeighbor"].data_ptr(), dev["AF_u"].data_ptr(), dev["AC_u"].data_ptr(), dev["AC_v"].data_ptr(),
        dev["b_u"].data_ptr(), dev["b_v"].data_ptr(), dev["u"].data_ptr(), dev["v"].data_ptr(),
        dev["mDot"].data_ptr(), normU, normV, out["resU"].data_ptr(), out["resV"].data_ptr(),
        out["resC"].data_ptr(), out["sums"].data_ptr(), stream, err, len(err))
    return st, err.value.decode()


def test_residual_static_matches_solver_residuals_twice():
    mesh, got = _solved_case()
    assert np.abs(got["res_U"]).max() > 0 and np.abs(got["res_Continuity"]).max() > 0
    dev = {k: torch.from_numpy(np.ascontiguousarray(mesh[k])).cuda()
           for k in ("cellFaceStart", "cellFaceIDs", "faceOwner", "faceNeighbor")}
    dev.update({k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in got.items()})
    N = int(mesh["nCells"])
    for normU, normV in ((0, 1), (0, 1), (2, 1)):
        out = {k: torch.full((N,), float("nan"), dtype=torch.float64, device="cuda") for k in ("resU", "resV", "resC")}
        out["sums"] = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
        st, msg = _call(mesh, dev, out, normU, normV)
        assert st == abi.OK, msg
        resU, resV, resC = (out[k].cpu().numpy() for k in ("resU", "resV", "resC"))
        np.testing.assert_allclose(resU, got["res_U"], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(resV, got["res_V"], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(resC, got["res_Continuity"], rtol=1e-12, atol=1e-300)
        stat = lambda r, n: r.sum() if n == 0 else (r * r).sum() if n == 1 else r.max()  # noqa: E731
        want = [stat(got["res_U"], normU), np.abs(got["AC_u"] * got["u"]).sum(), stat(got["res_V"], normV),
                np.abs(got["AC_v"] * got["v"]).sum(), np.abs(got["res_Continuity"]).sum()]
        np.testing.assert_allclose(out["sums"].cpu().numpy(), want, rtol=1e-10)


def test_residual_static_rejects_sizes_beyond_its_scratch():
    mesh, got = _solved_case()
    dev = {k: torch.from_numpy(np.ascontiguousarray(mesh[k])).cuda()
           for k in ("cellFaceStart", "cellFaceIDs", "faceOwner", "faceNeighbor")}
    dev.update({k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in got.items()})
    out = {k: torch.zeros(8, dtype=torch.float64, device="cuda") for k in ("resU", "resV", "resC", "sums")}
    st, msg = _call(mesh, dev, out, 0, 0, n_cells=4194304 + 1)
    assert st == abi.E_ARG and "static scratch limit" in msg
