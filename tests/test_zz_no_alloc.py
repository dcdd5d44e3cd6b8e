"""axisim_residual_static: the allocation-free residual entry point.

Some callers cannot allocate device memory at the point where they want the
residuals: a host whose GPU memory is all held by another allocator (or capped),
or a monitoring hook inside a time-critical loop where cudaMalloc/cudaFree would
stall the device. This entry point keeps its scratch in a fixed static device
array, so these tests check, besides the numbers, that a call allocates
nothing and that its error paths (bad indices, sizes beyond the scratch, host
pointers, a capturing stream) leave the next call clean.

Its inputs are the momentum systems, fields and face mass fluxes that a solve
left behind (read back through axisim_get_field); its per-cell outputs must
equal the residual arrays that the solve's own residual step wrote and the
oracle's after the same iterations, and its sums the sums of those arrays, on
two calls in a row (the second one reusing the static scratch the first left
behind).
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

NAMES = ("AF_u", "AC_u", "AC_v", "b_u", "b_v", "u", "v", "mDot", "res_U", "res_V", "res_Continuity")


def _solved_case(with_oracle=False):
    case = cases.expansion(scale=1 / 8, max_iter=30, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    s = abi.Solver(mesh, case.bc_fields(), case.settings)
    s.solve()
    got = {n: s.get(n) for n in NAMES}
    s.close()
    orc = None
    if with_oracle:
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
        import oracle
        o = oracle.Oracle(mesh, case.bc_fields(), case.settings)
        o.run()
        orc = {n: o.get(n) for n in ("res_U", "res_V", "res_Continuity", "AC_u", "AC_v", "u", "v")}
        o.close()
    return mesh, got, orc


def _device_inputs(mesh, got):
    dev = {k: torch.from_numpy(np.ascontiguousarray(mesh[k])).cuda()
           for k in ("cellFaceStart", "cellFaceIDs", "faceOwner", "faceNeighbor")}
    dev.update({k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in got.items()})
    return dev


def _outputs(n):
    out = {k: torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for k in ("resU", "resV", "resC")}
    out["sums"] = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
    return out


def _call(mesh, dev, out, normU, normV, n_cells=None, ptr=None):
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    p = (lambda k: dev[k].data_ptr()) if ptr is None else ptr
    st = abi.lib().axisim_residual_static(
        int(mesh["nCells"]) if n_cells is None else n_cells, int(mesh["nFaces"]), len(mesh["cellFaceIDs"]),
        p("cellFaceStart"), p("cellFaceIDs"), p("faceOwner"), p("faceNeighbor"), p("AF_u"), p("AC_u"), p("AC_v"),
        p("b_u"), p("b_v"), p("u"), p("v"), p("mDot"), normU, normV, out["resU"].data_ptr(), out["resV"].data_ptr(),
        out["resC"].data_ptr(), out["sums"].data_ptr(), stream, err, len(err))
    return st, err.value.decode()


def _stat(r, n):
    return r.sum() if n == 0 else (r * r).sum() if n == 1 else r.max()


def test_residual_static_matches_solver_and_oracle_twice_without_allocating():
    mesh, got, orc = _solved_case(with_oracle=True)
    assert np.abs(got["res_U"]).max() > 0 and np.abs(got["res_Continuity"]).max() > 0
    dev = _device_inputs(mesh, got)
    N = int(mesh["nCells"])
    outs = [_outputs(N) for _ in range(3)]
    torch.cuda.synchronize()
    # the first call of the process loads the library's module and looks up the
    # scratch address; every call after it must leave free device memory as it was
    st, msg = _call(mesh, dev, outs[0], 0, 1)
    assert st == abi.OK, msg
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for (normU, normV), out in zip(((0, 1), (2, 1)), outs[1:]):
        st, msg = _call(mesh, dev, out, normU, normV)
        assert st == abi.OK, msg
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, "a call changed the free device memory"
        resU, resV, resC = (out[k].cpu().numpy() for k in ("resU", "resV", "resC"))
        for mine, key in ((resU, "res_U"), (resV, "res_V"), (resC, "res_Continuity")):
            np.testing.assert_allclose(mine, got[key], rtol=1e-12, atol=1e-300)
            np.testing.assert_allclose(mine, orc[key], rtol=1e-12, atol=1e-300)
        want = [_stat(orc["res_U"], normU), np.abs(orc["AC_u"] * orc["u"]).sum(), _stat(orc["res_V"], normV),
                np.abs(orc["AC_v"] * orc["v"]).sum(), np.abs(orc["res_Continuity"]).sum()]
        np.testing.assert_allclose(out["sums"].cpu().numpy(), want, rtol=1e-10)


def test_residual_static_reports_bad_indices_then_runs_clean():
    mesh, got, _ = _solved_case()
    dev = _device_inputs(mesh, got)
    N = int(mesh["nCells"])
    bad = dict(dev)
    ids = dev["cellFaceIDs"].clone()
    ids[5] = int(mesh["nFaces"])  # one slot names a face past the end: skipped, counted
    bad["cellFaceIDs"] = ids
    out = _outputs(N)
    st, msg = _call(mesh, bad, out, 0, 0)
    assert st == abi.E_MESH and msg.startswith("1 cells"), (st, msg)
    # the next clean call starts from zeroed counters
    out = _outputs(N)
    st, msg = _call(mesh, dev, out, 0, 0)
    assert st == abi.OK and msg == "", (st, msg)
    np.testing.assert_allclose(out["resU"].cpu().numpy(), got["res_U"], rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(out["sums"].cpu().numpy()[4], np.abs(got["res_Continuity"]).sum(), rtol=1e-10)


def test_residual_static_rejects_host_pointers_and_capturing_streams():
    mesh, got, _ = _solved_case()
    dev = _device_inputs(mesh, got)
    N = int(mesh["nCells"])
    host = {k: np.ascontiguousarray(v) for k, v in got.items()}
    host.update({k: np.ascontiguousarray(mesh[k]) for k in ("cellFaceStart", "cellFaceIDs", "faceOwner",
                                                             "faceNeighbor")})
    out = _outputs(N)
    st, msg = _call(mesh, dev, out, 0, 0, ptr=lambda k: host[k].ctypes.data)
    assert st == abi.E_ARG and "device pointer" in msg, (st, msg)
    # a call on a stream under capture is refused before it touches the stream
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=side, capture_error_mode="thread_local"):
            out["sums"].zero_()
            st, msg = _call(mesh, dev, out, 0, 0)
    assert st == abi.E_ARG and "captured" in msg, (st, msg)
    del g
    out = _outputs(N)
    st, msg = _call(mesh, dev, out, 0, 0)
    assert st == abi.OK, msg
    np.testing.assert_allclose(out["resV"].cpu().numpy(), got["res_V"], rtol=1e-12, atol=1e-300)


def test_residual_static_rejects_sizes_beyond_its_scratch():
    mesh, got, _ = _solved_case()
    dev = _device_inputs(mesh, got)
    out = {k: torch.zeros(8, dtype=torch.float64, device="cuda") for k in ("resU", "resV", "resC", "sums")}
    st, msg = _call(mesh, dev, out, 0, 0, n_cells=4194304 + 1)
    assert st == abi.E_ARG and "static scratch limit" in msg
