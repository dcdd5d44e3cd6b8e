"""Host-side checks that need no GPU: the C ABI library loads and exports every
declared entry point, the C++ host preparation matches the oracle's
restatement of the reference, and the boundary defaults match boundary_func.cpp."""
import ctypes
import os
import re

import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    abi.build()
    return abi.lib()


def _declared():
    hdr = open(os.path.join(ROOT, "include", "axisim_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(axisim_[a-z0-9_]+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(abi.EXPORTS)
    assert lib.axisim_abi_version() == 1


def test_struct_layouts_match_reference_sizes():
    # ConfigSolver / ConfigSimple are static_assert'ed at 40 / 24 bytes (solver_struct.h:165, 238)
    assert ctypes.sizeof(abi.ConfigSolver) == 40
    assert ctypes.sizeof(abi.ConfigSimple) == 24


def _same_mesh(a, b):
    assert a["nCells"] == b["nCells"] and a["nFaces"] == b["nFaces"]
    for k in abi.MESH_KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("case", [cases.pipe(nr=12, nz=30), cases.expansion(scale=1 / 16),
                                  cases.expansion(scale=1 / 8, bias=1.3)], ids=["pipe", "expansion", "graded"])
def test_multiblock_matches_oracle_bitwise(lib, case):
    _same_mesh(abi.multiblock(case.blocks), oracle.multiblock(case.blocks))


def test_multiblock_geometry_invariants(lib):
    m = abi.multiblock(cases.expansion(scale=1 / 16).blocks)
    n = m["nCells"]
    assert m["status"] == 0
    # every cell of a quad mesh has four faces; interior faces appear in two cells
    assert np.all(np.diff(m["cellFaceStart"]) == 4)
    counts = np.bincount(m["cellFaceIDs"], minlength=m["nFaces"])
    interior = m["faceNeighbor"] >= 0
    assert np.all(counts[interior] == 2) and np.all(counts[~interior] == 1)
    # Pappus: volume = 2 pi r_c A2D, unit normals, total volume of the domain
    np.testing.assert_allclose(m["cellVolume"], 2 * np.pi * m["cellCenterR"] * m["cellArea2D"], rtol=1e-14)
    np.testing.assert_allclose(np.hypot(m["faceNormalZ"], m["faceNormalR"]), 1.0, rtol=1e-14)
    vol = np.pi * 0.002 ** 2 * 0.04 + np.pi * 0.006 ** 2 * 0.12
    np.testing.assert_allclose(m["cellVolume"].sum(), vol, rtol=1e-12)
    # boundary faces carry their group; interface faces none
    assert np.all(m["faceBoundaryGroupID"][interior] == -1)
    assert set(np.unique(m["faceBoundaryGroupID"][~interior])) == {0, 1, 2, 3}
    assert n == cases.cell_count(cases.expansion(scale=1 / 16))


def test_nonconformal_seam_drops_interfaces(lib):
    blocks = [cases.block(0, 0, (1.0, 4), (1.0, 3)), cases.block(1.0, 0, (1.0, 4), (1.0, 5))]
    a, b = abi.multiblock(blocks), oracle.multiblock(blocks)
    assert a["status"] == 1 and b["status"] == 1
    _same_mesh(a, b)
    assert np.all(a["faceNeighbor"][a["faceOwner"] < 12] != 12)


def test_resolve_bc_matches_boundary_defaults(lib):
    # (boundaryType, variable) -> default BCType, boundary_func.cpp:117-201
    for bt in range(5):
        for var, key in enumerate(("u", "v", "p", "T", "C")):
            t, v, p = abi.resolve_bc(bt, var)
            assert t == cases.default_bc_type(bt, key), (bt, var)
            assert v == 0.0 and p == 0
            # a user value only sticks where the variable is editable (boundary_func.cpp:333-378)
            t2, v2, _ = abi.resolve_bc(bt, var, (cases.DIRICHLET, 1.5))
            if cases.variable_editable(key, bt):
                assert (t2, v2) == (cases.DIRICHLET, 1.5)
            else:
                assert (t2, v2) == (t, 0.0)
    t, v, p = abi.resolve_bc(cases.VELOCITY_INLET, 0, (cases.PULSATILE, 0.3))
    assert (t, v, p) == (cases.DIRICHLET, 0.3, 1)


def test_python_bc_resolution_matches_library(lib):
    case = cases.pulsatile_expansion(scale=1 / 32)
    for var, key in enumerate(("u", "v", "p")):
        f = case.bc_fields()[key]
        for g in case.groups:
            user = g.bcs.get(key)
            t, v, p = abi.resolve_bc(g.btype, var, None if user is None else (user[0], user[1]))
            assert f["type"][g.id] == t and f["value"][g.id] == v and f["puls"][g.id] == p


def test_create_without_device_is_a_status_not_a_crash(lib):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = lib.axisim_create(None, ctypes.byref(h))
    assert st == abi.E_CUDA and not h.value


def test_cpp_adapter_compiles_and_links(lib, tmp_path):
    """The header-only C++ adapter (reference Solver member names) builds against the library."""
    src = tmp_path / "use_adapter.cpp"
    src.write_text(r'''
#include "axisim_solver.hpp"
#include <cstdio>
int main() {
    axisim_fluid f{1000.0, 1e-3, 4180.0, 0.6, 3e-9};
    try {
        axisim_b200::Solver s(f);
        s.configSimple.maxIter = 10;
        std::string why;
        std::printf("can continue: %d\n", (int)s.canContinue(&why));
    } catch (const std::exception& e) {
        std::printf("no device: %s\n", e.what());
    }
    return 0;
}
''')
    exe = tmp_path / "use_adapter"
    pkg = os.path.join(ROOT, "axisim-software_b200")
    r = __import__("subprocess").run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                                      "-L", pkg, "-laxisim_b200", "-Wl,-rpath," + pkg, "-lpthread"],
                                     capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = __import__("subprocess").run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0
