"""OpenFOAM case export (axisim/foam.py) against the reference's own exporter.

tests/golden/foam_*.json hold every file of a case exported by the
reference's manager/source/file_converter.cpp (compiled unchanged and driven
by oracle/ref_build/foam_driver.cpp; tests/golden/make_foam_golden.py). The
export here must reproduce each file byte for byte: the blockMeshDict (welded
vertex labels, gradings, patches named and de-collided from the group names),
the revolved polyMesh of a triangle mesh, the system and constant
dictionaries, and the 0/ field files.
"""
import json
import os
import sys

import pytest

from axisim import foam

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_foam_golden  # noqa: E402

CASES = make_foam_golden.foam_cases()


@pytest.mark.parametrize("name,spec", CASES, ids=[n for n, _ in CASES])
def test_export_matches_reference_byte_for_byte(name, spec, tmp_path):
    gold = json.load(open(os.path.join(HERE, "golden", "foam_" + name + ".json")))["files"]
    spec = dict(spec)
    files = foam.save_foam_case(str(tmp_path), spec.pop("groups"), spec.pop("settings"), **spec)
    assert sorted(files) == sorted(gold)
    for rel in files:
        got = open(tmp_path / rel, "rb").read().decode("utf-8")
        if got != gold[rel]:
            a, b = got.splitlines(), gold[rel].splitlines()
            first = next((i for i, (x, y) in enumerate(zip(a, b)) if x != y), min(len(a), len(b)))
            pytest.fail(f"{rel} differs at line {first + 1}: {a[first:first + 1]} vs {b[first:first + 1]}")


def test_numbers_and_names():
    assert foam.foam_number(0.05) == "0.05" and foam.foam_number(1 / 3) == "0.3333333333333333"
    assert foam.foam_number(0.1 + 0.2) == "0.30000000000000004"

    class G:
        def __init__(self, gid, name):
            self.id, self.name = gid, name
    assert foam.patch_name(G(1, "Outer wall (r=R)")) == "Outer_wall_r_R"
    assert foam.patch_name(G(7, "")) == "group7"
    assert foam.patch_name(G(2, "3 walls!")) == "group2_3_walls"
