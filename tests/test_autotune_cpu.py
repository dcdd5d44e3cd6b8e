"""Selection rule of the multigrid launch-shape autotuner (host code,
axisim::pickBlock): the default block size stays unless another candidate is
faster by more than the tolerance; unmeasured candidates are never chosen."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "axisim-software_b200", "csrc")

DRIVER = r'''
#include <cmath>
#include <cstdio>
#include "host_prep.hpp"
int main() {
    const std::vector<int> c = {64, 128, 256};
    const double nan = std::nan("");
    struct Case { std::vector<double> t; int def; double tol; };
    const Case cases[] = {
        {{10.0, 10.0, 10.0}, 2, 0.03},   // equal: keep the default
        {{9.8, 9.9, 10.0}, 2, 0.03},     // 2 % faster: within tolerance, keep the default
        {{9.0, 9.5, 10.0}, 2, 0.03},     // 10 % faster: switch to 64
        {{9.5, 9.0, 10.0}, 2, 0.03},     // 128 fastest
        {{9.0, 9.5, nan}, 2, 0.03},      // default unmeasured: the fastest measured
        {{-1.0, 0.0, nan}, 2, 0.03},     // nothing measured: the default
        {{nan, nan, nan}, 7, 0.03},      // nothing measured, default out of range: the first
        {{5.0, 12.0, 10.0}, 2, 1.5},     // wide tolerance keeps the default
    };
    for (const Case& k : cases) std::printf("%d\n", axisim::pickBlock(c, k.t, k.def, k.tol));
    return 0;
}
'''


def test_pick_block_rule(tmp_path):
    src = tmp_path / "pick.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "pick"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, "-I", os.path.join(ROOT, "include"), str(src),
                        os.path.join(CSRC, "host_prep.cpp"), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0 and "not found" in r.stderr:
        pytest.skip("no host C++ compiler")
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0
    assert [int(x) for x in out.stdout.split()] == [2, 2, 0, 1, 0, 2, 0, 2]
