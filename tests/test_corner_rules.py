"""The closed-form cube-corner rules of the CUDA kernels (csrc/corners.cuh),
compiled for the host, against the oracle's rule tables, which restate the
reference's per-point region lists (fv3core/utils/corners.py)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import corners as oc
from oracle._util import Tile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def device_rules(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    exe = str(tmp_path_factory.mktemp("corners") / "dump")
    subprocess.check_call(
        ["g++", "-O1", "-std=c++17", "-I/usr/local/cuda/include", "-o", exe,
         os.path.join(ROOT, "tests", "native", "corner_rules_dump.cpp")]
    )
    out = subprocess.check_output([exe], text=True)
    rules = {"cx": {}, "cy": {}, "bx": {}, "by": {}}
    for line in out.split("\n"):
        if line:
            k, i, j, si, sj = line.split()
            rules[k][(int(i), int(j))] = (int(si), int(sj))
    return rules


def _oracle_copy_rules(direction):
    t = Tile(12, 8)
    rules = oc._copy_rules_x(t) if direction == "x" else oc._copy_rules_y(t)
    return {(i, j): (i + di, j + dj) for (i, j), (di, dj) in rules}


@pytest.mark.parametrize("direction", ["x", "y"])
def test_copy_corners(device_rules, direction):
    assert device_rules["c" + direction] == _oracle_copy_rules(direction)


@pytest.mark.parametrize("direction", ["x", "y"])
def test_bgrid_corners(device_rules, direction):
    from oracle.d_sw import _fill_corners_bgrid

    t = Tile(12, 8)
    # recover the oracle's table by filling a field of unique ids
    q = np.arange(t.m * t.m, dtype=np.float64).reshape(t.m, t.m, 1)
    q2 = q.copy()
    _fill_corners_bgrid(t, q2, direction, 0, 1)
    changed = np.argwhere(q2[:, :, 0] != q[:, :, 0])
    table = {}
    for i, j in changed:
        src = int(q2[i, j, 0])
        table[(int(i), int(j))] = (src // t.m, src % t.m)
    dev = {k: v for k, v in device_rules["b" + direction].items() if v != k}
    assert dev == table
