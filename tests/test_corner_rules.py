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
    rules = {"cx": {}, "cy": {}, "bx": {}, "by": {}, "x3": {}, "x2": {}, "y3": {}, "y2": {}}
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


# ---------------------------------------------------------------- launch sets
# The kernels launch some passes over fewer points than the reference's
# stencils cover, relying on where the corner rules can apply.  These tests
# check those assumptions against the rules themselves (n = 12, h = 3).
S, E = 3, 14  # compute domain [S, E] in both directions


def test_corner_fill_launch_sets_cover_every_rule_point(device_rules):
    # c_sw launches its corner fills over i in {s-3..s-1, e+1..e+3} x j in
    # {js-1, je+1} (x rules) and the transpose (y rules)
    xs = {S - 3, S - 2, S - 1, E + 1, E + 2, E + 3}
    x_set = {(i, j) for i in xs for j in (S - 1, E + 1)}
    y_set = {(i, j) for i in (S - 1, E + 1) for j in xs}
    assert set(device_rules["x3"]) <= x_set and set(device_rules["x2"]) <= x_set
    assert set(device_rules["y3"]) <= y_set and set(device_rules["y2"]) <= y_set
    # fill_bgrid launches over the four 3 x 3 blocks
    bi = {S - 3, S - 2, S - 1, E + 2, E + 3, E + 4}
    blocks = {(i, j) for i in bi for j in bi}
    assert set(device_rules["bx"]) <= blocks and set(device_rules["by"]) <= blocks


def _deln_reads(lo, cx, cy):
    """(point, read) pairs of one del-n flux pass with lo halo rows."""
    out = []
    for i in range(S - lo, E + 2 + lo):
        for j in range(S - lo, E + 2 + lo):
            if i < E + 2 + lo and j < E + 1 + lo:
                out += [((i, j), cx.get(p, p)) for p in ((i - 1, j), (i, j))]
            if i < E + 1 + lo and j < E + 2 + lo:
                out += [((i, j), cy.get(p, p)) for p in ((i, j - 1), (i, j))]
    return out


@pytest.mark.parametrize("nmax", [1, 2, 3])
def test_fused_del_n_reads_stay_where_the_reference_computes_d2(device_rules, nmax):
    # delnflux_nosg computes d2 on the fly: every d2 point a pass reads
    # (after the corner mapping) must lie where the reference's d2 stencil
    # computed it, [s-1-nmax, e+2+nmax) for the first pass and
    # [s-nt-1, e+nt+2) for the later pass with nt halo rows
    cx, cy = device_rules["cx"], device_rules["cy"]

    def inside(p, lo_, hi_):
        return lo_ <= p[0] < hi_ and lo_ <= p[1] < hi_

    assert all(inside(r, S - 1 - nmax, E + 2 + nmax) for _, r in _deln_reads(nmax, cx, cy))
    for it in range(nmax):
        nt = nmax - 1 - it
        assert all(inside(r, S - nt - 1, E + nt + 2) for _, r in _deln_reads(nt, cx, cy))


def test_del_n_corner_fast_path_condition(device_rules):
    # a flux point skips the corner mapping unless i and j are both within
    # one point of the tile's edge rows; no read of a skipped point maps
    cx, cy = device_rules["cx"], device_rules["cy"]
    for (i, j), _ in _deln_reads(3, {}, {}):
        near = (i <= S or i >= E + 1) and (j <= S or j >= E + 1)
        if near:
            continue
        for p in ((i - 1, j), (i, j)):
            assert p not in cx
        for p in ((i, j - 1), (i, j)):
            assert p not in cy
