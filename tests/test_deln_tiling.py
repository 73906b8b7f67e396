"""Tiling of the fused del-n chain kernel (deln_chain_kernel in
fv3core_b200/csrc/transport.cuh), checked on the CPU by enumerating every
read of every pass.

A tile of TX = 32 - 2 nmax - 1 columns and 16 rows works in a window that
is the tile widened by nmax + 1 points (low sides) and nmax (high sides);
pass p computes fluxes on the tile widened by nmax - p points and d2 on the
window shrunk by p.  The kernel relies on:

* tiles it classes as fast have every pass's fluxes inside both flux
  regions (it writes them without region tests), no point of them meets the
  cube-corner condition (no corner mapping), and their window lies inside
  the arrays;
* in the other tiles, every d2 read of a later pass (p >= 1), corner-mapped
  where the reference maps it (delnflux.py copy_corners_x/y_nord), lies
  inside the window part computed for that pass and reads fluxes of the
  pass before that lie inside that pass's region (the host check
  deln_window_ok; where it fails the chain runs pass by pass);
* a pass-0 read mapped outside the window lies inside the arrays (the
  kernel reads damp q there from q).

The corner maps are the oracle's tables of the reference's copy rules,
which tests/test_corner_rules.py holds equal to the kernels' closed forms.
"""
import pytest

from oracle import corners as oc
from oracle._util import Tile

TY = 16


def _maps(n):
    t = Tile(n, 1)
    mx = {(i, j): (i + di, j + dj) for (i, j), (di, dj) in oc._copy_rules_x(t)}
    my = {(i, j): (i + di, j + dj) for (i, j), (di, dj) in oc._copy_rules_y(t)}
    return t, mx, my


def _check(n, nmax):
    t, mx, my = _maps(n)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    m = t.m
    tx = 32 - 2 * nmax - 1
    wy = TY + 2 * nmax + 1

    def fxr(lo, i, j):
        return s - lo <= i < e + 2 + lo and js - lo <= j < je + 1 + lo

    def fyr(lo, i, j):
        return s - lo <= i < e + 1 + lo and js - lo <= j < je + 2 + lo

    def corner(i, j):
        return (i <= s or i >= e + 1) and (j <= js or j >= je + 1)

    problems = []
    n_fast = n_slow = 0
    for i0 in range(s, e + 2, tx):
        for j0 in range(js, je + 2, TY):
            i1, j1 = min(i0 + tx, e + 2), min(j0 + TY, je + 2)
            wi0, wj0 = i0 - nmax - 1, j0 - nmax - 1
            near_x = i0 - nmax <= s or i1 - 1 + nmax >= e + 1
            near_y = j0 - nmax <= js or j1 - 1 + nmax >= je + 1
            slow = i1 == e + 2 or j1 == je + 2 or (near_x and near_y)
            if not slow:
                n_fast += 1
                if not (wi0 >= 0 and wj0 >= 0 and wi0 + 32 <= m and wj0 + wy <= m):
                    problems.append(("fast window outside the arrays", i0, j0))
                for p in range(nmax + 1):
                    lo = nmax - p
                    for i in range(i0 - lo, i1 + lo):
                        for j in range(j0 - lo, j1 + lo):
                            if not (fxr(lo, i, j) and fyr(lo, i, j)) or corner(i, j):
                                problems.append(("fast tile point", i0, j0, p, i, j))
                continue
            n_slow += 1
            for p in range(nmax + 1):
                lo = nmax - p
                for i in range(i0 - lo, i1 + lo):
                    for j in range(j0 - lo, j1 + lo):
                        c = corner(i, j)
                        for kind, region, mp in (("x", fxr, mx), ("y", fyr, my)):
                            if not region(lo, i, j):
                                continue
                            reads = [(i - 1, j), (i, j)] if kind == "x" else [(i, j - 1), (i, j)]
                            for q in reads:
                                ii, jj = mp.get(q, q) if c else q
                                xx, yy = ii - wi0, jj - wj0
                                if p == 0:
                                    inside = 0 <= xx < 32 and 0 <= yy < wy
                                    if not inside and not (0 <= ii < m and 0 <= jj < m):
                                        problems.append(("pass-0 read outside the arrays", i0, j0, i, j))
                                    continue
                                if not (p <= xx < 32 - p and p <= yy < wy - p):
                                    problems.append(("d2 read outside the window", i0, j0, p, i, j, ii, jj))
                                    continue
                                for a, b, reg in ((ii, jj, fxr), (ii + 1, jj, fxr), (ii, jj, fyr),
                                                  (ii, jj + 1, fyr)):
                                    if not reg(lo + 1, a, b):
                                        problems.append(("flux read outside its region", i0, j0, p, a, b))
    return problems, n_fast, n_slow


@pytest.mark.parametrize("nmax", [1, 2])
@pytest.mark.parametrize("n", [12, 24, 48, 96, 128, 192, 384])
def test_fused_chain_reads_stay_inside(n, nmax):
    problems, n_fast, n_slow = _check(n, nmax)
    assert not problems, problems[:5]
    if n >= 96:
        # most tiles take the path without region tests
        assert n_fast > n_slow


def test_fused_chain_reads_every_small_grid():
    """Every cube size from 4 to 64: the reads stay inside, so the fused
    kernel (not the pass-by-pass fallback) serves all of them."""
    for n in range(4, 65):
        for nmax in (1, 2):
            problems, _, _ = _check(n, nmax)
            assert not problems, (n, nmax, problems[:3])


def test_host_check_agrees_with_the_enumeration(tmp_path):
    """The library's own host check (deln_window_ok, compiled with nvcc for
    the host) accepts every grid with the 3-point halo that the enumeration
    above accepts (cube sizes 4 to 200), so the fused kernel serves them;
    with a 2-point halo it declines, and the chain runs pass by pass."""
    import os
    import shutil
    import subprocess

    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("no nvcc")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "deln_window_dump")
    subprocess.check_call([nvcc, "-std=c++17", "--expt-extended-lambda", "-O1", "-gencode",
                           "arch=compute_100a,code=sm_100a", "-o", exe,
                           os.path.join(root, "tests", "native", "deln_window_dump.cu")])
    ok = {}
    for line in subprocess.check_output([exe], text=True).split("\n"):
        if line:
            n, h, nmax, v = (int(x) for x in line.split())
            ok[(n, h, nmax)] = bool(v)
    for n in range(4, 201):
        for nmax in (1, 2):
            assert ok[(n, 3, nmax)], (n, nmax)
            assert not ok[(n, 2, nmax)], (n, nmax)
    for n in list(range(4, 41)) + [96, 128, 192]:
        for nmax in (1, 2):
            problems, _, _ = _check(n, nmax)
            assert not problems and ok[(n, 3, nmax)], (n, nmax)
