"""The closed-form halo sources of the CUDA gather (csrc/halo.cuh), compiled
for the host, against the package's gather tables, which the geometric halo
tests check against the cube's geometry."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from fv3core_b200 import halo_map as hm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3


@pytest.fixture(scope="module", params=[12, 7])
def device_map(request, tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    exe = str(tmp_path_factory.mktemp("halo") / "dump")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "native", "halo_dump.cpp")])
    out = subprocess.check_output([exe, str(request.param)], text=True)
    rows = {}
    misses = []
    for line in out.split("\n"):
        if not line:
            continue
        parts = line.split()
        if parts[0] == "miss":
            misses.append(parts)
            continue
        kind, comp, t, i, j, st, si, sj, sc, sg = parts[0], *map(int, parts[1:])
        rows.setdefault((kind, comp), {})[(t, i, j)] = (st, si, sj, sc, sg)
    return request.param, rows, misses


def test_no_misses(device_map):
    assert device_map[2] == []


@pytest.mark.parametrize("kind,s,nh", [("scalar3", 1, 3), ("scalar2", 1, 2), ("corner3", 0, 3)])
def test_scalar(device_map, kind, s, nh):
    n, rows, _ = device_map
    table = hm.scalar_table(n, H, s, s, nh)
    expect = {(r[0], r[1], r[2]): (r[3], r[4], r[5]) for r in table}
    got = {k: v[:3] for k, v in rows[(kind, 0)].items()}
    assert got == expect


@pytest.mark.parametrize("kind,xs,ys", [("dgrid", (1, 0), (0, 1)), ("cgrid", (0, 1), (1, 0))])
def test_vector(device_map, kind, xs, ys):
    n, rows, _ = device_map
    tables = hm.vector_tables(n, H, xs, ys, H)
    for comp in (0, 1):
        expect = {(r[0], r[1], r[2]): (r[3], r[4], r[5], r[6], r[7]) for r in tables[comp]}
        assert rows[(kind, comp)] == expect


def test_interface_sync(device_map):
    n, rows, _ = device_map
    table = hm.interface_sync_tables(n, H)
    expect = {}
    for r in table:
        expect.setdefault((r[1]), {})[(r[0], r[2], r[3])] = (r[4], r[6], r[7], r[5], r[8])
    for comp in (0, 1):
        assert rows[("sync", comp)] == expect[comp]
