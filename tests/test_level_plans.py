"""The host plans of the large-template LU (egspice_b200/csrc/tape.h
StreamPlan and ColPlan) on power-grid meshes: built for the host from
tape.cpp (tests/plans_host.cpp) and checked for every invariant the
streamed solves and the level-grouped refactor rely on (chunk shapes and
alignment for the bulk copies, each chunk's plan, rows in level order with
their entries, chunk-local columns, level ends; every column once, a level
reading only earlier levels, group counts, the U entry stream). The chunk
sizes are the kernels' (lane_levels.cuh)."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from egspice_b200 import decks

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "egspice_b200", "csrc")


def kernel_constants():
    src = open(os.path.join(CSRC, "lane_levels.cuh")).read()
    m = re.search(r"kRingSlots = (\d+), kRingChunk = (\d+), kRingRows = (\d+);", src)
    g = re.search(r"kRefGroups = (\d+);", open(os.path.join(CSRC, "lane_engine.cuh")).read())
    slots, chunk, rows = (int(x) for x in m.groups())
    return chunk, rows, slots, int(g.group(1))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("plans") / "plans_host")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, "-o", out, os.path.join(HERE, "plans_host.cpp"),
                    os.path.join(CSRC, "tape.cpp")], check=True, capture_output=True)
    return out


@pytest.mark.parametrize("side", [16, 40, 90])
def test_plans_of_a_mesh(oracle, checker, tmp_path, side):
    net = decks.power_grid(1, side=side, loads=min(400, 2 * side))
    cp, ri = np.asarray(net.col_ptr, np.uint32), np.asarray(net.row_idx, np.uint32)
    rng = np.random.default_rng(side)
    v = np.zeros(net.nnz)
    for j in range(net.n):
        for p in range(cp[j], cp[j + 1]):
            v[p] = 4.0 if ri[p] == j else -rng.uniform(0.5, 1.0)
    q = np.asarray(oracle.order(cp, ri), np.uint32)
    files = []
    for name, a in (("cp", cp), ("ri", ri), ("v", v), ("q", q)):
        f = str(tmp_path / f"{name}.bin")
        a.tofile(f)
        files.append(f)
    chunk, rows, slots, groups = kernel_constants()
    r = subprocess.run([checker] + files + [str(chunk), str(rows), str(slots), str(groups)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "forward:" in r.stdout and "backward:" in r.stdout and "columns:" in r.stdout
