"""Newton's residual gate (src/solver/converger.zig residualGate :340-350)
on CPU: the reference's known-answer test for the lane gate
(src/solver/kernels/lane.zig:731-760: zero diagonals, residuals from 0 to
inf and NaN, a finite and an infinite floor) replayed on the kernels' gate
(egspice_b200/csrc/lane_gates.cuh built for the host by
tests/gates_host.cpp) and the oracle's, against a restatement of
residualGate."""
import ctypes as C
import math
import os
import shutil
import subprocess

import pytest

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
RELTOL, VNTOL = 1e-3, 1e-6  # src/core/numerics.zig defaults


def _max(a, b):
    """Zig's @max on floats: the other operand of a NaN."""
    if math.isnan(a):
        return b
    if math.isnan(b):
        return a
    return max(a, b)


def residual_gate(floor, diag, xi):
    s = 1.0 if abs(diag) == 0 else abs(diag)
    return _max(floor, 10.0 * s * (RELTOL * abs(xi) + VNTOL))


@pytest.fixture(scope="module")
def gates(tmp_path_factory, oracle):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("gates") / "libgates_host.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out, os.path.join(HERE, "gates_host.cpp")],
                   check=True)
    dev = C.CDLL(out).dev_residual_gate
    orc = po.lib().orc_residual_gate
    for f in (dev, orc):
        f.argtypes = [C.c_double] * 5
        f.restype = C.c_double
    return (lambda fl, d, x: dev(fl, RELTOL, VNTOL, d, x)), (lambda fl, d, x: orc(fl, RELTOL, VNTOL, d, x))


def test_reference_gate_cases(gates):
    dev, orc = gates
    N, n = 3, 4
    diag = [2, 0, 3, 1]
    residuals = [0.0, 1e-12, 1e-6, 0.25, math.inf, math.nan]
    passed = failed = 0
    for floor in (1e-9, math.inf):
        for trial, r in enumerate(residuals):
            x = [[(i + l) * 0.125 for l in range(N)] for i in range(n)]
            vals = [[0.0 if (i + l) % 2 == 0 else 2.5e-3 for l in range(N)] for i in range(n)]
            rhs = [[r if i == (trial + l) % n else 0.0 for l in range(N)] for i in range(n)]
            for l in range(N):
                want = all(abs(rhs[i][l]) <= residual_gate(floor, vals[diag[i]][l], x[i][l]) for i in range(n))
                for gate in (dev, orc):
                    got = all(abs(rhs[i][l]) <= gate(floor, vals[diag[i]][l], x[i][l]) for i in range(n))
                    assert got == want, (floor, r, l)
                passed += want
                failed += not want
    assert passed and failed  # both verdicts occur


@pytest.mark.parametrize("floor", [0.0, 1e-9, math.inf])
@pytest.mark.parametrize("diag", [0.0, -0.0, 2.5e-3, -7.0, 1e300, math.nan])
@pytest.mark.parametrize("xi", [0.0, -1.8, 1e-15, 1e12, math.inf, math.nan])
def test_gate_values_agree_bitwise(gates, floor, diag, xi):
    dev, orc = gates
    want = residual_gate(floor, diag, xi)
    for gate in (dev, orc):
        got = gate(floor, diag, xi)
        assert (math.isnan(got) and math.isnan(want)) or got == want
