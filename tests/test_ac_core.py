"""The AC lanes' complex replay and solves (egspice_b200/csrc/lane_ac_core.cuh,
what k_ac runs per lane) built for the host by tests/ac_host.cpp, on CPU,
against dense complex solves (numpy): forward solves Y x = b and adjoint
(transpose) solves Y^T z = b for several right-hand sides and frequencies,
on random patterns and on the op-amp's G and C at its operating points
(branch rows with zero diagonals, so the tape pivots off the diagonal). The
GPU runs the same code through espl_ac_solve in tests/test_gpu_parity.py."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from egspice_b200 import abi, decks
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
f64p = C.POINTER(C.c_double)
u32p = C.POINTER(C.c_uint32)


@pytest.fixture(scope="module")
def dev_ac(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("ac") / "libac_host.so")
    src = [os.path.join(HERE, "ac_host.cpp"), os.path.join(HERE, "..", "egspice_b200", "csrc", "tape.cpp")]
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out] + src, check=True)
    f = C.CDLL(out).dev_ac
    f.argtypes = [C.c_uint32, u32p, u32p, C.c_uint32, f64p, f64p, f64p, C.c_uint32, f64p, f64p, C.c_uint32,
                  C.c_uint32, u32p, C.c_uint32, f64p, f64p]
    f.restype = C.c_int

    def run(col_ptr, row_idx, g, c, omega, rhs, rows, adjoint):
        """g, c: [nnz, P] (lanes interleaved); rhs complex [n_rhs, n]."""
        n = len(col_ptr) - 1
        P = g.shape[1]
        cp = np.ascontiguousarray(col_ptr, dtype=np.uint32)
        ri = np.ascontiguousarray(row_idx, dtype=np.uint32)
        g = np.ascontiguousarray(g, dtype=np.float64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        om = np.ascontiguousarray(omega, dtype=np.float64)
        b = np.atleast_2d(rhs)
        br, bi = np.ascontiguousarray(b.real), np.ascontiguousarray(b.imag)
        rw = np.ascontiguousarray(rows, dtype=np.uint32)
        re = np.zeros((P, len(om), len(b), len(rw)))
        im = np.zeros_like(re)
        assert f(n, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p), P, g.ctypes.data_as(f64p),
                 c.ctypes.data_as(f64p), om.ctypes.data_as(f64p), len(om), br.ctypes.data_as(f64p),
                 bi.ctypes.data_as(f64p), len(b), int(adjoint), rw.ctypes.data_as(u32p), len(rw),
                 re.ctypes.data_as(f64p), im.ctypes.data_as(f64p)) == 0
        return re + 1j * im

    return run


def _dense(col_ptr, row_idx, vals):
    n = len(col_ptr) - 1
    cols = np.repeat(np.arange(n), np.diff(np.asarray(col_ptr, dtype=np.int64)))
    a = np.zeros((n, n))
    np.add.at(a, (np.asarray(row_idx, dtype=np.int64), cols), vals)
    return a


def _check(dev_ac, col_ptr, row_idx, g, c, omega, rhs, rows, rtol):
    n = len(col_ptr) - 1
    for adjoint in (False, True):
        got = dev_ac(col_ptr, row_idx, g, c, omega, rhs, rows, adjoint)
        for l in range(g.shape[1]):
            G, Cm = _dense(col_ptr, row_idx, g[:, l]), _dense(col_ptr, row_idx, c[:, l])
            for f, w in enumerate(omega):
                Y = G + 1j * w * Cm
                for e, b in enumerate(np.atleast_2d(rhs)):
                    want = np.linalg.solve(Y.T if adjoint else Y, b)[list(rows)]
                    scale = np.abs(np.linalg.solve(Y.T if adjoint else Y, b)).max()
                    np.testing.assert_allclose(got[l, f, e], want, rtol=rtol, atol=rtol * scale,
                                               err_msg=f"adjoint={adjoint} lane {l} f {f} rhs {e}")


def test_random_patterns(dev_ac):
    rng = np.random.default_rng(3)
    for trial in range(20):
        n = int(rng.integers(2, 25))
        mask = rng.uniform(size=(n, n)) < 0.25
        np.fill_diagonal(mask, True)
        cols = [np.flatnonzero(mask[:, j]) for j in range(n)]
        col_ptr = np.concatenate([[0], np.cumsum([len(x) for x in cols])])
        row_idx = np.concatenate(cols)
        nnz, P = len(row_idx), 4
        diag = np.concatenate([x == j for j, x in enumerate(cols)])
        g = rng.normal(size=(nnz, P)) + np.where(diag, 4.0 * n, 0.0)[:, None]
        c = rng.normal(size=(nnz, P)) * 1e-3
        rhs = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
        _check(dev_ac, col_ptr, row_idx, g, c, [0.0, 10.0, 1e3], rhs, np.arange(n), 1e-10)


def test_opamp_planes(dev_ac, oracle):
    """The op-amp's G and C (the oracle's device models) at each lane's
    operating point: voltage-source branch rows have zero diagonals."""
    net = decks.miller_opamp(4)
    x, r = oracle.op_ladder(net, abi.newton_opts())
    assert (r[:, 0] == 1).all()
    nnz = len(net.row_idx)
    g = np.zeros((nnz, net.lanes))
    c = np.zeros((nnz, net.lanes))
    cn = po.CNet(net)
    for l in range(net.lanes):
        gl, cl = np.zeros(nnz), np.zeros(nnz)
        xl = np.ascontiguousarray(x[l])
        assert po.lib().orc_planes(C.byref(cn.c), l, xl.ctypes.data_as(f64p), gl.ctypes.data_as(f64p),
                                   cl.ctypes.data_as(f64p)) == 0
        g[:, l], c[:, l] = gl, cl
    n = net.n
    e = np.zeros((2, n), dtype=complex)
    e[0, net.node("out")] = 1.0                                           # the output node
    e[1, [b for b in net.batches if b.kind == decks.VSRC][0].term[0, 2]] = 1.0  # a branch row
    _check(dev_ac, net.col_ptr, net.row_idx, g, c, np.logspace(2, 10, 5) * 2 * np.pi, e, np.arange(n), 1e-8)
