"""ctypes binding of the oracle library (test infrastructure only).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
the product package never imports it.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess
from typing import Optional, Sequence, Tuple

import numpy as np

from egspice_b200.abi import (CNet, MeasPass, NetlistC, NewtonOpts, OrcNewtonResult, StepReport, TranOpts, f64p,
                              u32p)
from egspice_b200.decks import Netlist

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liborc.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_tran_meas.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.POINTER(MeasPass), C.c_uint32,
                                    f64p, f64p, f64p, C.c_void_p, C.c_uint32]
        L.orc_tran_meas.restype = C.c_int
        L.orc_meas_series.argtypes = [C.POINTER(MeasPass), f64p, f64p, C.c_uint32, f64p, f64p]
        L.orc_meas_series.restype = C.c_int
        L.orc_meas_table.argtypes = [C.POINTER(MeasPass), C.c_uint32, f64p, f64p, C.c_uint32, C.c_uint32, f64p, f64p]
        L.orc_meas_table.restype = C.c_int
        L.orc_planes.argtypes = [C.c_void_p, C.c_uint32, f64p, f64p, f64p]
        L.orc_planes.restype = C.c_int
        L.orc_op_ladder.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, f64p, C.c_void_p, C.c_uint32]
        L.orc_op_ladder.restype = C.c_int
        L.orc_order.argtypes = [C.c_uint32, u32p, u32p, u32p]
        L.orc_order.restype = C.c_int
        L.orc_order_ws.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_size_t]
        L.orc_order_ws.restype = C.c_int
        L.orc_amd_ws.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_size_t]
        L.orc_amd_ws.restype = C.c_int
        L.orc_ws_size.argtypes = [C.c_size_t, C.c_size_t]
        L.orc_ws_size.restype = C.c_size_t
        L.orc_chol_count.argtypes = [C.c_uint32, u32p, u32p, u32p, C.c_uint64]
        L.orc_chol_count.restype = C.c_uint64
        L.orc_lu_new.argtypes = [C.c_uint32, u32p, u32p]
        L.orc_lu_new.restype = C.c_void_p
        L.orc_lu_free.argtypes = [C.c_void_p]
        L.orc_lu_set_caps.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_double]
        L.orc_lu_factor.argtypes = [C.c_void_p, u32p, u32p, f64p, C.c_double]
        L.orc_lu_factor.restype = C.c_int
        L.orc_lu_refactor.argtypes = [C.c_void_p, u32p, f64p, C.c_double]
        L.orc_lu_refactor.restype = C.c_int
        L.orc_lu_solve.argtypes = [C.c_void_p, f64p, f64p]
        L.orc_lu_solve_t.argtypes = [C.c_void_p, f64p, f64p]
        L.orc_lu_tape.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_op_lanes.argtypes = [C.POINTER(NetlistC), C.c_uint32, C.c_uint32, C.POINTER(NewtonOpts), f64p, f64p,
                                   C.POINTER(OrcNewtonResult), C.c_uint32]
        L.orc_op_lanes.restype = C.c_int
        L.orc_tran_lanes.argtypes = [C.POINTER(NetlistC), C.c_uint32, C.c_uint32, C.POINTER(TranOpts), u32p,
                                     C.c_uint32, C.c_uint32, f64p, f64p, C.POINTER(StepReport), C.c_uint32,
                                     C.c_double, C.c_double, f64p, C.c_uint32]
        L.orc_tran_lanes.restype = C.c_int
        L.orc_device_probe.argtypes = [C.POINTER(NetlistC), C.c_uint32, C.c_uint32, C.c_uint32, f64p, f64p, f64p,
                                       f64p, f64p]
        L.orc_device_probe.restype = C.c_int
        L.orc_set_polish.argtypes = [C.c_uint32]
        L.orc_set_polish.restype = None
        L.orc_pnjlim.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.orc_pnjlim.restype = C.c_double
        L.orc_fetlim.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_fetlim.restype = C.c_double
        L.orc_limvds.argtypes = [C.c_double, C.c_double]
        L.orc_limvds.restype = C.c_double
        L.orc_normal_quantile.argtypes = [C.c_double]
        L.orc_normal_quantile.restype = C.c_double
        L.orc_site_key.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_site_key.restype = C.c_uint64
        L.orc_step_bound.argtypes = [C.c_uint32, C.c_uint32, f64p, f64p, f64p, f64p, f64p, C.c_uint32, f64p]
        L.orc_step_bound.restype = C.c_double
        _lib = L
    return _lib


@contextlib.contextmanager
def polish(digits: int):
    """Every oracle Newton solve inside the block polishes: after the
    reference's test passes it iterates until the step passes the test with
    the tolerances scaled by 10^-digits (orc_set_polish; the product's
    espl_create_opts.polish). Process-wide."""
    lib().orc_set_polish(int(digits))
    try:
        yield
    finally:
        lib().orc_set_polish(0)


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(u32p)


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(f64p)


def order(col_ptr, row_idx, slab_len: Optional[int] = None) -> Optional[np.ndarray]:
    """BTF + AMD column order (order.zig `order`); None on OutOfWorkspace."""
    n = len(col_ptr) - 1
    cp, cpp = _u32(col_ptr)
    ri, rip = _u32(row_idx)
    q = np.zeros(max(n, 1), dtype=np.uint32)
    if slab_len is None:
        r = lib().orc_order(n, cpp, rip, q.ctypes.data_as(u32p))
    else:
        slab = np.zeros(max(slab_len, 1), dtype=np.uint32)
        r = lib().orc_order_ws(n, cpp, rip, q.ctypes.data_as(u32p), slab.ctypes.data_as(u32p), slab_len)
    return None if r != 0 else q[:n]


def amd(col_ptr, row_idx, slab_len: Optional[int] = None) -> Optional[np.ndarray]:
    n = len(col_ptr) - 1
    cp, cpp = _u32(col_ptr)
    ri, rip = _u32(row_idx)
    if slab_len is None:
        slab_len = ws_size(n, int(cp[-1]))
    slab = np.zeros(max(slab_len, 1), dtype=np.uint32)
    q = np.zeros(max(n, 1), dtype=np.uint32)
    r = lib().orc_amd_ws(n, cpp, rip, q.ctypes.data_as(u32p), slab.ctypes.data_as(u32p), slab_len)
    return None if r != 0 else q[:n]


def ws_size(n: int, nnz: int) -> int:
    return int(lib().orc_ws_size(n, nnz))


def chol_count(col_ptr, row_idx, perm, cap=(1 << 64) - 1) -> int:
    n = len(col_ptr) - 1
    cp, cpp = _u32(col_ptr)
    ri, rip = _u32(row_idx)
    pm, pmp = _u32(perm)
    return int(lib().orc_chol_count(n, cpp, rip, pmp, cap))


class OrcTape(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nnz", C.c_uint32), ("nnz_l", C.c_uint32), ("nnz_u", C.c_uint32),
                ("q", u32p), ("pinv", u32p), ("lp", u32p), ("li", u32p), ("up", u32p), ("ui", u32p),
                ("prow", u32p), ("void_col", C.POINTER(C.c_uint8)), ("scaled_pivot", C.POINTER(C.c_uint8)),
                ("void_slots", u32p), ("n_void_slots", C.c_uint32), ("lx", f64p), ("ux", f64p),
                ("udiag", f64p), ("sn_dfs", C.c_uint32), ("n_panels", C.c_uint32)]


class SparseLu:
    """SparseLu over a caller-given column order."""

    def __init__(self, col_ptr, row_idx, q, diag_fill=0, fill_cap=0.0, keep_min=0.0):
        self.cp, self.cpp = _u32(col_ptr)
        self.ri, self.rip = _u32(row_idx)
        self.q, qp = _u32(q)
        self.n = len(self.cp) - 1
        self.h = lib().orc_lu_new(self.n, self.cpp, qp)
        lib().orc_lu_set_caps(self.h, diag_fill, fill_cap, keep_min)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_lu_free(self.h)
            self.h = None

    def factor(self, vals, pivot_tol=1e-3) -> int:
        v, vp = _f64(vals)
        return lib().orc_lu_factor(self.h, self.cpp, self.rip, vp, pivot_tol)

    def refactor(self, vals, growth=1e-12) -> int:
        v, vp = _f64(vals)
        return lib().orc_lu_refactor(self.h, self.cpp, vp, growth)

    def solve(self, b) -> np.ndarray:
        bb, bp = _f64(b)
        x = np.zeros(self.n)
        lib().orc_lu_solve(self.h, bp, x.ctypes.data_as(f64p))
        return x

    def solve_t(self, b) -> np.ndarray:
        bb, bp = _f64(b)
        x = np.zeros(self.n)
        lib().orc_lu_solve_t(self.h, bp, x.ctypes.data_as(f64p))
        return x

    def tape(self) -> dict:
        t = OrcTape()
        lib().orc_lu_tape(self.h, C.byref(t))
        n = t.n

        def cp(ptr, m, dt=np.uint32):
            return np.ctypeslib.as_array(ptr, shape=(m,)).astype(dt).copy() if m else np.zeros(0, dt)

        return {
            "q": cp(t.q, n), "pinv": cp(t.pinv, n), "lp": cp(t.lp, n + 1), "li": cp(t.li, t.nnz_l),
            "up": cp(t.up, n + 1), "ui": cp(t.ui, t.nnz_u), "prow": cp(t.prow, t.nnz),
            "void_col": cp(t.void_col, n, np.uint8), "scaled_pivot": cp(t.scaled_pivot, n, np.uint8),
            "void_slots": cp(t.void_slots, t.n_void_slots),
            "lx": cp(t.lx, t.nnz_l, np.float64), "ux": cp(t.ux, t.nnz_u, np.float64),
            "udiag": cp(t.udiag, n, np.float64), "sn_dfs": t.sn_dfs, "n_panels": t.n_panels,
        }


def op_lanes(net: Netlist, opts: NewtonOpts, lane0: int = 0, count: Optional[int] = None, x_in=None,
             threads: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """Operating points of lanes [lane0, lane0 + count); returns x [count, n]
    and results [count, 3] (converged, singular, iterations)."""
    if count is None:
        count = net.lanes - lane0
    cn = CNet(net)
    x = np.zeros((count, net.n))
    res = (OrcNewtonResult * count)()
    xin = None
    if x_in is not None:
        xi, xin = _f64(x_in)
    r = lib().orc_op_lanes(C.byref(cn.c), lane0, count, C.byref(opts), xin, x.ctypes.data_as(f64p), res, threads)
    assert r == 0
    out = np.array([[e.converged, e.singular, e.iterations] for e in res], dtype=np.int64)
    return x, out


def op_ladder(net: Netlist, opts: NewtonOpts, threads: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """Operating points of every lane through the continuation ladder from
    the cold start; returns x [lanes, n] and results [lanes, 3] (converged,
    singular, iterations over every rung)."""
    count = net.lanes
    cn = CNet(net)
    x = np.zeros((count, net.n))
    res = (OrcNewtonResult * count)()
    r = lib().orc_op_ladder(C.byref(cn.c), 0, count, C.byref(opts), x.ctypes.data_as(f64p), res, threads)
    assert r == 0
    out = np.array([[e.converged, e.singular, e.iterations] for e in res], dtype=np.int64)
    return x, out


def ac_lanes(net: Netlist, x: np.ndarray, vsrc: int, omega, rows) -> np.ndarray:
    """Small-signal AC response of every lane at its operating point x
    [lanes, n] to a unit AC voltage on voltage source number `vsrc`:
    (G + j omega C) x = e_branch, G and C from the oracle's device models,
    solved densely (numpy). Complex [lanes, len(omega), len(rows)]."""
    cn = CNet(net)
    n, nnz = net.n, len(net.row_idx)
    cp = np.asarray(net.col_ptr, dtype=np.int64)
    ri = np.asarray(net.row_idx, dtype=np.int64)
    cols = np.repeat(np.arange(n), np.diff(cp))
    vb = [b for b in net.batches if b.kind == 3][0]
    branch = int(np.asarray(vb.term).reshape(-1, 3)[vsrc, 2])
    out = np.zeros((net.lanes, len(omega), len(rows)), dtype=complex)
    g = np.zeros(nnz)
    c = np.zeros(nnz)
    for l in range(net.lanes):
        xl = np.ascontiguousarray(x[l], dtype=np.float64)
        assert lib().orc_planes(C.byref(cn.c), l, xl.ctypes.data_as(f64p), g.ctypes.data_as(f64p),
                                c.ctypes.data_as(f64p)) == 0
        G = np.zeros((n, n))
        Cm = np.zeros((n, n))
        np.add.at(G, (ri, cols), g)
        np.add.at(Cm, (ri, cols), c)
        e = np.zeros(n, dtype=complex)
        e[branch] = 1.0
        for f, w in enumerate(omega):
            out[l, f] = np.linalg.solve(G + 1j * w * Cm, e)[list(rows)]
    return out


def ac_solve_lanes(net: Netlist, x: np.ndarray, omega, rhs, rows, adjoint: bool = False) -> np.ndarray:
    """(G + j omega C) z = b, or its transpose when `adjoint`, for each row b
    of `rhs` (complex [n_rhs, n]) on every lane at its operating point x,
    G and C from the oracle's device models, solved densely (numpy).
    Complex [lanes, len(omega), n_rhs, len(rows)]."""
    cn = CNet(net)
    n, nnz = net.n, len(net.row_idx)
    cp = np.asarray(net.col_ptr, dtype=np.int64)
    ri = np.asarray(net.row_idx, dtype=np.int64)
    cols = np.repeat(np.arange(n), np.diff(cp))
    b = np.atleast_2d(np.asarray(rhs, dtype=complex))
    out = np.zeros((net.lanes, len(omega), len(b), len(rows)), dtype=complex)
    g = np.zeros(nnz)
    c = np.zeros(nnz)
    for l in range(net.lanes):
        xl = np.ascontiguousarray(x[l], dtype=np.float64)
        assert lib().orc_planes(C.byref(cn.c), l, xl.ctypes.data_as(f64p), g.ctypes.data_as(f64p),
                                c.ctypes.data_as(f64p)) == 0
        G = np.zeros((n, n))
        Cm = np.zeros((n, n))
        np.add.at(G, (ri, cols), g)
        np.add.at(Cm, (ri, cols), c)
        for f, w in enumerate(omega):
            Y = G + 1j * w * Cm
            out[l, f] = np.linalg.solve(Y.T if adjoint else Y, b.T).T[:, list(rows)]
    return out


KT4 = 4.0 * 1.38064852e-23 * 300.15  # 4kT at 27 C, the models' default temperature
Q2 = 2.0 * 1.6021766208e-19


def _mos_alone(b, i: int, lanes: int) -> Netlist:
    """MOS instance i of batch b alone, its four terminals on four distinct
    nodes, so a probe's drain-row Jacobian reads gm even where the deck ties
    the gate to the drain (a probe on the deck's own nodes sums the tied
    terminals' columns)."""
    from egspice_b200.decks import Builder
    p = np.asarray(b.param)[i]  # [9, lanes]: type, vto, kp, gamma, phi, lambda, is, w, l
    bl = Builder("mos", lanes)
    bl.m("d", "g", "s", "b", p[0], p[1], p[2], p[7], p[8], gamma=p[3], phi=p[4], lam=p[5], is_=p[6])
    return bl.freeze()


def noise_densities(net: Netlist, x: np.ndarray) -> np.ndarray:
    """White noise current densities [lanes, n_src] of the reference's
    models at each lane's x: resistors 4kT/R (resistor.va, R from the
    batch), diodes 2q|Id| without the gmin shunt (diode.va:326, Id from the
    oracle's device probe), MOS 4kT (2/3)|gm| (mos1.va:480-489, gm the
    probe's drain-row gate entry with the terminals apart); sources ordered
    resistors, diodes, MOS (batch order)."""
    out = []
    for kind in (1, 5, 6):
        for bi, b in enumerate(net.batches):
            if b.kind != kind:
                continue
            t = np.asarray(b.term, dtype=np.int64).reshape(len(b.term), -1)
            t = np.where(t == 0xFFFFFFFF, net.n, t)  # the ground reads 0 V
            for i in range(len(t)):
                if kind == 1:
                    out.append(KT4 / np.abs(np.asarray(b.param)[i, 0]))
                    continue
                alone = _mos_alone(b, i, net.lanes) if kind == 6 else None
                col = np.zeros(net.lanes)
                for l in range(net.lanes):
                    v = np.append(x[l], 0.0)[t[i]]
                    if kind == 5:
                        f, _, _, _ = device_probe(net, bi, i, l, v)
                        col[l] = Q2 * abs(f[0] - 1e-12 * (v[0] - v[1]))
                    else:
                        _, j, _, _ = device_probe(alone, 0, 0, l, v)
                        col[l] = KT4 * (2.0 / 3.0) * abs(j[0, 1])
                out.append(col)
    return np.stack(out, axis=1) if out else np.zeros((net.lanes, 0))


def noise_lanes(net: Netlist, x: np.ndarray, omega, out: int, terms: np.ndarray) -> np.ndarray:
    """Output noise density of unknown `out` [lanes, len(omega)]: the dense
    adjoint solve per lane and frequency, each source's density times
    |z[a] - z[b]|^2 (terms [n_src, 2], in noise_densities' order)."""
    e = np.zeros((1, net.n), dtype=complex)
    e[0, out] = 1.0
    z = ac_solve_lanes(net, x, omega, e, np.arange(net.n), adjoint=True)[:, :, 0, :]
    z = np.concatenate([z, np.zeros(z.shape[:2] + (1,), dtype=complex)], axis=2)  # the ground
    psd = noise_densities(net, x)
    h = z[:, :, terms[:, 0]] - z[:, :, terms[:, 1]]
    return np.einsum("ls,lfs->lf", psd, np.abs(h) ** 2)


def tran_lanes(net: Netlist, opts: TranOpts, lane0: int = 0, count: Optional[int] = None,
               probes: Sequence[int] = (), max_rows: int = 0, meas: Optional[Tuple[int, float, float]] = None,
               threads: int = 1):
    """Transients of lanes [lane0, lane0 + count). Returns (x_final [count, n],
    reports list, probe rows [count, max_rows, n_probes] or None, period
    [count] or None)."""
    if count is None:
        count = net.lanes - lane0
    cn = CNet(net)
    x = np.zeros((count, net.n))
    reps = (StepReport * count)()
    pr, prp = _u32(np.asarray(probes, dtype=np.uint32) if len(probes) else np.zeros(1, np.uint32))
    rows = None
    rowp = None
    if len(probes) and max_rows:
        rows = np.full((count, max_rows, len(probes)), np.nan)
        rowp = rows.ctypes.data_as(f64p)
    per = None
    perp = None
    mrow, mlev, mt0 = (0xFFFFFFFF, 0.0, 0.0)
    if meas is not None:
        mrow, mlev, mt0 = meas
        per = np.full(count, np.nan)
        perp = per.ctypes.data_as(f64p)
    r = lib().orc_tran_lanes(C.byref(cn.c), lane0, count, C.byref(opts), prp, len(probes), max_rows, rowp,
                             x.ctypes.data_as(f64p), reps, mrow, mlev, mt0, perp, threads)
    assert r == 0
    return x, list(reps), rows, per


def tran_meas(net: Netlist, opts: TranOpts, passes: Sequence[MeasPass], threads: int = 1):
    """Transients of every lane with streaming .meas passes. Returns
    (value [lanes, passes], at [lanes, passes], x_final, reports)."""
    count = net.lanes
    cn = CNet(net)
    n = len(passes)
    arr = (MeasPass * max(n, 1))(*passes)
    val = np.full((count, max(n, 1)), np.nan)
    at = np.full((count, max(n, 1)), np.nan)
    x = np.zeros((count, net.n))
    reps = (StepReport * count)()
    r = lib().orc_tran_meas(C.byref(cn.c), 0, count, C.byref(opts), arr, n, val.ctypes.data_as(f64p),
                            at.ctypes.data_as(f64p), x.ctypes.data_as(f64p), reps, threads)
    assert r == 0
    return val[:, :n], at[:, :n], x, list(reps)


def meas_series(p: MeasPass, xs, vs) -> Tuple[float, float]:
    """One pass over the samples (xs[k], vs[k])."""
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    vs = np.ascontiguousarray(vs, dtype=np.float64)
    v, a = C.c_double(), C.c_double()
    lib().orc_meas_series(C.byref(p), xs.ctypes.data_as(f64p), vs.ctypes.data_as(f64p), len(xs), C.byref(v),
                          C.byref(a))
    return v.value, a.value


def meas_table(passes: Sequence[MeasPass], xs, cols):
    """Passes over a table of samples: cols[k, u] is column u at xs[k]; a
    pass reads column `row` (and its level column). Returns (value, at),
    one entry per pass."""
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    cols = np.ascontiguousarray(cols, dtype=np.float64)
    assert cols.ndim == 2 and len(cols) == len(xs)
    n = len(passes)
    arr = (MeasPass * max(n, 1))(*passes)
    val = np.full(max(n, 1), np.nan)
    at = np.full(max(n, 1), np.nan)
    r = lib().orc_meas_table(arr, n, xs.ctypes.data_as(f64p), cols.ctypes.data_as(f64p), cols.shape[1], len(xs),
                             val.ctypes.data_as(f64p), at.ctypes.data_as(f64p))
    assert r == 0
    return val[:n], at[:n]


def device_probe(net: Netlist, batch: int, inst: int, lane: int, v):
    nt = {1: 2, 2: 2, 3: 3, 4: 2, 5: 2, 6: 4}[net.batches[batch].kind]
    cn = CNet(net)
    vv, vp = _f64(v)
    f = np.zeros(nt)
    j = np.zeros(nt * nt)
    q = np.zeros(nt)
    cj = np.zeros(nt * nt)
    r = lib().orc_device_probe(C.byref(cn.c), batch, inst, lane, vp, f.ctypes.data_as(f64p),
                               j.ctypes.data_as(f64p), q.ctypes.data_as(f64p), cj.ctypes.data_as(f64p))
    assert r == 0
    return f, j.reshape(nt, nt), q, cj.reshape(nt, nt)
