"""ctypes mirror of include/espice_lanes.h and Netlist -> espl_netlist."""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from .decks import Netlist

u32p = C.POINTER(C.c_uint32)
f64p = C.POINTER(C.c_double)


class Batch(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("count", C.c_uint32), ("term", u32p), ("param", f64p)]


class NetlistC(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nnz", C.c_uint32), ("col_ptr", u32p), ("row_idx", u32p),
                ("n_batches", C.c_uint32), ("batches", C.POINTER(Batch)), ("lanes", C.c_uint32)]


class NewtonOpts(C.Structure):
    _fields_ = [("reltol", C.c_double), ("abstol", C.c_double), ("vntol", C.c_double),
                ("gmin", C.c_double), ("residual_tol", C.c_double), ("max_iter", C.c_uint32),
                ("init_fix", C.c_uint32)]


class LaneNewton(C.Structure):
    _fields_ = [("bits", C.c_uint32), ("iterations", C.c_uint32), ("refactor_fallbacks", C.c_uint32),
                ("reserved", C.c_uint32)]


ABI_VERSION = 3


class CreateOpts(C.Structure):
    _fields_ = [("abi_version", C.c_uint32), ("precision", C.c_uint32), ("device", C.c_uint32),
                ("lanes_per_cta", C.c_uint32), ("refine_sweeps", C.c_uint32), ("polish", C.c_uint32)]


class TranOpts(C.Structure):
    _fields_ = [("t_stop", C.c_double), ("dt", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
                ("reltol", C.c_double), ("abstol", C.c_double), ("chgtol", C.c_double), ("trtol", C.c_double),
                ("vntol", C.c_double), ("residual_tol", C.c_double), ("method", C.c_uint32),
                ("fixed_step", C.c_uint32), ("max_iter", C.c_uint32), ("max_steps", C.c_uint32),
                ("predictor", C.c_uint32), ("polish_chord", C.c_uint32)]


class StepReport(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("attempts", C.c_uint64), ("nr_iters", C.c_uint64),
                ("steps", C.c_uint32), ("rejects", C.c_uint32), ("status", C.c_uint32),
                ("learned_retries", C.c_uint32), ("t_new", C.c_double), ("attempted_dt", C.c_double),
                ("event", C.c_uint32), ("reserved", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("newton_ms", C.c_double), ("launches", C.c_uint64),
                ("lane_iterations", C.c_uint64), ("lane_steps", C.c_uint64), ("dense_peels", C.c_uint32),
                ("retapes", C.c_uint32)]


class MeasPass(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("row", C.c_uint32), ("val", C.c_double), ("td", C.c_double),
                ("from_", C.c_double), ("to", C.c_double), ("at", C.c_double), ("rise", C.c_int32),
                ("fall", C.c_int32), ("cross", C.c_int32), ("level_row", C.c_uint32)]


MEAS_WHEN, MEAS_FIND_AT, MEAS_MIN, MEAS_MAX, MEAS_AVG, MEAS_INTEG, MEAS_RMS = 1, 2, 3, 4, 5, 6, 7
MEAS_DERIV_AT, MEAS_FIND_WHEN, MEAS_DERIV_WHEN, MEAS_TARG = 8, 9, 10, 11
MEAS_UNSET, MEAS_LAST = -1, -2
MEAS_MAX_PASSES = 16  # per template


def meas_pass(kind, row, val=0.0, td=0.0, from_=0.0, to=0.0, at=0.0, rise=MEAS_UNSET, fall=MEAS_UNSET,
              cross=MEAS_UNSET, level_row=None) -> MeasPass:
    """One espl_meas pass; `level_row` names the unknown a WHEN or TARG
    crossing is measured against (None: the constant `val`)."""
    return MeasPass(kind, row, val, td, from_, to, at, rise, fall, cross, 0 if level_row is None else level_row + 1)


class ClassInfo(C.Structure):
    _fields_ = [("tiles", C.c_uint32), ("wide", C.c_uint32), ("per_sm", C.c_uint32), ("smem_bytes", C.c_uint32),
                ("last_ms", C.c_double)]


class PlanChoice(C.Structure):
    """espl_plan_choice: a template's launch-plan choice (0 fields: automatic)."""
    _fields_ = [("tile", C.c_uint32), ("stage", C.c_uint32), ("per_sm", C.c_uint32), ("pad", C.c_uint32)]


class TuneReport(C.Structure):
    _fields_ = [("trials", C.c_uint32), ("cached", C.c_uint32), ("auto_ms", C.c_double), ("best_ms", C.c_double)]


TILE_AUTO, TILE_NARROW, TILE_WIDE = 0, 1, 2
STAGE_AUTO, STAGE_LU, STAGE_LU_GLOBAL_RECORDS, STAGE_INDEX, STAGE_NONE = 0, 1, 2, 3, 4


class OrcNewtonResult(C.Structure):
    _fields_ = [("converged", C.c_uint32), ("singular", C.c_uint32), ("iterations", C.c_uint32),
                ("reserved", C.c_uint32)]


ESPL_OK = 0
ESPL_FP64, ESPL_MIXED = 0, 1
CONVERGED, SINGULAR, PARKED = 4, 8, 32


def newton_opts(reltol=1e-3, abstol=1e-12, vntol=1e-6, gmin=0.0, residual_tol=1e-9, max_iter=100,
                init_fix=1) -> NewtonOpts:
    return NewtonOpts(reltol, abstol, vntol, gmin, residual_tol, max_iter, init_fix)


def tran_opts(t_stop, dt, dt_min=0.0, dt_max=0.0, reltol=1e-3, abstol=1e-12, chgtol=1e-14, trtol=7.0,
              vntol=1e-6, residual_tol=1e-9, method=1, fixed_step=0, max_iter=10, max_steps=1 << 30,
              predictor=1) -> TranOpts:
    return TranOpts(t_stop, dt, dt_min, dt_max, reltol, abstol, chgtol, trtol, vntol, residual_tol, method,
                    fixed_step, max_iter, max_steps, predictor, 0)


class CNet:
    """Keeps the numpy buffers behind one espl_netlist alive."""

    def __init__(self, net: Netlist):
        self.net = net
        self._keep: List[np.ndarray] = []
        cp = self._arr(net.col_ptr, np.uint32)
        ri = self._arr(net.row_idx, np.uint32)
        bs = (Batch * max(1, len(net.batches)))()
        for i, b in enumerate(net.batches):
            t = self._arr(b.term, np.uint32)
            p = self._arr(b.param, np.float64)
            bs[i] = Batch(b.kind, b.term.shape[0], t.ctypes.data_as(u32p), p.ctypes.data_as(f64p))
        self._bs = bs
        self.c = NetlistC(net.n, net.nnz, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p), len(net.batches),
                          C.cast(bs, C.POINTER(Batch)), net.lanes)

    def _arr(self, a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        self._keep.append(a)
        return a


def cnets(nets: Sequence[Netlist]):
    keep = [CNet(n) for n in nets]
    arr = (NetlistC * len(keep))(*[k.c for k in keep])
    return keep, arr
