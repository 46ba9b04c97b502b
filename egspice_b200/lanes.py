"""Python host mirror of the lane driver seam (include/espice_lanes.h).

`Lanes` owns one espl_lanes handle: the role of ESPice's `GpuLanes`
(src/analysis/gpu/lanes.zig) for a batch of sweep points, possibly drawn from
several templates of different sizes. The compute runs in the sm_100a
library egspice_b200/_lib/libespice_lanes.so; there is no CPU fallback, and
a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .abi import (ClassInfo, CreateOpts, MeasPass, LaneNewton, NetlistC, NewtonOpts, PlanChoice, StepReport, Stats,
                  TranOpts, TuneReport, f64p, u32p)
from .decks import Netlist

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libespice_lanes.so")
_lib = None


class LaneError(RuntimeError):
    pass


def lib():
    """Loads the CUDA lane library; raises when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LaneError(f"{LIB_PATH} is missing: run egspice_b200/build.py (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        L.espl_abi_version.restype = C.c_uint32
        L.espl_create.argtypes = [C.POINTER(NetlistC), C.c_uint32, C.POINTER(CreateOpts), C.c_double,
                                  C.POINTER(C.c_void_p)]
        L.espl_create.restype = C.c_uint32
        L.espl_destroy.argtypes = [C.c_void_p]
        L.espl_destroy.restype = C.c_uint32
        L.espl_tape_info.argtypes = [C.c_void_p, C.c_uint32, u32p, u32p, u32p]
        L.espl_tape_info.restype = C.c_uint32
        L.espl_copy_tape.argtypes = [C.c_void_p, C.c_uint32] + [u32p] * 7
        L.espl_copy_tape.restype = C.c_uint32
        L.espl_put_x.argtypes = [C.c_void_p, C.c_uint32, f64p, C.c_uint32]
        L.espl_put_x.restype = C.c_uint32
        L.espl_get_x.argtypes = [C.c_void_p, C.c_uint32, f64p]
        L.espl_get_x.restype = C.c_uint32
        L.espl_solve_static.argtypes = [C.c_void_p, C.POINTER(NewtonOpts), C.POINTER(LaneNewton)]
        L.espl_solve_static.restype = C.c_uint32
        L.espl_init_steps.argtypes = [C.c_void_p, C.POINTER(TranOpts)]
        L.espl_init_steps.restype = C.c_uint32
        L.espl_device_launch.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(StepReport)]
        L.espl_device_launch.restype = C.c_uint32
        L.espl_set_period_meas.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_double]
        L.espl_set_period_meas.restype = C.c_uint32
        L.espl_get_period_meas.argtypes = [C.c_void_p, C.c_uint32, f64p, u32p]
        L.espl_get_period_meas.restype = C.c_uint32
        L.espl_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.espl_get_stats.restype = C.c_uint32
        L.espl_ac.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, f64p, C.c_uint32, u32p, C.c_uint32, f64p, f64p]
        L.espl_ac.restype = C.c_uint32
        L.espl_ac_solve.argtypes = [C.c_void_p, C.c_uint32, f64p, C.c_uint32, f64p, f64p, C.c_uint32, C.c_uint32,
                                    u32p, C.c_uint32, f64p, f64p]
        L.espl_ac_solve.restype = C.c_uint32
        L.espl_noise_sources.argtypes = [C.c_void_p, C.c_uint32, f64p, u32p]
        L.espl_noise_sources.restype = C.c_uint32
        L.espl_meas_table.argtypes = [C.POINTER(MeasPass), C.c_uint32, f64p, f64p, C.c_uint32, C.c_uint32, f64p,
                                      f64p]
        L.espl_meas_table.restype = C.c_uint32
        L.espl_meas_done.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint8)]
        L.espl_meas_done.restype = C.c_uint32
        L.espl_request_stop.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint8)]
        L.espl_request_stop.restype = C.c_uint32
        L.espl_solve_op.argtypes = [C.c_void_p, C.POINTER(NewtonOpts), C.POINTER(LaneNewton)]
        L.espl_solve_op.restype = C.c_uint32
        L.espl_set_meas.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(MeasPass), C.c_uint32]
        L.espl_set_meas.restype = C.c_uint32
        L.espl_get_meas.argtypes = [C.c_void_p, C.c_uint32, f64p, f64p]
        L.espl_get_meas.restype = C.c_uint32
        L.espl_get_classes.argtypes = [C.c_void_p, C.POINTER(ClassInfo), C.c_uint32, u32p]
        L.espl_get_classes.restype = C.c_uint32
        L.espl_error_message.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.espl_error_message.restype = C.c_uint32
        L.espl_record_steps.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.espl_record_steps.restype = C.c_uint32
        L.espl_recorded_steps.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), u32p]
        L.espl_recorded_steps.restype = C.c_uint32
        L.espl_copy_recorded_steps.argtypes = [C.c_void_p, C.c_uint32, f64p, f64p, f64p, C.c_uint32]
        L.espl_copy_recorded_steps.restype = C.c_uint32
        L.espl_set_step_predictor.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.espl_set_step_predictor.restype = C.c_uint32
        L.espl_step_predict.argtypes = [C.c_void_p, C.c_uint32, f64p, f64p, f64p, f64p, f64p]
        L.espl_step_predict.restype = C.c_uint32
        L.espl_set_plan.argtypes = [C.c_void_p, C.POINTER(PlanChoice)]
        L.espl_set_plan.restype = C.c_uint32
        L.espl_get_plan.argtypes = [C.c_void_p, C.POINTER(PlanChoice)]
        L.espl_get_plan.restype = C.c_uint32
        L.espl_autotune.argtypes = [C.POINTER(NetlistC), C.c_uint32, C.POINTER(CreateOpts), C.c_double,
                                    C.POINTER(TranOpts), C.c_uint32, C.c_uint32, C.POINTER(PlanChoice),
                                    C.POINTER(TuneReport)]
        L.espl_autotune.restype = C.c_uint32
        _lib = L
    return _lib


PRECISION = {"fp64": abi.ESPL_FP64, "mixed": abi.ESPL_MIXED}


def autotune(nets: Sequence[Netlist], topts, precision: str = "fp64", dt0: float = 0.0, polish: int = 0,
             refine_sweeps: int = 0, device: int = 0, trial_steps: int = 100, max_trials: int = 12):
    """espl_autotune: the launch plan of `nets` for the transient `topts`,
    searched by timing `trial_steps` attempts per plan on scratch handles.
    Returns (choices, report): choices a list of PlanChoice for
    Lanes.set_plan, report a dict (trials, cached, auto_ms, best_ms)."""
    keep, arr = abi.cnets(list(nets))
    opts = CreateOpts(abi.ABI_VERSION, PRECISION[precision], device, 0, refine_sweeps, polish)
    out = (PlanChoice * len(nets))()
    rep = TuneReport()
    st = lib().espl_autotune(arr, len(nets), C.byref(opts), dt0, C.byref(topts), trial_steps, max_trials, out,
                             C.byref(rep))
    del keep
    if st != 0:
        raise LaneError(f"espl_autotune failed with status {st}")
    return list(out), dict(trials=rep.trials, cached=rep.cached, auto_ms=rep.auto_ms, best_ms=rep.best_ms)


def meas_table(passes: Sequence[MeasPass], xs, cols):
    """The measure passes over a host table (espl_meas_table): cols[k, u]
    is column u at scale xs[k]. Returns (value, at), one per pass."""
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    cols = np.ascontiguousarray(np.atleast_2d(cols), dtype=np.float64)
    n = len(passes)
    arr = (MeasPass * max(n, 1))(*passes)
    val = np.full(max(n, 1), np.nan)
    at = np.full(max(n, 1), np.nan)
    st = lib().espl_meas_table(arr, n, xs.ctypes.data_as(f64p), cols.ctypes.data_as(f64p), cols.shape[1], len(xs),
                               val.ctypes.data_as(f64p), at.ctypes.data_as(f64p))
    if st != 0:
        raise LaneError(f"espl_meas_table failed with status {st}")
    return val[:n], at[:n]


def noise_terminals(net: Netlist) -> np.ndarray:
    """The (from, to) unknowns of each noise source of `net`, in the order
    espl_noise_sources reports them: resistors (p, n), diodes (anode,
    cathode), MOS (drain, source); a grounded terminal reads net.n."""
    from .decks import DIODE, GROUND, MOS1, RES
    out = []
    for kind, cols in ((RES, (0, 1)), (DIODE, (0, 1)), (MOS1, (0, 2))):
        for b in net.batches:
            if b.kind == kind:
                t = np.asarray(b.term, dtype=np.int64).reshape(len(b.term), -1)
                t = np.where(t == GROUND, net.n, t)
                out += [(int(r[cols[0]]), int(r[cols[1]])) for r in t]
    return np.array(out, dtype=np.int64).reshape(-1, 2)


def noise_sum(psd: np.ndarray, z: np.ndarray, terms: np.ndarray) -> np.ndarray:
    """sum_s psd[l, s] |z[l, f, a_s] - z[l, f, b_s]|^2: the output density
    from source densities psd [lanes, n_src] and the adjoint solutions
    z [lanes, F, n] (z[u]: transfer from a unit current into unknown u to
    the output; index n, the ground, reads zero)."""
    if len(terms) == 0:
        return np.zeros(z.shape[:2])
    z = np.concatenate([z, np.zeros(z.shape[:2] + (1,), dtype=z.dtype)], axis=2)
    h = z[:, :, terms[:, 0]] - z[:, :, terms[:, 1]]
    return np.einsum("ls,lfs->lf", psd, np.abs(h) ** 2)


class Lanes:
    """Lanes of one or more templates on one GPU."""

    def __init__(self, nets: Sequence[Netlist], precision: str = "fp64", dt0: float = 0.0, device: int = 0,
                 refine_sweeps: int = 0, polish: int = 0):
        """`polish` k > 0: every Newton solve keeps iterating after the
        reference's convergence test passes until its step also passes the
        test with the tolerances scaled by 10^-k (espl_create_opts.polish)."""
        self.nets = list(nets)
        self._keep, arr = abi.cnets(self.nets)
        self._arr = arr
        opts = CreateOpts(abi.ABI_VERSION, PRECISION[precision], device, 0, refine_sweeps, polish)
        h = C.c_void_p()
        st = lib().espl_create(arr, len(self.nets), C.byref(opts), dt0, C.byref(h))
        if st != 0:
            raise LaneError(f"espl_create failed with status {st}")
        self.h = h
        self.total = sum(n.lanes for n in self.nets)

    def close(self):
        if getattr(self, "h", None):
            lib().espl_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, what: str):
        if st != 0:
            buf = C.create_string_buffer(512)
            lib().espl_error_message(self.h, buf, 512)
            raise LaneError(f"{what} failed with status {st}: {buf.value.decode()}")

    def put_x(self, net: int, x: np.ndarray, cold: bool):
        nl = self.nets[net]
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(nl.lanes, nl.n)
        self._check(lib().espl_put_x(self.h, net, x.ctypes.data_as(f64p), int(cold)), "espl_put_x")

    def cold_start(self):
        for i, nl in enumerate(self.nets):
            self.put_x(i, np.zeros((nl.lanes, nl.n)), True)

    def get_x(self, net: int) -> np.ndarray:
        nl = self.nets[net]
        x = np.zeros((nl.lanes, nl.n))
        self._check(lib().espl_get_x(self.h, net, x.ctypes.data_as(f64p)), "espl_get_x")
        return x

    def solve_static(self, opts: NewtonOpts) -> np.ndarray:
        """Newton per lane; returns [total, 3] of (bits, iterations, fp64 fallbacks)."""
        out = (LaneNewton * self.total)()
        self._check(lib().espl_solve_static(self.h, C.byref(opts), out), "espl_solve_static")
        return np.array([[o.bits, o.iterations, o.refactor_fallbacks] for o in out], dtype=np.int64)

    def solve_op(self, opts: NewtonOpts) -> np.ndarray:
        """The operating point from the cold start with the continuation
        ladder (plain rung, gmin stepping, source stepping, final solve);
        returns [total, 3] of (bits, iterations over every rung, fp64
        fallbacks)."""
        out = (LaneNewton * self.total)()
        self._check(lib().espl_solve_op(self.h, C.byref(opts), out), "espl_solve_op")
        return np.array([[o.bits, o.iterations, o.refactor_fallbacks] for o in out], dtype=np.int64)

    def ac(self, net: int, vsrc: int, omega, rows) -> np.ndarray:
        """Small-signal response to a unit AC voltage on voltage source
        `vsrc` of template `net` at angular frequencies `omega`: complex
        [lanes, len(omega), len(rows)]."""
        om = np.ascontiguousarray(omega, dtype=np.float64)
        rw = np.ascontiguousarray(rows, dtype=np.uint32)
        lanes = self.nets[net].lanes
        re = np.zeros((lanes, len(om), len(rw)))
        im = np.zeros((lanes, len(om), len(rw)))
        self._check(lib().espl_ac(self.h, net, vsrc, om.ctypes.data_as(f64p), len(om), rw.ctypes.data_as(u32p), len(rw),
                                  re.ctypes.data_as(f64p), im.ctypes.data_as(f64p)), "espl_ac")
        return re + 1j * im

    def ac_solve(self, net: int, omega, rhs, rows, adjoint: bool = False) -> np.ndarray:
        """(G + j omega C) x = b for each row b of `rhs` (complex [n_rhs, n],
        the same on every lane), or the transpose system when `adjoint`:
        complex [lanes, len(omega), n_rhs, len(rows)]."""
        om = np.ascontiguousarray(omega, dtype=np.float64)
        rw = np.ascontiguousarray(rows, dtype=np.uint32)
        b = np.atleast_2d(np.asarray(rhs, dtype=complex))
        br = np.ascontiguousarray(b.real)
        bi = np.ascontiguousarray(b.imag)
        lanes = self.nets[net].lanes
        re = np.zeros((lanes, len(om), len(b), len(rw)))
        im = np.zeros((lanes, len(om), len(b), len(rw)))
        self._check(lib().espl_ac_solve(self.h, net, om.ctypes.data_as(f64p), len(om), br.ctypes.data_as(f64p),
                                        bi.ctypes.data_as(f64p), len(b), int(adjoint), rw.ctypes.data_as(u32p),
                                        len(rw), re.ctypes.data_as(f64p), im.ctypes.data_as(f64p)), "espl_ac_solve")
        return re + 1j * im

    def noise_sources(self, net: int):
        """(psd [lanes, n_src] in A^2/Hz, terminals [n_src, 2]) of template
        `net`'s noise sources at the lanes' x: resistors, diodes, MOS."""
        n = C.c_uint32()
        self._check(lib().espl_noise_sources(self.h, net, None, C.byref(n)), "espl_noise_sources")
        psd = np.zeros((self.nets[net].lanes, max(n.value, 1)))
        self._check(lib().espl_noise_sources(self.h, net, psd.ctypes.data_as(f64p), C.byref(n)),
                    "espl_noise_sources")
        return psd[:, :n.value], noise_terminals(self.nets[net])

    def noise(self, net: int, omega, out: int, ref: Optional[int] = None) -> np.ndarray:
        """Output noise density (V^2/Hz, or A^2/Hz for a branch row) of
        unknown `out` (minus `ref`) at angular frequencies `omega`, every
        lane at its operating point: one adjoint solve per frequency and
        each source's density times its squared transfer. [lanes, len(omega)]."""
        nl = self.nets[net]
        b = np.zeros(nl.n, dtype=complex)
        b[out] = 1.0
        if ref is not None:
            b[ref] = -1.0
        psd, terms = self.noise_sources(net)
        z = self.ac_solve(net, omega, b[None, :], np.arange(nl.n), adjoint=True)[:, :, 0, :]
        return noise_sum(psd, z, terms)

    def init_steps(self, topts: TranOpts):
        self._check(lib().espl_init_steps(self.h, C.byref(topts)), "espl_init_steps")

    def device_launch(self, max_steps: int) -> List[StepReport]:
        reps = (StepReport * self.total)()
        self._check(lib().espl_device_launch(self.h, max_steps, reps), "espl_device_launch")
        return list(reps)

    def run_tran(self, topts: TranOpts, steps_per_launch: int = 256, max_launches: int = 100000):
        """Runs every lane to t_stop; returns the final reports."""
        self.init_steps(topts)
        reps = None
        for _ in range(max_launches):
            reps = self.device_launch(steps_per_launch)
            if all(r.status != 0 for r in reps):
                break
        return reps

    def set_period_meas(self, net: int, row: int, level: float, t_start: float):
        self._check(lib().espl_set_period_meas(self.h, net, row, level, t_start), "espl_set_period_meas")

    def period_meas(self, net: int):
        nl = self.nets[net]
        per = np.zeros(nl.lanes)
        cr = np.zeros(nl.lanes, dtype=np.uint32)
        self._check(lib().espl_get_period_meas(self.h, net, per.ctypes.data_as(f64p), cr.ctypes.data_as(u32p)),
                    "espl_get_period_meas")
        return per, cr

    def tape(self, net: int) -> dict:
        n, nl, nu = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._check(lib().espl_tape_info(self.h, net, C.byref(n), C.byref(nl), C.byref(nu)), "espl_tape_info")
        n, nl, nu = n.value, nl.value, nu.value
        arrs = {"q": n, "pinv": n, "lp": n + 1, "li": nl, "up": n + 1, "ui": nu, "flags": n}
        out = {k: np.zeros(max(v, 1), dtype=np.uint32) for k, v in arrs.items()}
        self._check(lib().espl_copy_tape(self.h, net, *[out[k].ctypes.data_as(u32p) for k in
                                                        ("q", "pinv", "lp", "li", "up", "ui", "flags")]),
                    "espl_copy_tape")
        return {k: out[k][:arrs[k]] for k in arrs}

    def set_meas(self, net: int, passes: Sequence[MeasPass]):
        """Streaming .meas passes of template `net` (abi.meas_pass), set
        before init_steps."""
        arr = (MeasPass * max(len(passes), 1))(*passes)
        self._check(lib().espl_set_meas(self.h, net, arr, len(passes)), "espl_set_meas")
        self._n_meas = getattr(self, "_n_meas", {})
        self._n_meas[net] = len(passes)

    def get_meas(self, net: int):
        """(value, at), each [lanes, passes]."""
        n = getattr(self, "_n_meas", {}).get(net, 0)
        lanes = self.nets[net].lanes
        v = np.full((lanes, max(n, 1)), np.nan)
        a = np.full((lanes, max(n, 1)), np.nan)
        self._check(lib().espl_get_meas(self.h, net, v.ctypes.data_as(f64p), a.ctypes.data_as(f64p)), "espl_get_meas")
        return v[:, :n], a[:, :n]

    def meas_done(self, net: int) -> np.ndarray:
        """[lanes, passes] bool: passes that have read their last sample."""
        n = getattr(self, "_n_meas", {}).get(net, 0)
        out = np.zeros((self.nets[net].lanes, max(n, 1)), dtype=np.uint8)
        if n:
            self._check(lib().espl_meas_done(self.h, net, out.ctypes.data_as(C.POINTER(C.c_uint8))),
                        "espl_meas_done")
        return out[:, :n].astype(bool)

    def request_stop(self, net: int, stop) -> None:
        """Stops the still-stepping lanes of template `net` where `stop`
        [lanes] is true, before the next device launch."""
        m = np.ascontiguousarray(np.asarray(stop, dtype=bool), dtype=np.uint8)
        assert m.shape == (self.nets[net].lanes,)
        self._check(lib().espl_request_stop(self.h, net, m.ctypes.data_as(C.POINTER(C.c_uint8))),
                    "espl_request_stop")

    def record_steps(self, net: int, lane_stride: int, from_step: int, capacity: int):
        """Records training samples of the learned step predictor from the
        accepted steps of template `net` (espl_record_steps): lanes l with
        l % lane_stride == 0, steps past `from_step`, at most `capacity`."""
        self._check(lib().espl_record_steps(self.h, net, lane_stride, from_step, capacity), "espl_record_steps")

    def recorded(self, net: int):
        """(x device pointer, y device pointer, count) of the samples
        recorded for template `net`."""
        x, y, n = C.c_void_p(), C.c_void_p(), C.c_uint32()
        self._check(lib().espl_recorded_steps(self.h, net, C.byref(x), C.byref(y), C.byref(n)), "espl_recorded_steps")
        return x.value, y.value, n.value

    def recorded_host(self, net: int):
        """Host copies of the recorded samples: x [count, 3 n + 1], y [count, n],
        tags [count, 5] (lane, accepted steps before, dt, h0, h1)."""
        n = self.nets[net].n
        _, _, k = self.recorded(net)
        x, y, t = np.zeros((max(k, 1), 3 * n + 1)), np.zeros((max(k, 1), n)), np.zeros((max(k, 1), 5))
        self._check(lib().espl_copy_recorded_steps(self.h, net, x.ctypes.data_as(f64p), y.ctypes.data_as(f64p),
                                                   t.ctypes.data_as(f64p), k), "espl_copy_recorded_steps")
        return x[:k], y[:k], t[:k]

    def set_step_predictor(self, net: int, mlp) -> None:
        """Attaches a trained `learned.Mlp` (3 n + 1 inputs, n outputs) as
        template `net`'s step predictor; None detaches."""
        self._check(lib().espl_set_step_predictor(self.h, net, mlp.h if mlp is not None else None),
                    "espl_set_step_predictor")

    def step_predict(self, net: int) -> dict:
        """The learned start of each lane's next attempt and the history it
        was computed from: x_start, cur, prev, prev2 [lanes, n] and steps
        [lanes, 3] (dt, h0, h1)."""
        nl = self.nets[net]
        out = {k: np.zeros((nl.lanes, nl.n)) for k in ("x_start", "cur", "prev", "prev2")}
        out["steps"] = np.zeros((nl.lanes, 3))
        self._check(lib().espl_step_predict(self.h, net, *[out[k].ctypes.data_as(f64p) for k in
                                                          ("x_start", "cur", "prev", "prev2", "steps")]),
                    "espl_step_predict")
        return out

    def classes(self) -> List[dict]:
        """The launch classes in launch order, each with its kernel's device
        time in the last solve or device launch."""
        n = C.c_uint32()
        self._check(lib().espl_get_classes(self.h, None, 0, C.byref(n)), "espl_get_classes")
        out = (ClassInfo * max(n.value, 1))()
        self._check(lib().espl_get_classes(self.h, out, n.value, C.byref(n)), "espl_get_classes")
        return [dict(tiles=c.tiles, wide=bool(c.wide), per_sm=c.per_sm, smem_bytes=c.smem_bytes, ms=c.last_ms)
                for c in out[:n.value]]

    def set_plan(self, choices=None):
        """Re-plans the launches (espl_set_plan): one PlanChoice per
        template, or None for the automatic plan."""
        arr = None
        if choices is not None:
            arr = (PlanChoice * len(self.nets))(*choices)
        self._check(lib().espl_set_plan(self.h, arr), "espl_set_plan")

    def plan(self) -> List[dict]:
        """The plan in effect, per template (espl_get_plan)."""
        out = (PlanChoice * len(self.nets))()
        self._check(lib().espl_get_plan(self.h, out), "espl_get_plan")
        return [dict(tile=c.tile, stage=c.stage, per_sm=c.per_sm) for c in out]

    def stats(self) -> Stats:
        s = Stats()
        self._check(lib().espl_get_stats(self.h, C.byref(s)), "espl_get_stats")
        return s
