"""The learned warm start (include/espice_learned.h) from Python.

`Mlp` wraps the tensor-core MLP of egspice_b200/csrc/mlp.cu: it is trained on
operating points the plain method solved and predicts start points for the
rest of a sweep. Newton from a predicted x is the same plain Newton
(espl_solve_static) with the same tolerances, so only the iteration count
changes; a lane that does not converge from its prediction is solved again
from the nominal start (bench.py run_learned_dc).

`learned_transient` is the transient's learned next-step predictor: the
plain linear predictor runs the first steps while the accepted steps are
recorded on the device, a network is trained on them there, and the rest of
the transient starts each attempt from the network's prediction (predictor
2), the plain Newton judging every step and retrying a failed learned start
from the linear predictor.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from .lanes import LaneError, lib

f64p = C.POINTER(C.c_double)
f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)


class TrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("lr_final", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint32)]


def train_opts(epochs: int = 300, batch: int = 512, lr: float = 3e-3, lr_final: float = 1e-4, seed: int = 1):
    return TrainOpts(epochs, batch, lr, lr_final, 0.9, 0.999, 1e-8, seed)


def _setup(L):
    if getattr(L, "_mlp_ready", False):
        return L
    L.espl_mlp_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p)]
    L.espl_mlp_destroy.argtypes = [C.c_void_p]
    L.espl_mlp_param_count.argtypes = [C.c_void_p, u32p]
    L.espl_mlp_get_params.argtypes = [C.c_void_p, f32p]
    L.espl_mlp_set_params.argtypes = [C.c_void_p, f32p]
    L.espl_mlp_set_scaling.argtypes = [C.c_void_p, f64p, f64p, C.c_uint32]
    L.espl_mlp_loss_grad.argtypes = [C.c_void_p, f64p, f64p, C.c_uint32, f64p, f32p]
    L.espl_mlp_train.argtypes = [C.c_void_p, f64p, f64p, C.c_uint32, C.POINTER(TrainOpts), f64p]
    L.espl_mlp_train_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(TrainOpts), f64p]
    L.espl_mlp_train_ms.argtypes = [C.c_void_p, f64p]
    L.espl_mlp_predict_ms.argtypes = [C.c_void_p, f64p]
    L.espl_mlp_predict.argtypes = [C.c_void_p, f64p, C.c_uint32, f64p]
    L.espl_mlp_predict_layers.argtypes = [C.c_void_p, f64p, C.c_uint32, f64p]
    L.espl_mlp_error_message.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    for f in ("create", "destroy", "param_count", "get_params", "set_params", "set_scaling", "loss_grad", "train",
              "train_device", "train_ms", "predict_ms", "predict", "predict_layers", "error_message"):
        getattr(L, "espl_mlp_" + f).restype = C.c_uint32
    L._mlp_ready = True
    return L


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Mlp:
    """in_dim -> 128 -> 128 -> out_dim, tanh hidden layers, on the GPU."""

    def __init__(self, in_dim: int, out_dim: int, capacity: int = 8192, seed: int = 1, device: int = 0):
        self.L = _setup(lib())
        h = C.c_void_p()
        st = self.L.espl_mlp_create(in_dim, out_dim, capacity, seed, device, C.byref(h))
        if st != 0:
            raise LaneError(f"espl_mlp_create failed with status {st}")
        self.h, self.in_dim, self.out_dim, self.capacity = h, in_dim, out_dim, capacity

    def _check(self, st, what):
        if st != 0:
            buf = C.create_string_buffer(512)
            self.L.espl_mlp_error_message(self.h, buf, 512)
            raise LaneError(f"{what} failed with status {st}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.espl_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def param_count(self) -> int:
        c = C.c_uint32()
        self._check(self.L.espl_mlp_param_count(self.h, C.byref(c)), "param_count")
        return c.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.param_count(), dtype=np.float32)
        self._check(self.L.espl_mlp_get_params(self.h, p.ctypes.data_as(f32p)), "get_params")
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.param_count()
        self._check(self.L.espl_mlp_set_params(self.h, p.ctypes.data_as(f32p)), "set_params")

    def set_scaling(self, x, y):
        x, y = _f64(x), _f64(y)
        self._check(self.L.espl_mlp_set_scaling(self.h, x.ctypes.data_as(f64p), y.ctypes.data_as(f64p), len(x)),
                    "set_scaling")

    def loss_grad(self, x, y) -> Tuple[float, np.ndarray]:
        x, y = _f64(x), _f64(y)
        loss = C.c_double()
        g = np.zeros(self.param_count(), dtype=np.float32)
        self._check(self.L.espl_mlp_loss_grad(self.h, x.ctypes.data_as(f64p), y.ctypes.data_as(f64p), len(x),
                                              C.byref(loss), g.ctypes.data_as(f32p)), "loss_grad")
        return loss.value, g

    def train(self, x, y, opts: Optional[TrainOpts] = None) -> np.ndarray:
        opts = opts or train_opts()
        x, y = _f64(x), _f64(y)
        losses = np.zeros(opts.epochs)
        self._check(self.L.espl_mlp_train(self.h, x.ctypes.data_as(f64p), y.ctypes.data_as(f64p), len(x),
                                          C.byref(opts), losses.ctypes.data_as(f64p)), "train")
        return losses

    def train_device(self, x_ptr: int, y_ptr: int, n: int, opts: Optional[TrainOpts] = None) -> np.ndarray:
        """Training on n rows already in device memory (espl_mlp_train_device),
        e.g. the transient's recorded steps (Lanes.recorded)."""
        opts = opts or train_opts()
        losses = np.zeros(opts.epochs)
        self._check(self.L.espl_mlp_train_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), n, C.byref(opts),
                                                 losses.ctypes.data_as(f64p)), "train_device")
        return losses

    def train_ms(self) -> float:
        """Device time of the last training (espl_mlp_train_ms)."""
        ms = C.c_double()
        self._check(self.L.espl_mlp_train_ms(self.h, C.byref(ms)), "train_ms")
        return ms.value

    def predict_ms(self) -> float:
        """Device time of the last fused prediction (espl_mlp_predict_ms)."""
        ms = C.c_double()
        self._check(self.L.espl_mlp_predict_ms(self.h, C.byref(ms)), "predict_ms")
        return ms.value

    def predict(self, x, fused: bool = True) -> np.ndarray:
        x = _f64(x)
        y = np.zeros((len(x), self.out_dim))
        f = self.L.espl_mlp_predict if fused else self.L.espl_mlp_predict_layers
        self._check(f(self.h, x.ctypes.data_as(f64p), len(x), y.ctypes.data_as(f64p)), "predict")
        return y

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def step_predictor_dims(n: int) -> Tuple[int, int]:
    """(inputs, outputs) of the step predictor of an n-unknown template."""
    return 3 * n + 1, n


def learned_transient(L, topts, net: int = 0, warm_steps: int = 1000, lane_stride: int = 64, capacity: int = 262144,
                      opts: Optional[TrainOpts] = None, seed: int = 7, steps_per_launch: int = 100000):
    """Runs the transient of every lane of `L` (a Lanes whose espl_init_steps
    has not run yet) with a learned step predictor on template `net`:
    `warm_steps` steps with the linear predictor while the recorder samples
    every `lane_stride`-th lane, training on the device, then the rest with
    predictor 2. Returns (reports, mlp, info)."""
    import time
    n = L.nets[net].n
    L.record_steps(net, lane_stride, 0, capacity)
    # predictor 2 without a network is the linear predictor
    topts.predictor = 2
    L.init_steps(topts)
    t0 = time.perf_counter()
    reps = L.device_launch(warm_steps)
    warm_reports = reps
    t_warm = time.perf_counter() - t0
    x_ptr, y_ptr, count = L.recorded(net)
    d_in, d_out = step_predictor_dims(n)
    opts = opts or train_opts(epochs=20, batch=4096, lr=3e-3, lr_final=3e-4)
    m = Mlp(d_in, d_out, capacity=max(opts.batch, 128), seed=seed, device=0)
    t1 = time.perf_counter()
    losses = m.train_device(x_ptr, y_ptr, count, opts)
    t_train = time.perf_counter() - t1
    L.record_steps(net, 1, 0, 0)
    L.set_step_predictor(net, m)
    t2 = time.perf_counter()
    while not all(r.status != 0 for r in reps):
        reps = L.device_launch(steps_per_launch)
    t_learned = time.perf_counter() - t2
    return reps, m, dict(samples=count, warm_s=t_warm, train_s=t_train, learned_s=t_learned,
                         final_loss=float(losses[-1]), warm_reports=warm_reports)
