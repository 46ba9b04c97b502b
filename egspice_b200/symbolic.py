"""Host symbolic seam of the lane library (no GPU needed): the BTF/AMD
column order and the lead lane's pivot tape, through the C ABI."""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from .abi import f64p, u32p
from .lanes import LaneError, lib


def _setup(L):
    if getattr(L, "_sym_ready", False):
        return L
    L.espl_order.argtypes = [C.c_uint32, u32p, u32p, u32p]
    L.espl_order.restype = C.c_uint32
    L.espl_tape_build.argtypes = [C.c_uint32, u32p, u32p, f64p, u32p, C.POINTER(C.c_void_p)]
    L.espl_tape_build.restype = C.c_uint32
    L.espl_tape_sizes.argtypes = [C.c_void_p, u32p, u32p, u32p]
    L.espl_tape_sizes.restype = C.c_uint32
    L.espl_tape_copy.argtypes = [C.c_void_p] + [u32p] * 9 + [f64p] * 3
    L.espl_tape_copy.restype = C.c_uint32
    L.espl_tape_free.argtypes = [C.c_void_p]
    L._sym_ready = True
    return L


def order(col_ptr, row_idx) -> Optional[np.ndarray]:
    L = _setup(lib())
    cp = np.ascontiguousarray(col_ptr, dtype=np.uint32)
    ri = np.ascontiguousarray(row_idx, dtype=np.uint32)
    n = len(cp) - 1
    q = np.zeros(max(n, 1), dtype=np.uint32)
    st = L.espl_order(n, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p), q.ctypes.data_as(u32p))
    return None if st != 0 else q[:n]


def tape(col_ptr, row_idx, vals, q) -> Optional[Dict[str, np.ndarray]]:
    L = _setup(lib())
    cp = np.ascontiguousarray(col_ptr, dtype=np.uint32)
    ri = np.ascontiguousarray(row_idx, dtype=np.uint32)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    qq = np.ascontiguousarray(q, dtype=np.uint32)
    n = len(cp) - 1
    h = C.c_void_p()
    st = L.espl_tape_build(n, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p), v.ctypes.data_as(f64p),
                           qq.ctypes.data_as(u32p), C.byref(h))
    if st != 0:
        return None
    try:
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        L.espl_tape_sizes(h, C.byref(a), C.byref(b), C.byref(c))
        nl, nu, nv = a.value, b.value, c.value
        nnz = int(cp[-1])
        sz = {"q": n, "pinv": n, "lp": n + 1, "li": nl, "up": n + 1, "ui": nu, "flags": n, "prow": nnz,
              "void_slots": nv}
        out = {k: np.zeros(max(s, 1), dtype=np.uint32) for k, s in sz.items()}
        fl = {"lx": nl, "ux": nu, "udiag": n}
        outf = {k: np.zeros(max(s, 1)) for k, s in fl.items()}
        L.espl_tape_copy(h, *[out[k].ctypes.data_as(u32p) for k in sz], *[outf[k].ctypes.data_as(f64p) for k in fl])
        res = {k: out[k][:sz[k]] for k in sz}
        res.update({k: outf[k][:fl[k]] for k in fl})
        return res
    finally:
        L.espl_tape_free(h)
