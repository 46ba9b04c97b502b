"""The C-ABI library loads without a GPU and exports every entry point
include/espice_lanes.h declares; the host symbolic seam answers on CPU."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(espl_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from egspice_b200 import abi
    from egspice_b200.lanes import lib
    L = lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), f"{s} missing from the library"
    assert L.espl_abi_version() == abi.ABI_VERSION


def test_create_without_a_gpu_reports_no_image_or_runs():
    """On a CPU-only host espl_create refuses with ESPL_NO_IMAGE (2) and
    leaves the out handle NULL; it never falls back to a CPU path."""
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import lib
    import torch
    if torch.cuda.is_available():
        return
    net = decks.inverter_chain(2)
    keep, arr = abi.cnets([net])
    h = ctypes.c_void_p(1234)
    st = lib().espl_create(arr, 1, None, 0.0, ctypes.byref(h))
    assert st == 2 and not h.value


def test_symbolic_seam_on_cpu():
    from egspice_b200 import symbolic
    cp = np.array([0, 2, 4], np.uint32)
    ri = np.array([0, 1, 0, 1], np.uint32)
    assert list(symbolic.order(cp, ri)) in ([0, 1], [1, 0])
    t = symbolic.tape(cp, ri, [2.0, 1.0, 1.0, 3.0], [0, 1])
    assert list(t["pinv"]) == [0, 1] and len(t["li"]) == 1 and len(t["ui"]) == 1
