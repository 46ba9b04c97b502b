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


def test_noalloc_replay_refuses_a_pattern_that_is_not_the_tapes():
    """espl_tape_replay_noalloc checks the caller's col_ptr on the host
    before any device work: a decreasing entry, an entry past nnz or a wrong
    first entry is ESPL_INVALID_ARGUMENT with the reason, so the replay
    never reads past the lanes' values. (The device pointers here are
    stand-ins that the refused call never reads.)"""
    import ctypes as C

    from egspice_b200.lanes import lib
    from egspice_b200 import symbolic
    L = symbolic._setup(lib())
    u32p = C.POINTER(C.c_uint32)
    L.espl_tape_replay_noalloc.argtypes = [C.c_void_p, u32p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    L.espl_tape_replay_noalloc.restype = C.c_uint32
    cp = np.array([0, 2, 4, 6], np.uint32)
    ri = np.array([0, 1, 0, 1, 1, 2], np.uint32)
    vals = np.array([4.0, 1.0, 1.0, 4.0, 1.0, 4.0])
    q = np.ascontiguousarray(symbolic.order(cp, ri), dtype=np.uint32)
    h = C.c_void_p()
    assert L.espl_tape_build(3, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p),
                             vals.ctypes.data_as(C.POINTER(C.c_double)), q.ctypes.data_as(u32p), C.byref(h)) == 0
    fake = C.c_void_p(256)
    try:
        for bad in ([0, 4, 2, 6], [0, 2, 7, 6], [1, 2, 4, 6]):
            b = np.array(bad, np.uint32)
            err = C.create_string_buffer(256)
            st = L.espl_tape_replay_noalloc(h, b.ctypes.data_as(u32p), fake, 4, fake, fake, fake, fake, None, err, 256)
            assert st == 1 and b"col_ptr" in err.value, (bad, st, err.value)
    finally:
        L.espl_tape_free(h)


def test_plan_entry_points_refuse_bad_arguments_without_a_gpu():
    """The launch-plan entry points check their arguments before any device
    work: a NULL handle or output is ESPL_INVALID_ARGUMENT; on a CPU-only
    host the autotuner reports the driver's refusal instead of searching."""
    import ctypes as C
    import torch
    from egspice_b200 import abi, decks
    from egspice_b200.abi import PlanChoice, TuneReport
    from egspice_b200.lanes import lib
    L = lib()
    assert C.sizeof(PlanChoice) == 16 and C.sizeof(TuneReport) == 24
    assert L.espl_set_plan(None, None) == 1
    assert L.espl_get_plan(None, None) == 1
    net = decks.inverter_chain(2)
    keep, arr = abi.cnets([net])
    opts = abi.CreateOpts(abi.ABI_VERSION, 0, 0, 0, 0, 0)
    topts = abi.tran_opts(t_stop=1e-9, dt=1e-12)
    out = (PlanChoice * 1)()
    rep = TuneReport()
    # no templates, no options, no output, or zero trial steps: refused
    assert L.espl_autotune(arr, 0, C.byref(opts), 0.0, C.byref(topts), 10, 4, out, C.byref(rep)) == 1
    assert L.espl_autotune(arr, 1, None, 0.0, C.byref(topts), 10, 4, out, C.byref(rep)) == 1
    assert L.espl_autotune(arr, 1, C.byref(opts), 0.0, C.byref(topts), 0, 4, out, C.byref(rep)) == 1
    if not torch.cuda.is_available():
        st = L.espl_autotune(arr, 1, C.byref(opts), 0.0, C.byref(topts), 10, 4, out, C.byref(rep))
        assert st == 2  # ESPL_NO_IMAGE, as espl_create
