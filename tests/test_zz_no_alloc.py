"""espl_tape_replay_noalloc, the replay entry point that allocates nothing,
called through the C ABI against the existing entry point for the same
factor: espl_tape_build + espl_tape_copy (the host factor of the lead
lane's values). Lanes carry the lead values scaled by powers of two, which
scale U and the pivots exactly and leave L unchanged, so the lanes' factors
must relate bit for bit by those scales, and each must match the host factor
to 1e-13 relative (the device contracts w -= l * u into one fused
multiply-add, the host rounds the product and the difference separately).
Two calls in a row with different lane counts must give the same bits for
the same scale, which checks that the shared work vector comes back to zero.
This file is collected last so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

from egspice_b200 import decks

pytestmark = pytest.mark.gpu

u32p = C.POINTER(C.c_uint32)
f64p = C.POINTER(C.c_double)
ESPL_TOO_LARGE = 8


def _lib():
    from egspice_b200.lanes import lib
    L = lib()
    L.espl_tape_build.argtypes = [C.c_uint32, u32p, u32p, f64p, u32p, C.POINTER(C.c_void_p)]
    L.espl_tape_build.restype = C.c_uint32
    L.espl_tape_sizes.argtypes = [C.c_void_p, u32p, u32p, u32p]
    L.espl_tape_sizes.restype = C.c_uint32
    L.espl_tape_copy.argtypes = [C.c_void_p] + [u32p] * 9 + [f64p] * 3
    L.espl_tape_copy.restype = C.c_uint32
    L.espl_tape_free.argtypes = [C.c_void_p]
    L.espl_tape_free.restype = None
    L.espl_tape_replay_noalloc.argtypes = [C.c_void_p, u32p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    L.espl_tape_replay_noalloc.restype = C.c_uint32
    return L


def _values(net):
    """A deterministic diagonally weighted fill of the pattern."""
    cp, ri = np.asarray(net.col_ptr), np.asarray(net.row_idx)
    v = np.empty(len(ri))
    for c in range(net.n):
        for p in range(cp[c], cp[c + 1]):
            r = ri[p]
            v[p] = 4.0 + 0.25 * ((r * 7 + c * 3) % 5) if r == c else -0.5 - 0.125 * ((r + 2 * c) % 3)
    return v


def _host_factor(L, net, vals):
    cp = np.ascontiguousarray(net.col_ptr, dtype=np.uint32)
    ri = np.ascontiguousarray(net.row_idx, dtype=np.uint32)
    from egspice_b200 import symbolic
    q = np.ascontiguousarray(symbolic.order(cp, ri), dtype=np.uint32)
    h = C.c_void_p()
    st = L.espl_tape_build(net.n, cp.ctypes.data_as(u32p), ri.ctypes.data_as(u32p), vals.ctypes.data_as(f64p),
                           q.ctypes.data_as(u32p), C.byref(h))
    assert st == 0
    a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    L.espl_tape_sizes(h, C.byref(a), C.byref(b), C.byref(c))
    lx, ux, ud = np.zeros(max(a.value, 1)), np.zeros(max(b.value, 1)), np.zeros(net.n)
    nul = C.cast(None, u32p)
    L.espl_tape_copy(h, *([nul] * 9), lx.ctypes.data_as(f64p), ux.ctypes.data_as(f64p), ud.ctypes.data_as(f64p))
    return h, cp, lx[:a.value], ux[:b.value], ud


def _replay(L, h, cp, vals, scales, nl, nu, n):
    import torch
    lanes = len(scales)
    dev = torch.device("cuda:0")
    a = torch.tensor(np.outer(vals, scales), dtype=torch.float64, device=dev).contiguous()
    lx = torch.full((max(nl, 1), lanes), np.nan, dtype=torch.float64, device=dev)
    ux = torch.full((max(nu, 1), lanes), np.nan, dtype=torch.float64, device=dev)
    ud = torch.full((n, lanes), np.nan, dtype=torch.float64, device=dev)
    stat = torch.full((lanes,), 7, dtype=torch.int32, device=dev)
    err = C.create_string_buffer(256)
    st = L.espl_tape_replay_noalloc(h, cp.ctypes.data_as(u32p), a.data_ptr(), lanes, lx.data_ptr(), ux.data_ptr(),
                                    ud.data_ptr(), stat.data_ptr(), None, err, 256)
    assert st == 0, err.value
    torch.cuda.synchronize()
    return lx.cpu().numpy()[:nl], ux.cpu().numpy()[:nu], ud.cpu().numpy(), stat.cpu().numpy()


@pytest.mark.parametrize("stages", [15, 31])
def test_noalloc_replay_matches_the_host_factor_twice(stages):
    L = _lib()
    net = decks.ring_oscillator(2, stages=stages)
    vals = _values(net)
    h, cp, lx0, ux0, ud0 = _host_factor(L, net, vals)
    try:
        unit = {}
        for lanes, shift in ((64, 3), (40, 5)):
            scales = 2.0 ** ((np.arange(lanes) % 7) - shift)
            lx, ux, ud, stat = _replay(L, h, cp, vals, scales, len(lx0), len(ux0), net.n)
            assert (stat == 0).all()
            # unscaled, every lane is the same factor, bit for bit
            lxu, uxu, udu = lx, ux / scales, ud / scales
            for k in range(1, lanes):
                assert np.array_equal(lxu[:, k], lxu[:, 0])
                assert np.array_equal(uxu[:, k], uxu[:, 0])
                assert np.array_equal(udu[:, k], udu[:, 0])
            # the same factor as the host's
            np.testing.assert_allclose(lxu[:, 0], lx0, rtol=1e-13, atol=0)
            np.testing.assert_allclose(uxu[:, 0], ux0, rtol=1e-13, atol=0)
            np.testing.assert_allclose(udu[:, 0], ud0, rtol=1e-13, atol=0)
            # and the same bits as the previous call
            for name, arr in (("lx", lxu[:, 0]), ("ux", uxu[:, 0]), ("ud", udu[:, 0])):
                if name in unit:
                    assert np.array_equal(arr, unit[name])
                unit[name] = arr.copy()
    finally:
        L.espl_tape_free(h)


def test_noalloc_replay_refuses_sizes_past_its_scratch():
    L = _lib()
    net = decks.ring_oscillator(2, stages=63)
    vals = _values(net)
    h, cp, lx0, ux0, ud0 = _host_factor(L, net, vals)
    try:
        lanes = (8 << 20) // (8 * net.n) + 1  # the work vector alone is past the limit
        err = C.create_string_buffer(256)
        st = L.espl_tape_replay_noalloc(h, cp.ctypes.data_as(u32p), 1, lanes, 1, 1, 1, 1, None, err, 256)
        assert st == ESPL_TOO_LARGE
        assert b"limit" in err.value
    finally:
        L.espl_tape_free(h)
