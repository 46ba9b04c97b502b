"""The .meas passes that read a second vector or the pass before them
(DERIV ... AT, FIND/DERIV ... WHEN, TRIG/TARG, WHEN against a level vector;
after the reference's src/output/scan.zig Cross/At/Find and the TARG stage
of src/output/measure.zig Stream.next), on CPU:

* known answers of the oracle (oracle/measure.c) on sampled sines;
* the kernels' own measure code (egspice_b200/csrc/lane_meas.cuh, compiled
  for the host by tests/meas_host.cpp) against the oracle, bit for bit, on
  seeded random sample tables and pass lists of every kind.

The GPU lanes run the same passes inside the transient in
tests/test_gpu_parity.py."""
import ctypes as C
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from egspice_b200 import abi
from egspice_b200.abi import MeasPass
from oracle import pyoracle as po

M = abi.meas_pass
MAX_PASSES = 16  # ESPL_MEAS_MAX_PASSES
HERE = os.path.dirname(os.path.abspath(__file__))
f64p = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def device_meas(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("meas") / "libmeas_host.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out, os.path.join(HERE, "meas_host.cpp")],
                   check=True)
    lib = C.CDLL(out)
    lib.dev_meas_table.argtypes = [C.POINTER(MeasPass), C.c_uint32, f64p, f64p, C.c_uint32, C.c_uint32, f64p, f64p]
    lib.dev_meas_table.restype = C.c_int

    def run(passes, xs, cols):
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        cols = np.ascontiguousarray(cols, dtype=np.float64)
        n = len(passes)
        arr = (MeasPass * max(n, 1))(*passes)
        val = np.full(max(n, 1), np.nan)
        at = np.full(max(n, 1), np.nan)
        assert lib.dev_meas_table(arr, n, xs.ctypes.data_as(f64p), cols.ctypes.data_as(f64p), cols.shape[1],
                                  len(xs), val.ctypes.data_as(f64p), at.ctypes.data_as(f64p)) == 0
        return val[:n], at[:n]

    return run


def _sines(t_end, n=4001):
    t = np.linspace(0.0, t_end, n)
    return t, np.stack([np.sin(t), np.cos(t)], axis=1)


def test_known_answers(oracle):
    t, cols = _sines(2 * math.pi)
    SIN, COS = 0, 1
    passes = [
        M(abi.MEAS_DERIV_AT, SIN, at=1.0),                          # d sin / dt at 1 = cos 1
        M(abi.MEAS_WHEN, SIN, val=0.5),                             # pi / 6
        M(abi.MEAS_FIND_WHEN, COS),                                 # cos(pi / 6)
        M(abi.MEAS_WHEN, SIN, val=0.5, fall=1),                     # 5 pi / 6
        M(abi.MEAS_DERIV_WHEN, SIN),                                # cos(5 pi / 6)
        M(abi.MEAS_WHEN, SIN, level_row=COS),                       # sin = cos: pi / 4
        M(abi.MEAS_WHEN, SIN, level_row=COS, cross=2),              # 5 pi / 4
        M(abi.MEAS_WHEN, SIN, val=0.5, rise=1),                     # TRIG at pi / 6
        M(abi.MEAS_TARG, SIN, val=0.5, fall=1),                     # TARG at 5 pi / 6
        M(abi.MEAS_WHEN, SIN, val=2.0),                             # never
        M(abi.MEAS_FIND_WHEN, COS),                                 # so NaN
    ]
    val, at = po.meas_table(passes, t, cols)
    assert val[0] == pytest.approx(math.cos(1.0), rel=2e-3)
    assert val[1] == pytest.approx(math.pi / 6, rel=1e-5)
    assert val[2] == pytest.approx(math.cos(math.pi / 6), rel=1e-5) and at[2] == val[1]
    assert val[4] == pytest.approx(math.cos(5 * math.pi / 6), rel=2e-3) and at[4] == val[3]
    assert val[5] == pytest.approx(math.pi / 4, rel=1e-5)
    assert val[6] == pytest.approx(5 * math.pi / 4, rel=1e-5)
    assert val[8] == pytest.approx(2 * math.pi / 3, rel=1e-5) and at[8] == pytest.approx(5 * math.pi / 6, rel=1e-5)
    assert math.isnan(val[9]) and math.isnan(val[10])


def test_targ_counts_from_the_trigger(oracle):
    """TARG's RISE=1 is the first rise after the TRIG event, not after t = 0
    (ngspice: TARG's TD is the TRIG time)."""
    t, cols = _sines(4 * math.pi, 8001)
    passes = [M(abi.MEAS_WHEN, 0, val=-0.5, fall=1),   # TRIG at 7 pi / 6
              M(abi.MEAS_TARG, 0, val=0.5, rise=1),    # the rise at 2 pi + pi / 6
              M(abi.MEAS_WHEN, 0, val=0.5, rise=1)]    # an independent WHEN: pi / 6
    val, at = po.meas_table(passes, t, cols)
    assert at[1] == pytest.approx(2 * math.pi + math.pi / 6, rel=1e-5)
    assert val[1] == pytest.approx(math.pi, rel=1e-5)
    assert val[2] == pytest.approx(math.pi / 6, rel=1e-5)


def test_passes_reading_a_late_when_stay_unresolved(oracle):
    """A FIND ... WHEN whose WHEN resolves only at the end of the run (LAST
    with no TO) never arms while the run streams."""
    t, cols = _sines(2 * math.pi)
    passes = [M(abi.MEAS_WHEN, 0, val=0.5, rise=abi.MEAS_LAST), M(abi.MEAS_FIND_WHEN, 1)]
    val, _ = po.meas_table(passes, t, cols)
    assert val[0] == pytest.approx(math.pi / 6, rel=1e-5)
    assert math.isnan(val[1])


def _random_table(rng):
    n = int(rng.integers(2, 400))
    steps = rng.uniform(0.2, 2.0, size=n - 1)
    for _ in range(int(rng.integers(0, 4))):  # runs of equal steps (Simpson panels)
        a = int(rng.integers(0, n - 1))
        steps[a:a + int(rng.integers(2, 12))] = steps[a]
    t = np.concatenate([[0.0], np.cumsum(steps)])
    walk = np.cumsum(rng.normal(size=n)) * 0.3
    wave = np.sin(t * rng.uniform(0.1, 1.0)) + 0.05 * rng.normal(size=n)
    flat = np.where(rng.uniform(size=n) < 0.5, 0.0, 1.0)  # samples on the level
    return t, np.stack([walk, wave, flat], axis=1)


def _random_pass(rng, kind, t, cols):
    u = int(rng.integers(0, cols.shape[1]))
    col = cols[:, u]
    kw = {}
    if kind in (abi.MEAS_WHEN, abi.MEAS_TARG):
        kw["val"] = float(rng.choice([rng.uniform(col.min(), col.max()), 0.0, 1.0, col[int(rng.integers(len(col)))]]))
        counts = [abi.MEAS_UNSET, abi.MEAS_LAST, 1, 2, 3]
        which = rng.integers(0, 4)
        if which < 3:
            kw[("rise", "fall", "cross")[which]] = int(rng.choice(counts))
        if rng.uniform() < 0.3:
            kw["level_row"] = int(rng.integers(0, cols.shape[1]))
        if kind == abi.MEAS_WHEN and rng.uniform() < 0.3:
            kw["td"] = float(rng.uniform(0, t[-1] / 2))
    elif kind in (abi.MEAS_FIND_AT, abi.MEAS_DERIV_AT):
        kw["at"] = float(rng.choice([rng.uniform(-1, t[-1] + 1), t[int(rng.integers(len(t)))]]))
    if kind not in (abi.MEAS_FIND_AT, abi.MEAS_DERIV_AT, abi.MEAS_FIND_WHEN, abi.MEAS_DERIV_WHEN) \
            and rng.uniform() < 0.4:
        a, b = sorted(rng.uniform(0, t[-1], size=2))
        kw["from_"] = float(rng.choice([a, t[int(rng.integers(len(t)))], 0.0]))
        kw["to"] = float(rng.choice([b, t[int(rng.integers(len(t)))], 0.0]))
    return M(kind, u, **kw)


def test_device_passes_match_the_oracle_bitwise(oracle, device_meas):
    rng = np.random.default_rng(20261203)
    chained = (abi.MEAS_FIND_WHEN, abi.MEAS_DERIV_WHEN, abi.MEAS_TARG)
    plain = (abi.MEAS_WHEN, abi.MEAS_FIND_AT, abi.MEAS_DERIV_AT, abi.MEAS_MIN, abi.MEAS_MAX, abi.MEAS_AVG,
             abi.MEAS_INTEG, abi.MEAS_RMS)
    resolved = {k: 0 for k in plain + chained}
    for _ in range(400):
        t, cols = _random_table(rng)
        passes = []
        want = int(rng.integers(1, MAX_PASSES + 1))
        while len(passes) < want:
            kind = int(rng.choice(plain))
            passes.append(_random_pass(rng, kind, t, cols))
            if kind == abi.MEAS_WHEN and rng.uniform() < 0.6 and len(passes) < MAX_PASSES:
                passes.append(_random_pass(rng, int(rng.choice(chained)), t, cols))
        ov, oa = po.meas_table(passes, t, cols)
        dv, da = device_meas(passes, t, cols)
        np.testing.assert_array_equal(dv, ov)
        np.testing.assert_array_equal(da, oa)
        for p, v in zip(passes, ov):
            resolved[p.kind] += not math.isnan(v)
    # every kind produced values, not only NaNs that trivially agree
    assert min(resolved.values()) >= 20, resolved


def test_library_host_table_matches_the_oracle(oracle):
    """espl_meas_table, the product's host entry running the kernels' measure
    code over a table (AC sweeps use it), bit for bit against the oracle."""
    from egspice_b200.lanes import meas_table
    rng = np.random.default_rng(7)
    chained = (abi.MEAS_FIND_WHEN, abi.MEAS_DERIV_WHEN, abi.MEAS_TARG)
    plain = (abi.MEAS_WHEN, abi.MEAS_FIND_AT, abi.MEAS_DERIV_AT, abi.MEAS_MIN, abi.MEAS_MAX, abi.MEAS_AVG,
             abi.MEAS_INTEG, abi.MEAS_RMS)
    for _ in range(100):
        t, cols = _random_table(rng)
        passes = []
        while len(passes) < 8:
            kind = int(rng.choice(plain))
            passes.append(_random_pass(rng, kind, t, cols))
            if kind == abi.MEAS_WHEN:
                passes.append(_random_pass(rng, int(rng.choice(chained)), t, cols))
        ov, oa = po.meas_table(passes, t, cols)
        lv, la = meas_table(passes, t, cols)
        np.testing.assert_array_equal(lv, ov)
        np.testing.assert_array_equal(la, oa)


def test_library_host_table_refuses_bad_passes():
    from egspice_b200.lanes import LaneError, meas_table
    t, cols = _sines(1.0, 11)
    for passes in ([M(abi.MEAS_FIND_WHEN, 0)],                              # no WHEN before it
                   [M(abi.MEAS_MAX, 0), M(abi.MEAS_TARG, 0, val=0.1)],      # TARG after a non-WHEN
                   [M(abi.MEAS_MAX, 2)],                                    # column out of range
                   [M(abi.MEAS_WHEN, 0, level_row=2)],                      # level column out of range
                   [M(99, 0)]):                                             # unknown kind
        with pytest.raises(LaneError, match="status 1"):
            meas_table(passes, t, cols)
    v, a = meas_table([], t, cols)
    assert v.size == 0 and a.size == 0
