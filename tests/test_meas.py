"""The streaming .meas passes of the oracle (oracle/measure.c, after the
reference's src/output/scan.zig) on CPU: known answers on a sampled sine,
and the passes over an RC transient against its analytic response. The GPU
lanes' passes are checked against these in tests/test_gpu_parity.py."""
import math

import numpy as np
import pytest

from egspice_b200 import abi, decks
from oracle import pyoracle as po

M = abi.meas_pass


@pytest.fixture(scope="module")
def sine():
    t = np.linspace(0.0, 2 * math.pi, 2001)
    return t, np.sin(t)


def test_sine_known_answers(oracle, sine):
    t, v = sine
    s = lambda p: po.meas_series(p, t, v)  # noqa: E731
    assert s(M(abi.MEAS_INTEG, 0, to=math.pi))[0] == pytest.approx(2.0, rel=1e-6)
    assert s(M(abi.MEAS_RMS, 0))[0] == pytest.approx(1 / math.sqrt(2), rel=1e-6)
    assert s(M(abi.MEAS_MAX, 0)) == (1.0, pytest.approx(math.pi / 2))
    assert s(M(abi.MEAS_MIN, 0)) == (-1.0, pytest.approx(3 * math.pi / 2))
    assert s(M(abi.MEAS_AVG, 0, to=math.pi))[0] == pytest.approx(2 / math.pi, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=0.5))[0] == pytest.approx(math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=0.5, fall=1))[0] == pytest.approx(5 * math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=-0.5, rise=1))[0] == pytest.approx(11 * math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=0.5, cross=2))[0] == pytest.approx(5 * math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=0.5, rise=abi.MEAS_LAST))[0] == pytest.approx(math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_WHEN, 0, val=0.5, td=1.0))[0] == pytest.approx(5 * math.pi / 6, rel=1e-5)
    assert s(M(abi.MEAS_FIND_AT, 0, at=1.0))[0] == pytest.approx(math.sin(1.0), rel=2e-6)  # linear between samples
    assert math.isnan(s(M(abi.MEAS_WHEN, 0, val=2.0))[0])


def test_rc_transient_passes(oracle):
    r, c, tr = np.array([1e3, 2e3]), np.array([1e-12, 1e-12]), 0.2e-9
    net = decks.rc_points(2, r, c, tr=tr)
    out, inp = net.node("out"), net.node("in")
    t_end = 6e-9
    opts = abi.tran_opts(t_stop=t_end, dt=1e-12, dt_max=5e-12, method=1, max_iter=20, reltol=1e-4)
    passes = [M(abi.MEAS_WHEN, out, val=0.5), M(abi.MEAS_MAX, inp), M(abi.MEAS_INTEG, inp),
              M(abi.MEAS_FIND_AT, out, at=2e-9), M(abi.MEAS_AVG, inp, from_=1e-9, to=5e-9)]
    val, at, _, reps = po.tran_meas(net, opts, passes)
    assert all(rp.status == 1 for rp in reps)
    for l in range(2):
        rc = r[l] * c[l]
        k = (rc / tr) * (math.exp(tr / rc) - 1)
        t50 = -rc * math.log(0.5 / k)
        assert val[l, 0] == pytest.approx(t50, rel=2e-3)
        assert val[l, 1] == 1.0 and at[l, 1] >= tr
        assert val[l, 2] == pytest.approx(t_end - tr / 2, rel=2e-3)
        assert val[l, 3] == pytest.approx(1 - k * math.exp(-2e-9 / rc), rel=2e-3)
        assert val[l, 4] == pytest.approx(1.0, rel=1e-9)
