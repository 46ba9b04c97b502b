"""The small-signal AC restatement of the oracle (pyoracle.ac_lanes: G and C
from the oracle's device models at the operating point, a dense complex
solve) on CPU, against the analytic response of an RC low pass. The GPU's
AC lanes (espl_ac) are checked against it in tests/test_gpu_parity.py."""
import numpy as np

from egspice_b200 import abi, decks


def test_rc_low_pass_response(oracle):
    r, c = np.array([1e3, 2e3, 5e3]), np.array([1e-12, 1e-12, 2e-13])
    net = decks.rc_points(3, r, c)
    x, res = oracle.op_lanes(net, abi.newton_opts())
    assert res[:, 0].all()
    om = np.logspace(5, 11, 13)
    h = oracle.ac_lanes(net, x, 0, om, [net.node("out"), net.node("in")])
    exact = 1.0 / (1.0 + 1j * om[None, :] * (r * c)[:, None])
    np.testing.assert_allclose(h[:, :, 0], exact, rtol=1e-12)
    np.testing.assert_allclose(h[:, :, 1], 1.0, rtol=1e-15)
