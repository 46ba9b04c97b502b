"""Noise on the AC lanes, host side (egspice_b200/lanes.py noise_terminals,
noise_sum) and the oracle's densities (oracle/pyoracle.py noise_densities,
after the reference's models: resistor.va 4kT/R, diode.va:326 2q|Id|,
mos1.va:480-489 4kT (2/3)|gm|), on CPU: an RC low pass against its
analytic output noise 4kTR / (1 + (wRC)^2), whose integral over frequency
is kT/C. The GPU densities (espl_noise_sources) and adjoint solves are
checked in tests/test_gpu_parity.py."""
import numpy as np

from egspice_b200 import abi, decks
from egspice_b200.lanes import noise_sum, noise_terminals
from oracle import pyoracle as po


def test_rc_output_noise(oracle):
    r, c = np.array([1e3, 5e3]), np.array([1e-12, 2e-13])
    net = decks.rc_points(2, r, c)
    x, res = oracle.op_lanes(net, abi.newton_opts())
    terms = noise_terminals(net)
    assert len(terms) == 1  # the resistor
    psd = po.noise_densities(net, x)
    np.testing.assert_allclose(psd[:, 0], po.KT4 / r, rtol=1e-12)
    om = np.logspace(4, 13, 400)
    e = np.zeros((1, net.n), dtype=complex)
    e[0, net.node("out")] = 1.0
    z = po.ac_solve_lanes(net, x, om, e, np.arange(net.n), adjoint=True)[:, :, 0, :]
    s = noise_sum(psd, z, terms)
    want = po.KT4 * r[:, None] / (1.0 + (om[None, :] * (r * c)[:, None]) ** 2)
    np.testing.assert_allclose(s, want, rtol=1e-9)
    np.testing.assert_allclose(po.noise_lanes(net, x, om, net.node("out"), terms), want, rtol=1e-9)
    # integrated over f = w / 2 pi: kT / C
    f = om / (2 * np.pi)
    total = np.trapezoid(s, f, axis=1) + s[:, -1] * f[-1]  # the tail beyond f[-1] falls as 1/f^2
    np.testing.assert_allclose(total, po.KT4 / 4 / c, rtol=2e-3)


def test_terminals_follow_the_source_order():
    net = decks.miller_opamp(1)
    t = noise_terminals(net)
    kinds = [b.kind for b in net.batches]
    n_res = sum(len(b.term) for b in net.batches if b.kind == decks.RES)
    n_mos = sum(len(b.term) for b in net.batches if b.kind == decks.MOS1)
    assert len(t) == n_res + n_mos and decks.MOS1 in kinds
    mos = [b for b in net.batches if b.kind == decks.MOS1][0]
    want = np.asarray(mos.term, dtype=np.int64)[:, [0, 2]]
    np.testing.assert_array_equal(t[n_res:], np.where(want == decks.GROUND, net.n, want))
    assert noise_sum(np.zeros((1, 0)), np.zeros((1, 3, net.n)), t[:0]).shape == (1, 3)
