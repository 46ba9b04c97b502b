"""AC sweeps as points (egspice_b200/points.py) on CPU: the `.ac` card's
frequencies as ngspice steps them, the AC sources' excitation, and `.meas
ac` cards over magnitude/dB/phase columns through the lanes' measure passes
on the host, on an RC response written out analytically. The lanes' AC
solves themselves run in tests/test_gpu_parity.py."""
import math

import numpy as np
import pytest

from egspice_b200 import points as pt
from egspice_b200.netlist import DeckError, read_deck, read_measures

DECK = """RC AC
vin in 0 dc 0 ac 1
r1 in out {rval}
c1 out 0 1p
.param rval=1k
.ac dec 50 1meg 10g
.meas ac bw when vdb(out)=-3 fall=1
.meas ac g1m find vdb(out) at=1meg
.meas ac ph find vp(out) when vdb(out)=-3
.meas ac peak max vm(out)
.end
"""


def test_frequencies():
    f = pt.ac_frequencies(DECK)
    assert f[0] == 1e6 and f[-1] <= 1e10 * (1 + 1e-12) and len(f) == 201
    np.testing.assert_allclose(f[1] / f[0], 10 ** (1 / 50))
    lin = pt.ac_frequencies(DECK.replace(".ac dec 50 1meg 10g", ".ac lin 5 1k 5k"))
    np.testing.assert_array_equal(lin, [1e3, 2e3, 3e3, 4e3, 5e3])
    oc = pt.ac_frequencies(DECK.replace(".ac dec 50 1meg 10g", ".ac oct 1 1 16"))
    np.testing.assert_allclose(oc, [1, 2, 4, 8, 16])
    with pytest.raises(DeckError, match="dec\\|oct\\|lin"):
        pt.ac_frequencies(DECK.replace(".ac dec 50", ".ac log 50"))


def test_excitation():
    net = read_deck(DECK + "", lanes=1, params={"rval": 1e3})
    b = pt.ac_rhs(net)
    assert b[net.branch_names["vin"]] == 1.0 and np.count_nonzero(b) == 1
    cur = read_deck("i source\ni1 0 out dc 0 ac 2 90\nr1 out 0 1k\n.end\n", lanes=1)
    b = pt.ac_rhs(cur)
    np.testing.assert_allclose(b[cur.node("out")], 2j, atol=1e-15)  # from ground into out


def test_ac_measures_on_an_rc_response():
    r = np.array([1e3, 2e3])
    net = read_deck(DECK, lanes=2, params={"rval": r})
    ms = read_measures(DECK, net, params={"rval": r})
    assert [m.analysis for m in ms] == ["ac"] * 4 and ms[0].columns == [("db", net.node("out"))]
    f = pt.ac_frequencies(DECK)
    w = 2 * np.pi * f
    h = 1.0 / (1.0 + 1j * w[None, :] * (r * 1e-12)[:, None])  # v(out) of the unit AC input
    z = np.zeros((2, len(f), net.n), dtype=complex)
    z[:, :, net.node("out")] = h
    got = pt.ac_measure_values(ms, f, z)
    f3 = math.sqrt(10 ** 0.3 - 1) / (2 * np.pi * r * 1e-12)
    np.testing.assert_allclose(got["bw"], f3, rtol=2e-3)  # linear between sweep points
    np.testing.assert_allclose(got["g1m"], 20 * np.log10(np.abs(h[:, 0])), rtol=1e-12)
    np.testing.assert_allclose(got["ph"], -np.arctan(2 * np.pi * f3 * r * 1e-12), rtol=2e-3)
    np.testing.assert_allclose(got["peak"], np.abs(h[:, 0]), rtol=1e-12)


def test_ac_points_checks():
    p = pt.Points(DECK, ["rval"])
    assert p.freqs is not None and p.need_op and p.topts is None
    with pytest.raises(DeckError, match="needs the deck's .ac"):
        pt.Points(DECK.replace(".ac dec 50 1meg 10g\n", ".op\n"), ["rval"])
    with pytest.raises(DeckError, match="AC value"):
        pt.Points(DECK.replace("ac 1\n", "\n"), ["rval"])
