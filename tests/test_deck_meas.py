"""`.meas tran` cards read into the lanes' streaming measure passes
(egspice_b200/netlist.py read_measures), on CPU: the passes each card
becomes, the values the oracle's transient gives them on an RC deck against
the analytic response, and the cards outside the lanes' measures refused.
The same deck runs on the GPU in tests/test_gpu_parity.py."""
import math

import numpy as np
import pytest

from egspice_b200 import abi
from egspice_b200.netlist import DeckError, measure_passes, measure_values, read_deck, read_measures

RC_DECK = """RC step response with measures
vin in 0 dc 0 pulse(0 1 0 {tr} {tr} 1 2)
r1 in out rval
c1 out 0 1p
.param tr=0.2n half=0.5
.tran 1p 6n
.meas tran t50 when v(out)=half
.meas tran rise trig v(out) val=0.1 rise=1 targ v(out) val=0.9 rise=1
.meas tran v2n find v(out) at=2n
.meas tran slope2n deriv v(out) at=2n
.meas tran iin find i(vin) at=2n
.meas tran early find v(out) when v(in)=0.5
.meas tran swing pp v(out)
.meas tran top max v(out) from=1n to=5n
.meas tran area integ v(in) to=5n
.end
"""


def _rc(lanes=2):
    r = np.array([1e3, 1.5e3])[:lanes]
    net = read_deck(RC_DECK, lanes=lanes, params={"rval": r})
    return net, r


def test_cards_become_passes():
    net, _ = _rc()
    ms = read_measures(RC_DECK, net, params={"rval": np.array([1e3, 1.5e3])})
    assert [m.name for m in ms] == ["t50", "rise", "v2n", "slope2n", "iin", "early", "swing", "top", "area"]
    out, inp = net.node("out"), net.node("in")
    kinds = [[p.kind for p in m.passes] for m in ms]
    assert kinds == [[abi.MEAS_WHEN], [abi.MEAS_WHEN, abi.MEAS_TARG], [abi.MEAS_FIND_AT], [abi.MEAS_DERIV_AT],
                     [abi.MEAS_FIND_AT], [abi.MEAS_WHEN, abi.MEAS_FIND_WHEN], [abi.MEAS_MAX, abi.MEAS_MIN],
                     [abi.MEAS_MAX], [abi.MEAS_INTEG]]
    assert ms[0].passes[0].row == out and ms[0].passes[0].val == 0.5
    trig, targ = ms[1].passes
    assert (trig.val, trig.rise, targ.val, targ.rise) == (0.1, 1, 0.9, 1)
    assert ms[4].passes[0].row == net.branch_names["vin"]
    assert ms[5].passes[0].row == inp and ms[5].passes[1].row == out
    assert ms[7].passes[0].from_ == 1e-9 and ms[7].passes[0].to == 5e-9
    assert ms[6].pp and len(measure_passes(ms)) == 12


def test_rc_measures_against_the_analytic_response(oracle):
    net, r = _rc()
    ms = read_measures(RC_DECK, net, params={"rval": r})
    opts = abi.tran_opts(t_stop=6e-9, dt=1e-12, dt_max=5e-12, method=1, max_iter=20, reltol=1e-4)
    val, _, _, reps = oracle.tran_meas(net, opts, measure_passes(ms))
    assert all(rp.status == 1 for rp in reps)
    got = measure_values(ms, val)
    tr = 0.2e-9
    for l in range(2):
        rc = r[l] * 1e-12
        k = (rc / tr) * (math.exp(tr / rc) - 1)  # v(out) = 1 - k exp(-t / rc) past the ramp
        assert got["t50"][l] == pytest.approx(-rc * math.log(0.5 / k), rel=2e-3)
        assert got["rise"][l] == pytest.approx(rc * math.log(9.0), rel=2e-3)
        assert got["v2n"][l] == pytest.approx(1 - k * math.exp(-2e-9 / rc), rel=2e-3)
        assert got["slope2n"][l] == pytest.approx(k / rc * math.exp(-2e-9 / rc), rel=5e-3)
        # the source's branch current: from its + node through it, -(v_in - v_out) / R
        assert got["iin"][l] == pytest.approx(-k * math.exp(-2e-9 / rc) / r[l], rel=5e-3)
        assert 0 < got["early"][l] < 0.05
        assert got["swing"][l] == pytest.approx(1 - k * math.exp(-6e-9 / rc), rel=2e-3)
        assert got["top"][l] == pytest.approx(1 - k * math.exp(-5e-9 / rc), rel=2e-3)
        assert got["area"][l] == pytest.approx(5e-9 - tr / 2, rel=2e-3)


@pytest.mark.parametrize("card,msg", [
    (".meas dc g1 max v(out)", "only .meas tran"),
    (".meas tran d1 find v(out,in) at=1n", "only v\\(node\\)"),
    (".meas tran d2 trig at=1n targ v(out) val=0.5 rise=1", "AT= is outside"),
    (".meas tran d3 when v(out)=0.5 rise=1 fall=1", "one of RISE"),
    (".meas tran d4 when v(nowhere)=0.5", "no node"),
    (".meas tran d5 when v(out)=0.5 rise=0", "count from 1"),
    (".meas tran d6 when v(out)=rval", "same on every lane"),
    (".meas tran d7 find v(out) when v(in)=0.5 minat=1", "MINAT"),
    (".meas tran d8 max_at v(out)", "MAX_AT"),
    (".meas tran d9 when v(out)=0.5\n.meas tran d9 max v(out)", "second measure"),
])
def test_measures_outside_the_lanes_are_refused(card, msg):
    net, r = _rc()
    text = RC_DECK.replace(".end", card + "\n.end")
    with pytest.raises(DeckError, match=msg):
        read_measures(text, net, params={"rval": r})


def test_too_many_passes_are_refused():
    net, r = _rc()
    text = RC_DECK.replace(".end", "".join(f".meas tran p{k} pp v(out)\n" for k in range(3)) + ".end")
    ms = read_measures(text, net, params={"rval": r})
    with pytest.raises(DeckError, match="a template takes 16"):
        measure_passes(ms)


def test_point_measures_and_reasons():
    """espice_copy_point_measures' rules (include/espice.h :324-338): a
    failed point reads NaN throughout with the first failure's reason; a
    point with a measure that never resolved reads NaN there and names it."""
    from types import SimpleNamespace as R

    from egspice_b200 import netlist as nl
    net, r = _rc()
    ms = read_measures(RC_DECK, net, params={"rval": r})
    lanes, n_pass = 5, len(measure_passes(ms))
    value = np.arange(lanes * n_pass, dtype=np.float64).reshape(lanes, n_pass) + 1.0
    value[3, 0] = np.nan                              # t50 never happened on lane 3
    reports = [R(status=1), R(status=2), R(status=1), R(status=1), R(status=4)]
    op = np.zeros((lanes, 4), dtype=np.uint32)
    op[:, 0] = abi.CONVERGED
    op[2, 0] = abi.SINGULAR                           # lane 2's operating point failed
    out, reasons = nl.point_measures(ms, value, ["T50", "swing"], reports=reports, op=op)
    assert out.shape == (lanes, 2)
    assert list(reasons) == [nl.REASON_OK, nl.REASON_TIMESTEP_TOO_SMALL, nl.REASON_SINGULAR_MATRIX,
                             nl.REASON_MEASURE_UNRESOLVED, nl.REASON_OTHER]
    swing = measure_passes(ms).index(ms[6].passes[0])
    assert out[0, 0] == value[0, 0] and out[0, 1] == value[0, swing] - value[0, swing + 1]
    assert np.isnan(out[1:3]).all() and np.isnan(out[4]).all()
    assert np.isnan(out[3, 0]) and not np.isnan(out[3, 1])
    with pytest.raises(DeckError, match="UnknownMeasure"):
        nl.point_measures(ms, value, ["nope"])


def test_param_measures():
    """`.meas tran name param='expr'` over the measures before it and the
    deck's parameters, per lane; unknown names refused at read time."""
    net, r = _rc()
    text = RC_DECK.replace(".end", ".meas tran mid param='(t50 + rise) / 2 + 0 * half'\n"
                                   ".meas tran scaled param='swing * 1k'\n.end")
    ms = read_measures(text, net, params={"rval": r})
    assert [m.name for m in ms][-2:] == ["mid", "scaled"] and ms[-1].passes == []
    n_pass = len(measure_passes(ms))
    value = np.random.default_rng(1).uniform(1, 2, size=(2, n_pass))
    got = measure_values(ms, value)
    np.testing.assert_allclose(got["mid"], (got["t50"] + got["rise"]) / 2)
    np.testing.assert_allclose(got["scaled"], got["swing"] * 1e3)
    bad = RC_DECK.replace(".end", ".meas tran oops param='t50 + nosuch'\n.end")
    with pytest.raises(DeckError, match="unknown parameter 'nosuch'"):
        read_measures(bad, net, params={"rval": r})
    later = RC_DECK.replace(".meas tran t50 when v(out)=half", ".meas tran early2 param='t50 * 2'\n"
                                                               ".meas tran t50 when v(out)=half")
    with pytest.raises(DeckError, match="unknown parameter 't50'"):
        read_measures(later, net, params={"rval": r})


def test_stopped_lanes_count_as_done_only_when_asked():
    from types import SimpleNamespace as R

    from egspice_b200 import netlist as nl
    net, r = _rc()
    ms = read_measures(RC_DECK, net, params={"rval": r})
    value = np.ones((2, len(measure_passes(ms))))
    reports = [R(status=4), R(status=1)]
    _, reasons = nl.point_measures(ms, value, ["t50"], reports=reports)
    assert list(reasons) == [nl.REASON_OTHER, nl.REASON_OK]
    _, reasons = nl.point_measures(ms, value, ["t50"], reports=reports, stopped_ok=True)
    assert list(reasons) == [nl.REASON_OK, nl.REASON_OK]
