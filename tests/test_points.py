"""The points API mirror (egspice_b200/points.py, after include/espice.h
:244-362) on CPU: the template's checks at creation, append_points' ids and
refusals, copy_point_measures' and release_points' errors. Running points
needs the GPU lanes (tests/test_gpu_parity.py test_points_*)."""
import numpy as np
import pytest

from egspice_b200 import points as pt
from egspice_b200.netlist import DeckError, parse_number

DECK = """RC points
vin in 0 dc 0 pulse(0 1 0 0.2n 0.2n 1 2)
r1 in out {rval}
c1 out 0 {cval}
.param rval=1k cval=1p lvl=0.5
.tran 1p 6n
.meas tran t50 when v(out)=lvl
.meas tran v2n find v(out) at=2n
.end
"""


def test_template_checks():
    p = pt.Points(DECK, ["rval", "cval"])
    assert [m.name for m in p.measures] == ["t50", "v2n"]
    # numbers as ngspice reads them; TMAX = min(TSTEP, TSTOP / 50)
    assert p.topts.t_stop == parse_number("6n") and p.topts.dt_max == parse_number("1p")
    assert pt.Points.lane_width() == 16384
    with pytest.raises(DeckError, match="neither a .tran nor an .op"):
        pt.Points(DECK.replace(".tran 1p 6n\n", ""), ["rval"])
    with pytest.raises(DeckError, match="UIC"):
        pt.Points(DECK.replace(".tran 1p 6n", ".tran 1p 6n uic"), ["rval"])
    with pytest.raises(pt.PointsError, match="SweptTemplate"):
        pt.Points(DECK.replace(".end", ".step param rval 1k 2k 1k\n.end"), ["rval"])
    with pytest.raises(DeckError, match="same on every lane"):
        pt.Points(DECK, ["rval", "lvl"])  # a measure reads a live parameter


def test_append_copy_release():
    p = pt.Points(DECK, ["rval", "cval"])
    assert p.append_points([[1e3, 1e-12], [2e3, 1e-12]]) == 0
    assert p.append_points([[1e3, np.nan]]) == 2          # appended already failed
    with pytest.raises(pt.PointsError) as e:
        p.append_points(np.zeros((0, 2)))
    assert e.value.status == pt.INVALID_ARGUMENT
    with pytest.raises(pt.PointsError) as e:
        p.copy_point_measures(0, 2, ["t50"])               # not run yet
    assert e.value.status == pt.RESULT_UNAVAILABLE
    v, r = p.copy_point_measures(2, 1, ["T50", "v2n"])      # the refused point is complete
    assert np.isnan(v).all() and list(r) == [pt.REASON_INVALID_PARAMETER]
    with pytest.raises(pt.PointsError) as e:
        p.copy_point_measures(1, 5, ["t50"])
    assert e.value.status == pt.INVALID_QUERY
    with pytest.raises(pt.PointsError) as e:
        p.copy_point_measures(2, 1, ["nope"])
    assert (e.value.status, e.value.name) == (pt.INVALID_ARGUMENT, "UnknownMeasure")
    p.release_points(2, 1)
    with pytest.raises(pt.PointsError) as e:
        p.copy_point_measures(2, 1, ["t50"])
    assert e.value.status == pt.RESULT_UNAVAILABLE
    with pytest.raises(pt.PointsError, match="NoLiveParameters"):
        pt.Points(DECK, []).append_points([[1.0]])


def test_op_decks_and_op_measures():
    op_deck = """leakage of a divider
vdd vdd 0 1.8
r1 vdd mid {rtop}
r2 mid 0 10k
.param rtop=10k
.op
.meas op vmid find v(mid)
.meas op idd find i(vdd)
.end
"""
    p = pt.Points(op_deck, ["rtop"])
    assert p.topts is None and p.need_op
    assert [m.op_row is not None for m in p.measures] == [True, True]
    with pytest.raises(DeckError, match="needs the deck's .tran"):
        pt.Points(op_deck.replace(".end", ".meas tran t1 max v(mid)\n.end"), ["rtop"])
    with pytest.raises(DeckError, match="neither a .tran nor an .op"):
        pt.Points(op_deck.replace(".op\n", ""), ["rtop"])
    with pytest.raises(DeckError, match="FIND vector"):
        pt.Points(op_deck.replace("find v(mid)", "max v(mid)"), ["rtop"])
    q = pt.Points(DECK.replace(".end", ".meas op v0 find v(out)\n.end"), ["rval", "cval"])
    assert q.topts is not None and q.need_op
