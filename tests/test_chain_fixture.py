"""The reference's lane lockstep fixture (src/tests/espice.zig:3072-3122,
extracted into tests/golden/chain_deck.json by extract_chain_deck.py): an
8-stage inverter chain with RC wires written with a subcircuit, three
TRIG/TARG measures, and 19 rows of (wn, wp, rw, cw, td): 16 sizings, a moved
input edge, an extreme wire and a shorted wire with a negative capacitance.
On CPU: the deck reads, the oracle's measures behave as the rows were drawn
to make them (the moved edge keeps the delays, the extreme wire never
switches), and the points layer refuses the shorted row as appended. The
GPU lanes run the rows in three orders in tests/test_gpu_parity.py."""
import json
import os

import numpy as np
import pytest

from egspice_b200 import abi
from egspice_b200 import points as pt
from egspice_b200.netlist import measure_passes, measure_values, read_deck, read_measures

FIXTURE = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "chain_deck.json")))
ROWS = np.array(FIXTURE["rows"])
LIVE = FIXTURE["live"]


def test_deck_reads():
    net = read_deck(FIXTURE["deck"], lanes=2, params={k: ROWS[:2, j] for j, k in enumerate(LIVE)})
    assert net.n == 21  # 8 stages x (y, z) + in + vdd + ground + two branches
    assert {"n8", "x1.y", "x8.y"} <= set(net.node_names)
    ms = read_measures(FIXTURE["deck"], net, params={k: ROWS[:2, j] for j, k in enumerate(LIVE)})
    assert [m.name for m in ms] == ["tpd", "trise", "tfall"]
    assert all([p.kind for p in m.passes] == [abi.MEAS_WHEN, abi.MEAS_TARG] for m in ms)


def test_oracle_measures_on_the_rows(oracle):
    rows = ROWS[:18]
    params = {k: rows[:, j] for j, k in enumerate(LIVE)}
    net = read_deck(FIXTURE["deck"], lanes=len(rows), params=params)
    ms = read_measures(FIXTURE["deck"], net, params=params)
    opts = pt.Points(FIXTURE["deck"], LIVE).topts
    vo, _, _, ro = oracle.tran_meas(net, opts, measure_passes(ms), threads=8)
    assert all(r.status == 1 for r in ro)
    w = measure_values(ms, vo)
    for name in ("tpd", "trise", "tfall"):
        assert np.isfinite(w[name][:17]).all(), name
        assert (w[name][:16] > 0).all()
        # row 16 moves the input edge from 20 ps to 37 ps: the same delays
        assert w[name][16] == pytest.approx(w[name][0], rel=1e-3)
        assert np.isnan(w[name][17])  # a 1 GOhm wire: n8 never switches
    assert w["tpd"][:16].max() > 3 * w["tpd"][:16].min()  # the sizings spread the delay


def test_points_refuse_the_shorted_row():
    p = pt.Points(FIXTURE["deck"], LIVE)
    assert p.append_points(ROWS) == 0
    assert p.state[:18] == [0] * 18 and p.state[18] == 1
    v, r = p.copy_point_measures(18, 1, ["tpd"])
    assert np.isnan(v).all() and r[0] == pt.REASON_TOPOLOGY_CHANGED
