"""The deck reader (egspice_b200/netlist.py) on CPU: SPICE numbers as
ngspice reads them, and decks written as text that freeze to exactly the
netlists the seeded generators build (pattern, device batches and per-lane
parameters), including a Monte Carlo deck whose per-device draws come in as
per-lane parameters; cards outside the lanes' subset are refused."""
import math

import numpy as np
import pytest

from egspice_b200 import decks
from egspice_b200.netlist import DeckError, parse_number, read_deck


def test_numbers():
    assert parse_number("10meg") == 1e7
    assert parse_number("1k") == 1e3
    assert parse_number("1.8") == 1.8
    assert parse_number("1.8v") == 1.8          # a unit letter scales by 1
    assert parse_number("0.1n") == 1e-10        # one mantissa, then the power of ten
    assert parse_number("2.5u") == 25 * 1e-7
    assert parse_number("1mil") == 25.4 * 1e-6
    assert parse_number("-2.5e3k") == -25 * 1e5
    assert parse_number("1d3") == 1e3
    assert parse_number(".5p") == 5 * 1e-13
    assert parse_number("abc") is None
    assert math.copysign(1.0, parse_number("-0")) == -1.0


def _same(a, b, rtol=0.0):
    assert a.n == b.n and a.nnz == b.nnz
    assert np.array_equal(a.col_ptr, b.col_ptr) and np.array_equal(a.row_idx, b.row_idx)
    ka = sorted(a.batches, key=lambda x: x.kind)
    kb = sorted(b.batches, key=lambda x: x.kind)
    assert [x.kind for x in ka] == [x.kind for x in kb]
    for x, y in zip(ka, kb):
        assert np.array_equal(x.term, y.term), x.kind
        np.testing.assert_allclose(x.param, y.param, rtol=rtol, atol=0)


def test_rc_deck_matches_the_generator():
    r = np.array([1e3, 2e3, 5e3, 1e4])
    c = np.array([1e-12, 0.5e-12, 2e-13, 2e-13])
    text = """RC low pass, one lane per (R, C)
* a pulse into an RC
vin in 0 dc 0 pulse(0 1 0 {tr} {tr} 1 2)
r1 in out rval
c1 out 0 {cval}   ; per lane
.param tr=0.2n
.tran 1p 8n
.end
"""
    net = read_deck(text, lanes=4, params={"rval": r, "cval": c})
    _same(net, decks.rc_points(4, r, c, tr=parse_number("0.2n")))
    assert net.node("out") == decks.rc_points(4, r, c).node("out")


def test_monte_carlo_inverter_chain_matches_the_generator():
    points, stages = 64, 16
    seeds = np.uint64(1) + np.arange(points, dtype=np.uint64)
    params, lines = {}, ["16-stage CMOS inverter chain", "vdd vdd 0 dc 1.8", "vin in 0 0.9"]
    prev = "in"
    for s in range(stages):
        for k, nm in enumerate(("dvn", "dkn", "dvp", "dkp")):
            params[f"{nm}{s}"] = (0.020 if nm[1] == "v" else 0.05) * decks.mc_normal(seeds, 4 * s + k)
        out = f"s{s + 1}"
        lines += [f"mn{s} {out} {prev} 0 0 nch{s} w=2u l=0.18u",
                  f"mp{s} {out} {prev} vdd vdd pch{s} w=4u",
                  f"+ l=0.18u",
                  f"c{s} {out} 0 10f",
                  f".model nch{s} nmos (level=1 vto={{0.45+dvn{s}}} kp={{2e-4*(1+dkn{s})}})",
                  f".model pch{s} pmos level=1 vto={{-0.45+dvp{s}}} kp={{8e-5*(1+dkp{s})}}"]
        prev = out
    lines.append(".end")
    net = read_deck("\n".join(lines), lanes=points, params=params)
    ref = decks.inverter_chain(points)
    # numbers read as ngspice reads them may differ from Python's literals in the last bit
    _same(net, ref, rtol=4e-16)
    assert net.sweep.shape == (points, 4 * stages)
    np.testing.assert_array_equal(net.sweep, ref.sweep)


@pytest.mark.parametrize("card,msg", [
    ("l1 a 0 1n", "element"),
    ("v1 a 0 sin(0 1 1meg)", "PULSE"),
    (".ic v(a)=1", "card"),
    ("m1 a a 0 0 nx\n.model nx nmos level=1 tox=10n", "TOX"),
    ("d1 a 0 dx\n.model dx d rs=10", "series resistance"),
    ("m1 a a 0 0 nx\n.model nx nmos level=2", "level-1"),
    ("r1 a 0 rbad", "cannot read"),
])
def test_cards_outside_the_subset_are_refused(card, msg):
    with pytest.raises(DeckError, match=msg):
        read_deck("title\nv0 a 0 1\n" + card + "\n.end\n")


def test_subcircuits_flatten_to_the_flat_deck():
    """`.subckt` definitions (nested) and `x` instances expand to the same
    netlist as the deck written out flat, internal nodes named inst.node as
    ngspice names them."""
    models = ".model nx nmos level=1 vto=0.4 kp=150u\n.model px pmos level=1 vto=-0.4 kp=60u\n"
    sub = """subckt chain
vdd vdd 0 1.8
vin a0 0 dc 0.3
.subckt inv in out sup
mn out in 0 0 nx w=1u l=0.2u
mp out in sup sup px w=2u l=0.2u
.ends
.subckt buf in out sup
x1 in mid sup inv
x2 mid out sup inv
cl mid 0 2f
.ends
xa a0 a1 vdd buf
xb a1 a2 vdd buf
r1 a2 0 10k
""" + models + ".end\n"
    flat = """flat chain
vdd vdd 0 1.8
vin a0 0 dc 0.3
""" + "".join(f"mn.{x} {o} {i} 0 0 nx w=1u l=0.2u\nmp.{x} {o} {i} vdd vdd px w=2u l=0.2u\n"
              for x, i, o in (("xa.x1", "a0", "xa.mid"), ("xa.x2", "xa.mid", "a1"),
                              ("xb.x1", "a1", "xb.mid"), ("xb.x2", "xb.mid", "a2"))) + """cl.xa xa.mid 0 2f
cl.xb xb.mid 0 2f
r1 a2 0 10k
""" + models + ".end\n"
    a, b = read_deck(sub, lanes=3), read_deck(flat, lanes=3)
    _same(a, b)
    assert a.node_names == b.node_names and "xa.mid" in a.node_names


@pytest.mark.parametrize("card,msg", [
    (".subckt s a b\nr1 a b 1k\n", "no .ends"),
    (".subckt s a b\nr1 a b 1k\n.ends\nx1 a s", "takes 2 nodes"),
    (".subckt s a b\nr1 a b 1k\n.ends\nx1 a 0 s w=1", "instance parameters"),
    (".subckt s a b params: w=1\nr1 a b 1k\n.ends", "subcircuit parameters"),
    ("x1 a 0 nosuch", "unknown subcircuit"),
    (".subckt s a b\nx1 a b s\n.ends\nx1 a 0 s", "deeper than 32"),
])
def test_subcircuit_errors(card, msg):
    with pytest.raises(DeckError, match=msg):
        read_deck("title\nv0 a 0 1\n" + card + "\n.end\n")
