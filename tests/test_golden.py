"""The committed golden fixtures (tests/golden/golden.json, written by
tests/golden/make_golden.py from the FP64 oracle) against the oracle and the
product's host symbolic analysis, on CPU. Column orders and pivot tapes are
integer work and must match bit for bit; operating points and transients
within 1e-12 relative (the oracle is deterministic C; the slack covers a
libm that rounds an exp or log differently on another host)."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as mg  # noqa: E402


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        return json.load(f)


def test_orders_and_tapes(golden, oracle):
    po = oracle
    from egspice_b200 import symbolic
    for name, net in mg.patterns().items():
        q = po.order(net.col_ptr, net.row_idx)
        assert [int(v) for v in q] == golden["orders"][name], name
        assert [int(v) for v in symbolic.order(net.col_ptr, net.row_idx)] == golden["orders"][name], name
        vals = mg.lead_matrix(net)
        lu = po.SparseLu(net.col_ptr, net.row_idx, q)
        assert lu.factor(vals) == 0
        t = lu.tape()
        prod = symbolic.tape(net.col_ptr, net.row_idx, vals, q)
        for k, ref in golden["tapes"][name].items():
            assert [int(v) for v in t[k]] == ref, (name, k)
            assert [int(v) for v in prod[k]] == ref, (name, k, "product")


def test_operating_points(golden, oracle):
    for name, net, opts, x0 in mg.op_cases():
        x, res = oracle.op_lanes(net, opts, x_in=x0)
        g = golden["op"][name]
        assert res[:, 2].tolist() == g["iterations"], name
        np.testing.assert_allclose(x, np.array(g["x"]), rtol=1e-12, atol=1e-15)


def test_transients(golden, oracle):
    for name, net, topts, meas in mg.tran_cases():
        m = (net.node(meas[0]), meas[1], meas[2]) if meas else None
        x, reps, _, per = oracle.tran_lanes(net, topts, meas=m)
        g = golden["tran"][name]
        assert [r.steps for r in reps] == g["steps"], name
        assert [r.rejects for r in reps] == g["rejects"], name
        np.testing.assert_allclose(x, np.array(g["x"]), rtol=1e-12, atol=1e-15)
        if g["period"] is not None:
            np.testing.assert_allclose(per, np.array(g["period"]), rtol=1e-12)
