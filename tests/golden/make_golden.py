"""Generates the golden fixtures under tests/golden/ from the FP64 oracle.

The reference ships no stored vectors for this path (its solver tests draw
random systems, its GPU-vs-CPU test compares two live runs), so the fixtures
pin the oracle's outputs on small cases of the benchmark decks: the column
orders and pivot tapes of the decks' patterns (integer, compared bit for
bit), operating points, and short transients with their step counts and
.meas period. tests/test_golden.py checks the oracle and the product's host
symbolic against them on CPU; tests/test_gpu_parity.py checks the GPU lanes
against them. Run from the repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def patterns():
    """Name -> netlist of the deck patterns whose order and tape are pinned."""
    from egspice_b200 import decks
    return {
        "chain16": decks.inverter_chain(2),
        "opamp": decks.miller_opamp(2),
        "ring15": decks.ring_oscillator(2, stages=15),
        "ring31": decks.ring_oscillator(2, stages=31),
        "ring63": decks.ring_oscillator(2, stages=63),
        "ladder200": decks.rc_diode_ladder(200, 2, seed=1),
        "grid12": decks.power_grid(2, side=12, loads=10),
    }


def lead_matrix(net):
    """The lead lane's A at its cold operating point: x = 0 with the MODEINITJCT
    seeds is what the first tape is built from; here the pattern's values are
    a deterministic diagonally weighted fill, enough to pin the symbolic
    analysis and the pivot decisions of a well-posed matrix."""
    cp = np.asarray(net.col_ptr, dtype=np.int64)
    ri = np.asarray(net.row_idx, dtype=np.int64)
    vals = np.empty(len(ri))
    for c in range(net.n):
        for p in range(cp[c], cp[c + 1]):
            r = ri[p]
            vals[p] = 4.0 + 0.25 * ((r * 7 + c * 3) % 5) if r == c else -0.5 - 0.125 * ((r + 2 * c) % 3)
    return vals


def op_cases():
    from egspice_b200 import abi, decks
    chain = decks.inverter_chain(4)
    opamp = decks.miller_opamp(4)
    x0 = np.zeros((opamp.lanes, opamp.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, opamp.node(k)] = v
    return [("chain16_cold", chain, abi.newton_opts(), None),
            ("opamp_warm", opamp, abi.newton_opts(init_fix=0), x0)]


def tran_cases():
    from egspice_b200 import abi, decks
    ring = decks.ring_oscillator(2, stages=15)
    topts = abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=600, predictor=1)
    ladder = decks.rc_diode_ladder(200, 2, seed=1)
    lopts = abi.tran_opts(t_stop=0.5e-9, dt=10e-12, fixed_step=1, method=1, max_iter=50)
    return [("ring15_lte", ring, topts, ("s1", 0.9, 1e-9)), ("ladder200_fixed", ladder, lopts, None)]


def main():
    from egspice_b200 import abi  # noqa: F401
    from oracle import pyoracle as po
    out = {"orders": {}, "tapes": {}, "op": {}, "tran": {}}
    for name, net in patterns().items():
        q = po.order(net.col_ptr, net.row_idx)
        out["orders"][name] = [int(v) for v in q]
        lu = po.SparseLu(net.col_ptr, net.row_idx, q)
        assert lu.factor(lead_matrix(net)) == 0
        t = lu.tape()
        out["tapes"][name] = {k: [int(v) for v in t[k]] for k in ("pinv", "lp", "li", "up", "ui", "prow")}
    for name, net, opts, x0 in op_cases():
        x, res = po.op_lanes(net, opts, x_in=x0)
        out["op"][name] = {"x": x.tolist(), "iterations": res[:, 2].tolist(), "converged": res[:, 0].tolist()}
    for name, net, topts, meas in tran_cases():
        m = (net.node(meas[0]), meas[1], meas[2]) if meas else None
        x, reps, _, per = po.tran_lanes(net, topts, meas=m)
        out["tran"][name] = {"x": x.tolist(), "steps": [int(r.steps) for r in reps],
                             "rejects": [int(r.rejects) for r in reps],
                             "period": None if per is None else [float(v) for v in per]}
    path = os.path.join(HERE, "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=None, separators=(",", ":"))
        f.write("\n")
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
