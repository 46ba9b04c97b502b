"""The operating-point continuation ladder of the oracle (op.zig solveLadder
/ afterPlain restated in oracle/circuit.c) on CPU: from the cold start the
plain rung leaves most op-amp lanes unconverged; the ladder (gmin stepping,
source stepping, the final solve) converges every one, onto the fixed point
a warm start near the nominal operating point finds. The GPU ladder
(espl_solve_op) is checked against it in tests/test_gpu_parity.py."""
import numpy as np

from egspice_b200 import abi, decks


def _nominal(net):
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    return x0


def test_ladder_converges_cold_opamp_lanes(oracle):
    net = decks.miller_opamp(64)
    opts = abi.newton_opts()
    _, plain = oracle.op_lanes(net, opts, threads=8)
    x, res = oracle.op_ladder(net, opts, threads=8)
    assert plain[:, 0].sum() < 16, "the plain rung alone converges few cold op-amp lanes"
    assert (res[:, 0] == 1).all()
    assert (res[:, 2] >= plain[:, 2]).all()  # iterations count every rung
    xw, rw = oracle.op_lanes(net, abi.newton_opts(init_fix=0), x_in=_nominal(net), threads=8)
    assert (rw[:, 0] == 1).all()
    cur = np.asarray(net.current_rows, dtype=bool)
    tol = opts.reltol * np.maximum(np.abs(x), np.abs(xw)) + np.where(cur, opts.abstol, opts.vntol)
    assert float((np.abs(x - xw) / tol).max()) <= 2.0


def test_ladder_keeps_plain_lanes(oracle):
    """Lanes the plain rung converges keep its answer and count."""
    net = decks.inverter_chain(64)
    opts = abi.newton_opts()
    xp, rp = oracle.op_lanes(net, opts, threads=8)
    x, res = oracle.op_ladder(net, opts, threads=8)
    ok = rp[:, 0] == 1
    assert (res[:, 0] == 1).all()
    assert np.array_equal(x[ok], xp[ok]) and np.array_equal(res[ok, 2], rp[ok, 2])
