"""The Newton polish (espl_create_opts.polish) on the GPU against the
oracle's (orc_set_polish): once a lane's step passes the reference's test,
Newton goes on until the step also passes it with the tolerances scaled by
10^-6. The converged point is then the solution of the step's equations to
far below the Newton tolerance, so it no longer depends on where Newton
started: GPU lanes in FP64 and in mixed precision, from the linear predictor
or from none, all meet the 1e-6 bar against the polished oracle on every
lane, where without the polish two predictors move the ring's period by
~4e-4 relative."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.lanes import Lanes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-9
POLISH = 6


def worst(x, xr):
    return float((np.abs(x - xr) / (RTOL * np.abs(xr) + ATOL)).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ring_polished_independent_of_the_predictor(oracle, precision):
    """The 31-stage ring of the benchmark, 32 Monte-Carlo lanes, 1,500 LTE
    steps: the period and the final state of every lane, from the linear
    predictor and from none, against the polished oracle."""
    net = decks.ring_oscillator(32, stages=31)
    out = net.node("s1")
    opts = abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=1500, predictor=1)
    with oracle.polish(POLISH):
        xo, ro, _, po = oracle.tran_lanes(net, opts, meas=(out, 0.9, 1e-9), threads=8)
    assert np.isfinite(po).all()
    for pred in (1, 0):
        opts.predictor = pred
        with Lanes([net], precision=precision, polish=POLISH) as L:
            L.set_period_meas(0, out, 0.9, 1e-9)
            reps = L.run_tran(opts, steps_per_launch=2000)
            per, cr = L.period_meas(0)
            x = L.get_x(0)
        assert all(r.status == 1 and r.steps == 1500 for r in reps), pred
        assert float((np.abs(per - po) / (RTOL * np.abs(po))).max()) <= 1.0, (pred, per, po)
        assert worst(x, xo) <= 1.0, pred


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_opamp_polished_from_two_starts(oracle, precision):
    """Config-4's op-amp, 512 Monte-Carlo lanes: from the nominal operating
    point and from a start 10 mV (rms) off each lane's solution, the polished
    GPU lanes land on the polished oracle's points within the 1e-6 bar on
    every lane, and on each other (unpolished, the two starts differ by
    hundreds of times the bar on the oracle)."""
    net = decks.miller_opamp(512)
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    opts = abi.newton_opts(init_fix=0)
    with oracle.polish(POLISH):
        xo, ro = oracle.op_lanes(net, opts, x_in=x0, threads=8)
    assert (ro[:, 0] == 1).all()
    x1 = xo + 0.01 * np.random.default_rng(3).standard_normal(x0.shape) * (x0 != 0)
    xs = []
    for start in (x0, x1):
        with Lanes([net], precision=precision, polish=POLISH) as L:
            L.put_x(0, start, False)
            r = L.solve_static(opts)
            xs.append(L.get_x(0))
        assert ((r[:, 0] & abi.CONVERGED) != 0).all()
        assert worst(xs[-1], xo) <= 1.0
    assert worst(xs[1], xs[0]) <= 1.0


def test_ladder_polished_meets_the_bar(oracle):
    """espl_solve_op from the cold start on 256 op-amp lanes with the polish:
    every lane converges onto the polished oracle ladder's point within the
    1e-6 bar (unpolished, two ladders that step differently agree only to the
    Newton tolerance)."""
    net = decks.miller_opamp(256)
    opts = abi.newton_opts()
    with oracle.polish(POLISH):
        xo, ro = oracle.op_ladder(net, opts, threads=8)
    with Lanes([net], polish=POLISH) as L:
        r = L.solve_op(opts)
        x = L.get_x(0)
    assert (ro[:, 0] == 1).all()
    assert ((r[:, 0] & abi.CONVERGED) != 0).all()
    assert worst(x, xo) <= 1.0
