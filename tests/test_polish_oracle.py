"""The polish on the oracle (CPU): why it exists and that it does its job.
The reference's Newton publishes the iterate whose following step is inside
reltol |x| + vntol, so two start points (two predictors, a learned start)
end on different points within that tolerance; in a transient the
difference feeds the step control and moves the ring's period by ~4e-4
relative. With the polish (orc_set_polish, the product's
espl_create_opts.polish) the start no longer matters at the 1e-6 bar."""
import numpy as np

from egspice_b200 import abi, decks

RTOL, ATOL = 1e-6, 1e-9


def worst(x, xr):
    return float((np.abs(x - xr) / (RTOL * np.abs(xr) + ATOL)).max())


def _ring(oracle, digits, predictor):
    net = decks.ring_oscillator(8, stages=31)
    out = net.node("s1")
    opts = abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=1500,
                         predictor=predictor)
    with oracle.polish(digits):
        x, reps, _, per = oracle.tran_lanes(net, opts, meas=(out, 0.9, 1e-9), threads=8)
    return x, per, sum(r.nr_iters for r in reps) / sum(r.attempts for r in reps)


def test_ring_period_independent_of_the_predictor_only_when_polished(oracle):
    x1, p1, it1 = _ring(oracle, 0, 1)
    x0, p0, it0 = _ring(oracle, 0, 0)
    assert float(np.abs(p1 - p0).max() / np.abs(p1).max()) > 1e-5  # unpolished: far past the bar
    x1p, p1p, it1p = _ring(oracle, 6, 1)
    x0p, p0p, it0p = _ring(oracle, 6, 0)
    assert float((np.abs(p1p - p0p) / (RTOL * np.abs(p1p))).max()) <= 1.0
    assert worst(x0p, x1p) <= 1.0
    # the polish costs iterations, and a better start saves some of them
    assert it1p > it1 and it0p > it1p


def test_opamp_two_starts_within_the_bar_only_when_polished(oracle):
    net = decks.miller_opamp(128)
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    opts = abi.newton_opts(init_fix=0)
    with oracle.polish(6):
        xa, ra = oracle.op_lanes(net, opts, x_in=x0, threads=8)
    x1 = xa + 0.01 * np.random.default_rng(3).standard_normal(x0.shape) * (x0 != 0)
    got = {}
    for digits in (0, 6):
        with oracle.polish(digits):
            xp, rp = oracle.op_lanes(net, opts, x_in=x0, threads=8)
            xb, rb = oracle.op_lanes(net, opts, x_in=x1, threads=8)
        assert (rp[:, 0] == 1).all() and (rb[:, 0] == 1).all()
        got[digits] = worst(xb, xp)
    assert got[0] > 10.0 and got[6] <= 1e-2, got
