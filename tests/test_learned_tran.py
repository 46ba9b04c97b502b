"""The transient's learned next-step predictor on the GPU (include/espice_learned.h).

The recorder's samples against the oracle's own trajectory; the predictor
kernel (tcgen05, lane-interleaved histories) against the network's row-major
inference on features built here from the same histories; and the whole
learned transient (linear warm-up with the recorder, training on the
device, learned starts) against the polished FP64 oracle on every lane, in
fewer Newton iterations than the linear predictor. Tolerance of the results:
|x - x_ref| <= 1e-6 |x_ref| + 1e-9 and the period within 1e-6 relative."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.lanes import Lanes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-9
POLISH = 6


def ring_opts(steps):
    return abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=steps, predictor=2)


def features(cur, prev, prev2, steps, dt_max):
    """The predictor's inputs (espice_learned.h): cur, (dt/h0)(cur - prev),
    (dt/h1)(prev - prev2), dt/dt_max."""
    dt, h0, h1 = steps[:, 0:1], steps[:, 1:2], steps[:, 2:3]
    return np.concatenate([cur, (dt / h0) * (cur - prev), (dt / h1) * (prev - prev2), dt / dt_max], axis=1)


def test_recorder_samples_follow_the_oracle_trajectory(oracle):
    """FP64 lanes record (features, target) of their accepted steps; the
    oracle's rows of the same lanes give the same samples."""
    net = decks.ring_oscillator(64, stages=31)
    n = net.n
    opts = ring_opts(120)
    with Lanes([net], polish=POLISH) as L:
        L.record_steps(0, 16, 0, 4096)
        L.init_steps(opts)
        reps = L.device_launch(100000)
        x, y, tags = L.recorded_host(0)
    assert all(r.status == 1 and r.steps == 120 for r in reps)
    lanes = sorted(set(tags[:, 0].astype(int)))
    assert lanes == [0, 16, 32, 48]
    assert len(tags) == 4 * (120 - 3)
    with oracle.polish(POLISH):
        _, _, rows, _ = oracle.tran_lanes(net, opts, lane0=0, count=49, probes=list(range(n)), max_rows=120,
                                          threads=8)
    worst = 0.0
    for k in range(len(tags)):
        l, s, dt, h0, h1 = int(tags[k, 0]), int(tags[k, 1]), tags[k, 2], tags[k, 3], tags[k, 4]
        cur, prev, prev2, nxt = rows[l, s - 1], rows[l, s - 2], rows[l, s - 3], rows[l, s]
        f = features(cur[None], prev[None], prev2[None], np.array([[dt, h0, h1]]), opts.dt_max)[0]
        t = nxt - (cur + (dt / h0) * (cur - prev))
        scale = 1e-6 * np.maximum(np.abs(np.concatenate([f, t])), 1.0)
        worst = max(worst, float((np.abs(np.concatenate([x[k] - f, y[k] - t])) / scale).max()))
    assert worst <= 1.0, worst


def test_predictor_kernel_matches_the_network():
    """k_step_predict (features from the lane-interleaved histories, the
    network on the tensor cores, the start written back lane-interleaved)
    against espl_mlp_predict on features built here: the same BF16 inputs
    and MMAs, so the starts agree to rounding."""
    from egspice_b200.learned import Mlp, step_predictor_dims, train_opts
    net = decks.ring_oscillator(256, stages=31)
    n = net.n
    opts = ring_opts(300)
    with Lanes([net], precision="mixed", polish=POLISH) as L:
        L.record_steps(0, 4, 0, 65536)
        L.init_steps(opts)
        L.device_launch(300 - 40)
        xp, yp, count = L.recorded(0)
        assert count > 10000
        _, ys, _ = L.recorded_host(0)
        d_in, d_out = step_predictor_dims(n)
        with Mlp(d_in, d_out, capacity=4096, seed=3) as m:
            losses = m.train_device(xp, yp, count, train_opts(epochs=6, batch=2048, lr=3e-3, lr_final=1e-3))
            assert np.isfinite(losses).all() and losses[-1] < losses[0]
            L.set_step_predictor(0, m)
            out = L.step_predict(0)
            live = np.isfinite(out["x_start"]).all(axis=1)
            assert live.sum() >= 200
            f = features(out["cur"], out["prev"], out["prev2"], out["steps"], opts.dt_max)[live]
            y = m.predict(f)
    cur, prev, st = out["cur"][live], out["prev"][live], out["steps"][live]
    xlin = cur + (st[:, 0:1] / st[:, 1:2]) * (cur - prev)
    got = out["x_start"][live]
    # unknowns whose target never varied (the ground, the supply node) start
    # at x_lin plus that constant, exactly; the network's output for them is
    # not used (espl_mlp_predict, which de-standardizes every output, would
    # add it)
    const = ys.std(axis=0) == 0.0
    assert const[0] and const.sum() < n // 2
    assert np.array_equal(got[:, const], xlin[:, const] + ys[0, const])
    want = xlin + y
    err = np.abs(got[:, ~const] - want[:, ~const]) / (1.0 + np.abs(want[:, ~const]))
    assert float(err.max()) <= 1e-9, float(err.max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_learned_transient_meets_the_bar_in_fewer_iterations(oracle, precision):
    """256 ring lanes, 1,500 LTE steps, polished to 10^-6 of the Newton
    tolerances: 400 steps with the linear
    predictor and the recorder, the network trained on the device, the rest
    from learned starts (an attempt at a time, a CUDA graph per attempt).
    Every lane's period and final state meet the bar against the polished
    oracle; the learned part takes fewer Newton iterations per attempt than
    the same lanes with the linear predictor; the accepted steps are the
    same."""
    from egspice_b200.learned import learned_transient, train_opts
    net = decks.ring_oscillator(256, stages=31)
    out = net.node("s1")
    steps = 1500
    opts = ring_opts(steps)
    opts.predictor = 1
    with oracle.polish(POLISH):
        xo, ro, _, po = oracle.tran_lanes(net, opts, meas=(out, 0.9, 1e-9), threads=8)
    assert np.isfinite(po).all()

    def run(learned):
        with Lanes([net], precision=precision, polish=POLISH) as L:
            L.set_period_meas(0, out, 0.9, 1e-9)
            if learned:
                reps, m, info = learned_transient(L, ring_opts(steps), warm_steps=400, lane_stride=2,
                                                  opts=train_opts(epochs=30, batch=4096, lr=3e-3, lr_final=3e-4))
                m.close()
                warm = info["warm_reports"]
            else:
                o = ring_opts(steps)
                o.predictor = 1
                L.init_steps(o)
                warm = L.device_launch(400)
                reps = L.device_launch(100000)
                info = None
            per, _ = L.period_meas(0)
            return reps, warm, L.get_x(0), per, info

    reps_p, warm_p, x_p, per_p, _ = run(False)
    reps_l, warm_l, x_l, per_l, info = run(True)
    for reps in (reps_p, reps_l):
        assert all(r.status == 1 and r.steps == steps for r in reps)
    for x, per in ((x_p, per_p), (x_l, per_l)):
        assert float((np.abs(per - po) / (RTOL * np.abs(po))).max()) <= 1.0
        assert float((np.abs(x - xo) / (RTOL * np.abs(xo) + ATOL)).max()) <= 1.0

    def tail(reps, warm):
        it = sum(r.nr_iters - w.nr_iters for r, w in zip(reps, warm))
        at = sum(r.attempts - w.attempts for r, w in zip(reps, warm))
        return it / at

    ipa_p, ipa_l = tail(reps_p, warm_p), tail(reps_l, warm_l)
    retries = sum(r.learned_retries for r in reps_l)
    same_rejects = float(np.mean([a.rejects == b.rejects for a, b in zip(reps_p, reps_l)]))
    print(f"{precision}: Newton iterations per attempt after the warm-up: linear {ipa_p:.3f}, learned {ipa_l:.3f}; "
          f"learned retries {retries}; lanes with the plain run's rejects {same_rejects:.3f}; "
          f"{ {k: v for k, v in info.items() if k != 'warm_reports'} }")
    assert ipa_l <= 0.92 * ipa_p, (ipa_p, ipa_l)
    assert same_rejects >= 0.9
