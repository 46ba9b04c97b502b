"""GPU lanes through the C ABI against the CPU FP64 oracle on the same
seeded decks. Tolerance: |x - x_ref| <= 1e-6 |x_ref| + 1e-9 (V or A), the
bar of the reference's GPU-vs-CPU lane test (src/tests/espice.zig:3387)."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.lanes import Lanes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-9


def worst(x, xr):
    return float((np.abs(x - xr) / (RTOL * np.abs(xr) + ATOL)).max())


def opamp_start(net):
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    return x0


def test_tape_bit_exact_with_oracle(oracle):
    net = decks.inverter_chain(32)
    with Lanes([net]) as L:
        t = L.tape(0)
    q = oracle.order(net.col_ptr, net.row_idx)
    assert np.array_equal(t["q"], q)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_inverter_chain_cold_operating_points(oracle, precision):
    """Config 1 at its size: 1,024 Monte-Carlo points of the 16-stage chain
    from the cold start.

    The plain rung alone (solve_static from x = 0 with INITFIX): where both
    sides converge, every lane meets the bar. From a cold start the limiting
    walk amplifies last-bit differences (a fused multiply-add, the last bit
    of exp), so a lane near the 100-iteration limit can converge on one side
    and not the other; at most 2 % of lanes may differ that way (1.2 % on a
    B200).

    The whole operating point (solve_op: the plain rung, then the
    continuation ladder for the lanes it leaves) with the polish, against
    the oracle's ladder with the same polish: every lane converges on both
    sides and every lane meets the bar."""
    net = decks.inverter_chain(1024)
    opts = abi.newton_opts()
    xo, ro = oracle.op_lanes(net, opts, threads=8)
    with Lanes([net], precision=precision) as L:
        r = L.solve_static(opts)
        x = L.get_x(0)
    ok = (r[:, 0] & abi.CONVERGED) != 0
    oracle_ok = ro[:, 0] == 1
    assert oracle_ok.mean() >= 0.99
    both = ok & oracle_ok
    assert (ok != oracle_ok).mean() <= 0.02, np.nonzero(ok != oracle_ok)[0].tolist()
    assert worst(x[both], xo[both]) <= 1.0
    with oracle.polish(6):
        xl, rl = oracle.op_ladder(net, opts, threads=8)
    with Lanes([net], precision=precision, polish=6) as L:
        r = L.solve_op(opts)
        x = L.get_x(0)
    assert (rl[:, 0] == 1).all()
    assert ((r[:, 0] & abi.CONVERGED) != 0).all()
    assert worst(x, xl) <= 1.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_opamp_warm_operating_points(oracle, precision):
    net = decks.miller_opamp(512)
    x0 = opamp_start(net)
    opts = abi.newton_opts(init_fix=0)
    xo, ro = oracle.op_lanes(net, opts, x_in=x0, threads=8)
    with Lanes([net], precision=precision) as L:
        L.put_x(0, x0, False)
        r = L.solve_static(opts)
        x = L.get_x(0)
    assert ((r[:, 0] & abi.CONVERGED) != 0).all()
    assert worst(x, xo) <= 1.0
    if precision == "fp64":
        assert np.array_equal(r[:, 1], ro[:, 2])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uneven_ladders_one_launch(oracle, precision):
    nets = [decks.rc_diode_ladder(n, 40, seed=s) for n, s in ((200, 1), (517, 2), (1203, 3))]
    topts = abi.tran_opts(t_stop=2e-9, dt=10e-12, fixed_step=1, method=1, max_iter=50)
    with Lanes(nets, precision=precision, dt0=10e-12) as L:
        reps = L.run_tran(topts, steps_per_launch=64)
        xs = [L.get_x(i) for i in range(len(nets))]
    assert all(r.status == 1 and r.steps == 200 for r in reps)
    for nl, x in zip(nets, xs):
        xo, ro, _, _ = oracle.tran_lanes(nl, topts, threads=8)
        assert worst(x, xo) <= 1.0, nl.name


@pytest.mark.parametrize("method", [1, 2])
def test_rc_points_lte_control(oracle, method):
    """Trapezoidal (1) and gear-2 (2) steps under LTE control: the same
    accepted and rejected steps as the oracle, lane by lane."""
    r = np.array([1e3, 2e3, 5e3, 1e4])
    c = np.array([1e-12, 0.5e-12, 2e-13, 2e-13])
    net = decks.rc_points(4, r, c, tr=0.2e-9)
    opts = abi.tran_opts(t_stop=8e-9, dt=1e-12, dt_max=20e-12, method=method, max_iter=20, reltol=1e-4)
    with Lanes([net]) as L:
        reps = L.run_tran(opts, steps_per_launch=4096)
        x = L.get_x(0)
    xo, ro, _, _ = oracle.tran_lanes(net, opts)
    for a, b in zip(reps, ro):
        assert a.status == 1 and a.steps == b.steps and a.rejects == b.rejects
    assert worst(x, xo) <= 1.0


def test_step_report_events():
    """The step report's per-attempt fields (StepReport, kernels/lane.zig
    :441-451) on a 15-stage ring: one attempt per launch, so each report
    shows that attempt --
    event 2 (accepted: t is t_new) or 3 (rejected: t is unchanged, the next
    dt smaller than the attempted one) -- and a finished lane reads idle
    (0), its last attempt's t_new its final time."""
    net = decks.ring_oscillator(4, stages=15)
    opts = abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=400)
    seen = set()
    with Lanes([net]) as L:
        L.init_steps(opts)
        prev = [0.0] * 4
        for _ in range(4000):
            reps = L.device_launch(1)
            for k, rp in enumerate(reps):
                if rp.status != 0:
                    continue
                seen.add(rp.event)
                assert rp.event in (2, 3)
                assert rp.attempted_dt > 0 and rp.t_new == prev[k] + rp.attempted_dt
                if rp.event == 2:
                    assert rp.t == rp.t_new
                else:
                    assert rp.t == prev[k] and rp.dt < rp.attempted_dt
                prev[k] = rp.t
            if all(rp.status != 0 for rp in reps):
                break
    assert seen == {2, 3}  # the ring's LTE control rejects some steps
    for rp in reps:
        assert rp.status == 1 and rp.steps == 400 and rp.event == 0 and rp.t_new == rp.t


@pytest.mark.parametrize("method", [1, 2])
def test_ring_oscillator_period(oracle, method):
    net = decks.ring_oscillator(16, stages=15)
    out = net.node("s3")
    opts = abi.tran_opts(t_stop=3e-9, dt=1e-12, dt_max=5e-12, method=method, max_iter=20)
    with Lanes([net]) as L:
        L.set_period_meas(0, out, 0.9, 0.5e-9)
        reps = L.run_tran(opts, steps_per_launch=2048)
        per, cr = L.period_meas(0)
    _, ro, _, po = oracle.tran_lanes(net, opts, meas=(out, 0.9, 0.5e-9), threads=8)
    assert all(r.status == 1 for r in reps)
    assert np.all(cr >= 3)
    assert np.all(np.abs(per - po) <= 1e-6 * np.abs(po)), (per, po)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_golden_fixtures_on_the_gpu(precision):
    """The committed oracle fixtures (tests/golden), without the oracle: FP64
    lanes reproduce them to 1e-12 with the same iteration and step counts;
    mixed lanes meet the 1e-6 bar."""
    import json
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_golden as mg
    with open(os.path.join(here, "golden", "golden.json")) as f:
        g = json.load(f)
    tight = precision == "fp64"
    for name, net, opts, x0 in mg.op_cases():
        with Lanes([net], precision=precision) as L:
            if x0 is not None:
                L.put_x(0, x0, False)
            r = L.solve_static(opts)
            x = L.get_x(0)
        xr = np.array(g["op"][name]["x"])
        assert ((r[:, 0] & abi.CONVERGED) != 0).all(), name
        assert worst(x, xr) <= 1.0, name
        if tight and opts.init_fix == 0:
            # a warm start takes the oracle's path: the same iterations and x
            # to rounding (a cold start's limiting walk may take other
            # iterations: the device fuses multiply-adds the oracle rounds
            # twice, and the walk amplifies that)
            assert r[:, 1].tolist() == g["op"][name]["iterations"], name
            np.testing.assert_allclose(x, xr, rtol=1e-12, atol=1e-15)
    for name, net, topts, meas in mg.tran_cases():
        with Lanes([net], precision=precision, dt0=topts.dt) as L:
            if meas:
                L.set_period_meas(0, net.node(meas[0]), meas[1], meas[2])
            reps = L.run_tran(topts, steps_per_launch=10000)
            x = L.get_x(0)
            per = L.period_meas(0)[0] if meas else None
        gt = g["tran"][name]
        xr = np.array(gt["x"])
        if tight:
            assert [rp.steps for rp in reps] == gt["steps"], name
            assert [rp.rejects for rp in reps] == gt["rejects"], name
            np.testing.assert_allclose(x, xr, rtol=1e-12, atol=1e-15)
            if per is not None:
                np.testing.assert_allclose(per, np.array(gt["period"]), rtol=1e-12)
        else:
            assert worst(x, xr) <= 1.0, name
            if per is not None:
                assert float(np.abs(per - np.array(gt["period"])).max()) <= 1e-6 * float(np.abs(gt["period"]).max())


@pytest.mark.parametrize("precision,refine", [("fp64", 0), ("mixed", 0), ("mixed", 1)])
def test_power_grid_transient(oracle, precision, refine):
    """Config-3 shape at a test size: a 16 x 16 resistive mesh with decaps,
    corner pads and current-pulse loads, trapezoidal fixed steps; in mixed
    mode with and without the FP64-residual refinement sweep."""
    net = decks.power_grid(6, side=16, loads=24)
    topts = abi.tran_opts(t_stop=1e-9, dt=10e-12, fixed_step=1, method=1, max_iter=20)
    with Lanes([net], precision=precision, dt0=topts.dt, refine_sweeps=refine) as L:
        reps = L.run_tran(topts, steps_per_launch=4096)
        x = L.get_x(0)
    assert all(r.status == 1 and r.steps == 100 for r in reps)
    xo, _, _, _ = oracle.tran_lanes(net, topts, threads=6)
    assert worst(x, xo) <= 1.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_power_grid_full_size(oracle, precision):
    """Config 3 at its size: 256 lanes of the 200 x 200 mesh (40,005
    unknowns, 2.1 million factor entries per lane), trapezoidal fixed steps
    (20 here) through the large-template LU (the whole tile refactors by
    columns and solves by levels, lane_levels.cuh); four lanes against the
    oracle."""
    net = decks.power_grid(256, side=200, loads=400)
    topts = abi.tran_opts(t_stop=20 * 10e-12, dt=10e-12, fixed_step=1, method=1, max_iter=20)
    with Lanes([net], precision=precision, dt0=topts.dt) as L:
        cl = L.classes()
        reps = L.run_tran(topts, steps_per_launch=4096)
        x = L.get_x(0)
    assert all(r.status == 1 and r.steps == 20 for r in reps)
    assert all(r.nr_iters == 40 for r in reps)  # a linear circuit: two Newton iterations per step
    assert len(cl) == 1 and cl[0]["wide"] and cl[0]["tiles"] == 256 // 2  # 2-lane parts, one CTA each
    pick = [0, 85, 170, 255]
    for l in pick:
        xo, _, _, _ = oracle.tran_lanes(net, topts, lane0=l, count=1, threads=1)
        assert worst(x[l:l + 1], xo) <= 1.0, l


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_inverter_pair_width_step(oracle, precision):
    """The reference's GPU-vs-CPU lane deck shape (src/tests/espice.zig:
    3353-3389): two inverters with a .step over the NMOS width, cold
    operating points, every lane within the 1e-6 bar of the CPU run."""
    net = decks.inverter_pair(64)
    opts = abi.newton_opts()
    xo, ro = oracle.op_lanes(net, opts, threads=8)
    with Lanes([net], precision=precision) as L:
        r = L.solve_static(opts)
        x = L.get_x(0)
    assert ((r[:, 0] & abi.CONVERGED) != 0).all() and (ro[:, 0] == 1).all()
    assert worst(x, xo) <= 1.0


def test_backward_euler_lte_steps(oracle):
    """Backward Euler under LTE control: the same accepted and rejected
    steps as the oracle."""
    r = np.array([1e3, 5e3, 2e4])
    c = np.array([1e-12, 2e-13, 5e-14])
    net = decks.rc_points(3, r, c, tr=0.1e-9)
    opts = abi.tran_opts(t_stop=5e-9, dt=1e-12, dt_max=20e-12, method=0, max_iter=20, reltol=1e-4)
    with Lanes([net]) as L:
        reps = L.run_tran(opts, steps_per_launch=4096)
        x = L.get_x(0)
    xo, ro, _, _ = oracle.tran_lanes(net, opts)
    for a, b in zip(reps, ro):
        assert a.status == 1 and a.steps == b.steps and a.rejects == b.rejects
    assert worst(x, xo) <= 1.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deck_text_dc_sweep(oracle, precision):
    """A deck read from SPICE text (egspice_b200/netlist.py) drives the
    lanes: a 4-stage inverter chain whose input sweeps 0 .. 1.8 V across 64
    lanes, cold operating points against the oracle on the same netlist."""
    from egspice_b200.netlist import read_deck
    text = """inverter chain, input swept per lane
vdd vdd 0 dc 1.8
vin s0 0 dc {vin}
.model nch nmos level=1 vto=0.45 kp=200u lambda=0.02
.model pch pmos level=1 vto=-0.45 kp=80u lambda=0.02
""" + "".join(f"mn{k} s{k + 1} s{k} 0 0 nch w=2u l=0.18u\nmp{k} s{k + 1} s{k} vdd vdd pch w=4u l=0.18u\n"
              for k in range(4)) + ".op\n.end\n"
    net = read_deck(text, lanes=64, params={"vin": np.linspace(0.0, 1.8, 64)})
    opts = abi.newton_opts()
    xo, ro = oracle.op_lanes(net, opts, threads=8)
    with Lanes([net], precision=precision) as L:
        r = L.solve_static(opts)
        x = L.get_x(0)
    ok = (r[:, 0] & abi.CONVERGED) != 0
    assert (ok | (ro[:, 0] != 1)).all()
    assert ok.mean() >= 0.95
    both = ok & (ro[:, 0] == 1)
    assert worst(x[both], xo[both]) <= 1.0
    out = x[:, net.node("s4")]
    assert out[0] < 0.1 and out[-1] > 1.7  # four inversions: the output follows the input to its rail


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deck_measures(oracle, precision):
    """`.meas tran` cards of a deck (egspice_b200/netlist.py read_measures)
    on the lanes against the oracle: 64 RC lanes with per-lane R, every kind
    of card the lanes take, a source current among the vectors."""
    from egspice_b200.netlist import measure_passes, measure_values, read_deck, read_measures
    text = """RC step response with measures
vin in 0 dc 0 pulse(0 1 0 0.2n 0.2n 1 2)
r1 in out rval
c1 out 0 1p
.meas tran t50 when v(out)=0.5
.meas tran rise trig v(out) val=0.1 rise=1 targ v(out) val=0.9 rise=1
.meas tran v2n find v(out) at=2n
.meas tran slope2n deriv v(out) at=2n
.meas tran iin find i(vin) at=2n
.meas tran early find v(out) when v(in)=0.5
.meas tran swing pp v(out)
.meas tran avg avg v(out) from=1n to=5n
.meas tran rms rms v(out) from=1n
.meas tran area integ v(in) to=5n
.end
"""
    params = {"rval": np.random.default_rng(5).uniform(0.5e3, 1.5e3, 64)}
    net = read_deck(text, lanes=64, params=params)
    ms = read_measures(text, net, params=params)
    opts = abi.tran_opts(t_stop=6e-9, dt=1e-12, dt_max=5e-12, method=1, max_iter=20)
    vo, _, _, ro = oracle.tran_meas(net, opts, measure_passes(ms), threads=8)
    with Lanes([net], precision=precision) as L:
        L.set_meas(0, measure_passes(ms))
        reps = L.run_tran(opts, steps_per_launch=2048)
        v, _ = L.get_meas(0)
    assert all(r.status == 1 for r in reps)
    got, want = measure_values(ms, v), measure_values(ms, vo)
    # the 1e-6 bar; voltages with its 1e-9 V floor, amperes 1e-12 A, times
    # and the integral relative only; a slope over one step: its samples'
    # floor over the step (V/s)
    atol = {"v2n": 1e-9, "early": 1e-9, "swing": 1e-9, "avg": 1e-9, "rms": 1e-9, "iin": 1e-12, "slope2n": 1e3}
    for name in want:
        assert np.isfinite(want[name]).all(), name
        np.testing.assert_allclose(got[name], want[name], rtol=1e-5 if name == "slope2n" else 1e-6,
                                   atol=atol.get(name, 0.0), err_msg=name)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_streaming_meas_passes(oracle, precision):
    """The device .meas passes (include/espice_lanes.h espl_set_meas) on the
    ring oscillator against the oracle's (oracle/measure.c) over the same
    transient: WHEN with a count and a delay, MAX, MIN, AVG and RMS over a
    window, INTEG, FIND ... AT."""
    net = decks.ring_oscillator(16, stages=15)
    s1, s3, s5 = net.node("s1"), net.node("s3"), net.node("s5")
    M = abi.meas_pass
    passes = [M(abi.MEAS_WHEN, s3, val=0.9, td=0.5e-9, rise=2), M(abi.MEAS_WHEN, s1, val=0.9, cross=abi.MEAS_LAST),
              M(abi.MEAS_MAX, s3), M(abi.MEAS_MIN, s3, from_=1e-9), M(abi.MEAS_AVG, s3, from_=1e-9, to=2.5e-9),
              M(abi.MEAS_INTEG, s1), M(abi.MEAS_RMS, s1, from_=1e-9), M(abi.MEAS_FIND_AT, s5, at=2.2e-9)]
    opts = abi.tran_opts(t_stop=3e-9, dt=1e-12, dt_max=5e-12, method=1, max_iter=20)
    vo, ao, _, ro = oracle.tran_meas(net, opts, passes, threads=8)
    with Lanes([net], precision=precision) as L:
        L.set_meas(0, passes)
        reps = L.run_tran(opts, steps_per_launch=2048)
        v, a = L.get_meas(0)
    assert all(r.status == 1 for r in reps)
    assert np.isfinite(vo).all() and np.isfinite(v).all()
    # the 1e-6 bar; voltages with the bar's 1e-9 V floor, times and the
    # integral (V s) relative only
    for k in range(len(passes)):
        atol = 1e-9 if k in (2, 3, 4, 6, 7) else 0.0
        np.testing.assert_allclose(v[:, k], vo[:, k], rtol=1e-6, atol=atol, err_msg=f"pass {k}")
    # where an extremum was taken is not pinned: the rails are flat, and the
    # last of several samples within an ulp of the extremum is the one kept
    assert ((a[:, 2:4] >= 0) & (a[:, 2:4] <= opts.t_stop)).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chained_meas_passes(oracle, precision):
    """The passes that read another vector or the pass before them, on the
    ring oscillator against the oracle: FIND and DERIV at a WHEN event,
    DERIV at a time, WHEN one node crosses another, and a TRIG/TARG pair
    whose TARG counts from the TRIG event."""
    net = decks.ring_oscillator(16, stages=15)
    s1, s3, s4 = net.node("s1"), net.node("s3"), net.node("s4")
    M = abi.meas_pass
    passes = [M(abi.MEAS_WHEN, s3, val=0.9, td=0.5e-9, rise=2),   # 0: the event
              M(abi.MEAS_FIND_WHEN, s4),                           # 1: s4 (falling) there
              M(abi.MEAS_WHEN, s3, val=0.9, td=0.5e-9, rise=2),
              M(abi.MEAS_DERIV_WHEN, s4),                          # 3: its slope there
              M(abi.MEAS_DERIV_AT, s3, at=2.2e-9),                 # 4
              M(abi.MEAS_WHEN, s1, level_row=s3, cross=2),         # 5: s1 = s3
              M(abi.MEAS_WHEN, s1, val=0.9, rise=1),               # 6: TRIG
              M(abi.MEAS_TARG, s3, val=0.9, fall=1)]               # 7: TARG
    opts = abi.tran_opts(t_stop=3e-9, dt=1e-12, dt_max=5e-12, method=1, max_iter=20)
    vo, ao, _, ro = oracle.tran_meas(net, opts, passes, threads=8)
    with Lanes([net], precision=precision) as L:
        L.set_meas(0, passes)
        reps = L.run_tran(opts, steps_per_launch=2048)
        v, a = L.get_meas(0)
    assert all(r.status == 1 for r in reps)
    assert np.isfinite(vo).all() and np.isfinite(v).all()
    for k in (0, 5, 6):  # event times
        np.testing.assert_allclose(v[:, k], vo[:, k], rtol=1e-6, err_msg=f"pass {k}")
    np.testing.assert_allclose(a[:, 7], ao[:, 7], rtol=1e-6)  # the TARG time
    np.testing.assert_allclose(v[:, 7], vo[:, 7], rtol=0, atol=2e-6 * opts.t_stop)
    np.testing.assert_array_equal(a[:, 1], v[:, 0])  # FIND reads at the WHEN's event
    # a value at an event moves with the event: slope x time difference
    slope_tol = np.abs(vo[:, 3]) * 2 * np.abs(v[:, 0] - vo[:, 0])
    assert (np.abs(v[:, 1] - vo[:, 1]) <= 1e-6 * np.abs(vo[:, 1]) + 1e-9 + slope_tol).all()
    # slopes of one step: a sample's error over the step (V/s)
    for k in (3, 4):
        np.testing.assert_allclose(v[:, k], vo[:, k], rtol=1e-3, atol=1e6, err_msg=f"pass {k}")
    assert (np.abs(vo[:, 3]) > 1e9).all() and (np.abs(vo[:, 4]) > 1e8).any()  # the slopes are not flat


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_operating_point_ladder(oracle, precision):
    """espl_solve_op from the cold start: the op-amp lanes the plain rung
    leaves unconverged walk the continuation ladder on the device and all
    converge, onto the oracle ladder's fixed point within the Newton
    tolerance (each lane's ladder may step differently once a Newton count
    differs by one); lanes the plain rung converges keep the plain answer."""
    net = decks.miller_opamp(256)
    opts = abi.newton_opts()
    xo, ro = oracle.op_ladder(net, opts, threads=8)
    with Lanes([net], precision=precision) as L:
        r = L.solve_op(opts)
        x = L.get_x(0)
    assert (ro[:, 0] == 1).all()
    assert ((r[:, 0] & abi.CONVERGED) != 0).all(), int(((r[:, 0] & abi.CONVERGED) != 0).sum())
    cur = np.asarray(net.current_rows, dtype=bool)
    tol = opts.reltol * np.maximum(np.abs(x), np.abs(xo)) + np.where(cur, opts.abstol, opts.vntol)
    assert float((np.abs(x - xo) / tol).max()) <= 2.0
    same = float((r[:, 1] == ro[:, 2]).mean())
    print(f"lanes with the oracle's ladder iteration count: {same:.2f}")
    if precision == "fp64":
        assert same >= 0.5


def test_ac_lanes(oracle):
    """espl_ac: an RC low pass against its analytic response, and the op-amp
    (64 Monte Carlo lanes at their warm operating points) from its input
    source to its output over a frequency sweep, against the oracle's dense
    complex solve at the same operating points."""
    r, c = np.array([1e3, 2e3, 5e3]), np.array([1e-12, 1e-12, 2e-13])
    rc = decks.rc_points(3, r, c)
    om = np.logspace(5, 11, 13)
    with Lanes([rc]) as L:
        L.solve_static(abi.newton_opts())
        h = L.ac(0, 0, om, [rc.node("out")])
    np.testing.assert_allclose(h[:, :, 0], 1.0 / (1.0 + 1j * om[None, :] * (r * c)[:, None]), rtol=1e-12)
    net = decks.miller_opamp(64)
    om = np.logspace(2, 10, 17)
    out = net.node("out")
    with Lanes([net]) as L:
        L.put_x(0, opamp_start(net), False)
        res = L.solve_static(abi.newton_opts(init_fix=0))
        x = L.get_x(0)
        h = L.ac(0, 1, om, [out])
    assert ((res[:, 0] & abi.CONVERGED) != 0).all()
    ho = oracle.ac_lanes(net, x, 1, om, [out])
    assert np.isfinite(h).all()
    np.testing.assert_allclose(h, ho, rtol=1e-8, atol=1e-12 * np.abs(ho).max())


def test_ac_solve_lists_and_adjoints(oracle):
    """espl_ac_solve on the op-amp's 64 lanes at their warm operating
    points: two right-hand sides (the output node, the input source's branch
    row), forward and adjoint (transpose) solves against the oracle's dense
    solves; espl_ac is the forward solve of the branch row, and the two
    modes agree by reciprocity (z[branch] of the adjoint of e_out is x[out]
    of the forward of e_branch)."""
    net = decks.miller_opamp(64)
    om = np.logspace(2, 10, 9)
    out = net.node("out")
    branch = int([b for b in net.batches if b.kind == decks.VSRC][0].term[1, 2])
    n = net.n
    rhs = np.zeros((2, n), dtype=complex)
    rhs[0, out] = 1.0
    rhs[1, branch] = 1.0
    rows = np.arange(n)
    with Lanes([net]) as L:
        L.put_x(0, opamp_start(net), False)
        res = L.solve_static(abi.newton_opts(init_fix=0))
        x = L.get_x(0)
        fwd = L.ac_solve(0, om, rhs, rows)
        adj = L.ac_solve(0, om, rhs, rows, adjoint=True)
        h = L.ac(0, 1, om, rows)
    assert ((res[:, 0] & abi.CONVERGED) != 0).all()
    assert np.isfinite(fwd).all() and np.isfinite(adj).all()
    np.testing.assert_array_equal(h, fwd[:, :, 1])
    for got, adjoint in ((fwd, False), (adj, True)):
        want = oracle.ac_solve_lanes(net, x, om, rhs, rows, adjoint=adjoint)
        scale = np.abs(want).max(axis=3, keepdims=True)
        assert (np.abs(got - want) <= 1e-8 * np.abs(want) + 1e-12 * scale).all(), adjoint
    np.testing.assert_allclose(adj[:, :, 0, branch], fwd[:, :, 1, out], rtol=1e-9)


def test_noise_lanes(oracle):
    """espl_noise_sources and the adjoint solves: an RC low pass against its
    analytic output noise 4kTR / (1 + (wRC)^2), and the op-amp's 64 lanes at
    their warm operating points (MOS channel noise) against the oracle's
    densities and dense adjoint solves."""
    r, c = np.array([1e3, 2e3, 5e3]), np.array([1e-12, 1e-12, 2e-13])
    rc = decks.rc_points(3, r, c)
    om = np.logspace(5, 12, 15)
    with Lanes([rc]) as L:
        L.solve_static(abi.newton_opts())
        s = L.noise(0, om, rc.node("out"))
    want = oracle.KT4 * r[:, None] / (1.0 + (om[None, :] * (r * c)[:, None]) ** 2)
    np.testing.assert_allclose(s, want, rtol=1e-9)
    net = decks.miller_opamp(64)
    om = np.logspace(2, 10, 9)
    out = net.node("out")
    with Lanes([net]) as L:
        L.put_x(0, opamp_start(net), False)
        res = L.solve_static(abi.newton_opts(init_fix=0))
        x = L.get_x(0)
        psd, terms = L.noise_sources(0)
        s = L.noise(0, om, out)
    assert ((res[:, 0] & abi.CONVERGED) != 0).all()
    np.testing.assert_allclose(psd, oracle.noise_densities(net, x), rtol=1e-9, atol=1e-40)
    assert (psd > 0).any()
    np.testing.assert_allclose(s, oracle.noise_lanes(net, x, om, out, terms), rtol=1e-8)


def test_points_api(oracle):
    """The points mirror (egspice_b200/points.py, include/espice.h :244-362)
    on the lanes: 100 RC points appended in two calls and run as one batch,
    copied by id against the oracle's transient of the same values; the same
    rows appended in the reverse order give the same measures (a point's
    measures depend on its values, not its batch); a non-finite row comes
    back failed."""
    from egspice_b200 import points as pt
    from egspice_b200.netlist import measure_passes, measure_values, read_deck, read_measures
    deck = """RC points
vin in 0 dc 0 pulse(0 1 0 0.2n 0.2n 1 2)
r1 in out {rval}
c1 out 0 {cval}
.param rval=1k cval=1p
.tran 1p 6n
.meas tran t50 when v(out)=0.5
.meas tran v2n find v(out) at=2n
.meas tran rise trig v(out) val=0.1 rise=1 targ v(out) val=0.9 rise=1
.end
"""
    rng = np.random.default_rng(11)
    rows = np.stack([rng.uniform(0.5e3, 1.5e3, 100), rng.uniform(0.5e-12, 1.5e-12, 100)], axis=1)
    p = pt.Points(deck, ["rval", "cval"])
    a0 = p.append_points(rows[:60])
    a1 = p.append_points(rows[60:])
    bad = p.append_points([[1e3, np.inf]])
    assert (a0, a1, bad) == (0, 60, 100)
    p.run()
    names = ["t50", "v2n", "rise"]
    v, r = p.copy_point_measures(0, 100, names)
    assert (r == 0).all()
    vb, rb = p.copy_point_measures(bad, 1, names)
    assert np.isnan(vb).all() and rb[0] == pt.REASON_INVALID_PARAMETER
    params = {"rval": rows[:, 0], "cval": rows[:, 1]}
    net = read_deck(deck, lanes=100, params=params)
    ms = read_measures(deck, net, params=params)
    vo, _, _, ro = oracle.tran_meas(net, p.topts, measure_passes(ms), threads=8)
    want = measure_values(ms, vo)
    for j, name in enumerate(names):
        np.testing.assert_allclose(v[:, j], want[name], rtol=1e-6, atol=1e-9 if name == "v2n" else 0.0,
                                   err_msg=name)
    q = pt.Points(deck, ["rval", "cval"])
    q.append_points(rows[::-1])
    q.run()
    vr, _ = q.copy_point_measures(0, 100, names)
    np.testing.assert_allclose(vr[::-1], v, rtol=1e-9, atol=1e-15)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chain_fixture_points_in_three_orders(oracle, precision):
    """The reference's lane lockstep fixture (tests/golden/chain_deck.json,
    from src/tests/espice.zig:3072-3122) as points on the lanes, appended in
    the identity, reversed and a shuffled order: each row's TRIG/TARG
    measures and reason are bitwise the same in every order and match the
    oracle's transient of the row; the extreme wire is unresolved, the
    shorted wire refused as a topology change."""
    import json
    import os

    from egspice_b200 import points as pt
    from egspice_b200.netlist import measure_passes, measure_values, read_deck, read_measures
    fx = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "chain_deck.json")))
    rows, live, deck = np.array(fx["rows"]), fx["live"], fx["deck"]
    names = ["tpd", "trise", "tfall"]
    k = len(rows)
    orders = [np.arange(k), np.arange(k)[::-1], np.random.default_rng(207).permutation(k)]
    runs = []
    for order in orders:
        p = pt.Points(deck, live, precision=precision)
        p.append_points(rows[order])
        p.run()
        v, r = p.copy_point_measures(0, k, names)
        back = np.empty_like(v)
        back[order] = v
        rb = np.empty_like(r)
        rb[order] = r
        runs.append((back, rb))
    # every batch is led by the deck's own .param values, so every order
    # replays the same tape and each point's measures are the same bits
    # (src/tests/c_api.zig:884-920 expectSameBits)
    for v, r in runs[1:]:
        np.testing.assert_array_equal(r, runs[0][1])
        np.testing.assert_array_equal(v, runs[0][0])
    v, r = runs[0]
    assert list(r[:17]) == [0] * 17
    assert r[17] == 5 and r[18] == pt.REASON_TOPOLOGY_CHANGED  # MEASURE_UNRESOLVED, refused
    ok = rows[:18]
    params = {name: ok[:, j] for j, name in enumerate(live)}
    net = read_deck(deck, lanes=len(ok), params=params)
    ms = read_measures(deck, net, params=params)
    vo, _, _, _ = oracle.tran_meas(net, pt.Points(deck, live).topts, measure_passes(ms), threads=8)
    want = measure_values(ms, vo)
    for j, name in enumerate(names):
        np.testing.assert_allclose(v[:17, j], want[name][:17], rtol=1e-6, err_msg=name)
        assert np.isnan(v[17, j]) and np.isnan(want[name][17])


def test_points_operating_points():
    """An .op deck as points (egspice_b200/points.py): `.meas op ... find`
    reads each point's operating point; a resistive divider against its
    analytic node voltage and supply current (the source's branch current,
    from its + node through it: minus the current it delivers)."""
    from egspice_b200 import points as pt
    deck = """divider
vdd vdd 0 1.8
r1 vdd mid {rtop}
r2 mid 0 10k
.param rtop=10k
.op
.meas op vmid find v(mid)
.meas op idd find i(vdd)
.end
"""
    rtop = np.linspace(1e3, 1e5, 50)
    p = pt.Points(deck, ["rtop"])
    p.append_points(rtop[:, None])
    p.run()
    v, r = p.copy_point_measures(0, 50, ["vmid", "idd"])
    assert (r == 0).all()
    np.testing.assert_allclose(v[:, 0], 1.8 * 1e4 / (rtop + 1e4), rtol=1e-9)
    np.testing.assert_allclose(v[:, 1], -1.8 / (rtop + 1e4), rtol=1e-9)


def test_early_stop():
    """espl_meas_done / espl_request_stop: RC lanes whose measures all
    resolve early stop there (report status 4 before t_stop) with the same
    measures as the full run; the points layer's early_stop gives the same
    values and reasons as without it."""
    from egspice_b200 import points as pt
    from egspice_b200.netlist import measure_passes, read_deck, read_measures
    deck = """RC points
vin in 0 dc 0 pulse(0 1 0 0.2n 0.2n 1 2)
r1 in out {rval}
c1 out 0 1p
.param rval=1k
.tran 1p 20n
.meas tran t50 when v(out)=0.5
.meas tran rise trig v(out) val=0.1 rise=1 targ v(out) val=0.9 rise=1
.end
"""
    rval = np.linspace(0.5e3, 1.5e3, 40)
    params = {"rval": rval}
    net = read_deck(deck, lanes=40, params=params)
    passes = measure_passes(read_measures(deck, net, params=params))
    opts = pt.Points(deck, ["rval"]).topts
    with Lanes([net]) as L:
        L.set_meas(0, passes)
        full = L.run_tran(opts, steps_per_launch=2048)
        v_full, _ = L.get_meas(0)
    with Lanes([net]) as L:
        L.set_meas(0, passes)
        L.init_steps(opts)
        reps = None
        for _ in range(1000):
            reps = L.device_launch(256)
            if all(r.status != 0 for r in reps):
                break
            done = L.meas_done(0).all(axis=1)
            if done.any():
                L.request_stop(0, done)
        v_stop, _ = L.get_meas(0)
    assert all(r.status == 1 for r in full)
    assert all(r.status == 4 for r in reps) and max(r.t for r in reps) < opts.t_stop
    # launches of 256 steps resume the same step sequence as launches of 2048
    np.testing.assert_allclose(v_stop, v_full, rtol=1e-9)
    a = pt.Points(deck, ["rval"])
    b = pt.Points(deck, ["rval"], early_stop=True)
    for p in (a, b):
        p.append_points(rval[:, None])
        p.run()
    va, ra = a.copy_point_measures(0, 40, ["t50", "rise"])
    vb, rb = b.copy_point_measures(0, 40, ["t50", "rise"])
    np.testing.assert_allclose(va, vb, rtol=1e-9)
    assert (ra == 0).all() and (rb == 0).all()


def test_points_ac_measures(oracle):
    """An .ac deck as points: the operating point, the lanes' AC solve of
    the AC sources' excitation, and `.meas ac` cards (a -3 dB bandwidth, a
    gain at a frequency, a phase at an event, a peak) against the same
    measures of the oracle's dense AC solves, and the bandwidth against the
    RC's analytic 3 dB point."""
    import math

    from egspice_b200 import points as pt
    from egspice_b200.netlist import read_deck, read_measures
    deck = """RC AC
vin in 0 dc 0 ac 1
r1 in out {rval}
c1 out 0 1p
.param rval=1k
.ac dec 50 1meg 10g
.meas ac bw when vdb(out)=-3 fall=1
.meas ac g1m find vdb(out) at=1meg
.meas ac ph find vp(out) when vdb(out)=-3
.meas ac peak max vm(out)
.end
"""
    r = np.linspace(0.5e3, 2e3, 20)
    p = pt.Points(deck, ["rval"])
    p.append_points(r[:, None])
    p.run()
    names = ["bw", "g1m", "ph", "peak"]
    v, reasons = p.copy_point_measures(0, 20, names)
    assert (reasons == 0).all()
    net = read_deck(deck, lanes=20, params={"rval": r})
    ms = read_measures(deck, net, params={"rval": r})
    x = np.zeros((20, net.n))
    z = oracle.ac_solve_lanes(net, x, 2 * np.pi * p.freqs, pt.ac_rhs(net)[None, :], np.arange(net.n))[:, :, 0, :]
    want = pt.ac_measure_values(ms, p.freqs, z)
    for j, name in enumerate(names):
        np.testing.assert_allclose(v[:, j], want[name], rtol=1e-8, atol=1e-12, err_msg=name)
    f3 = math.sqrt(10 ** 0.3 - 1) / (2 * np.pi * r * 1e-12)
    np.testing.assert_allclose(v[:, 0], f3, rtol=2e-3)
