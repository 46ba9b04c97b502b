"""Edge cases of the GPU lanes through the C ABI, against the CPU FP64
oracle: lane counts that are not a multiple of the 32-lane tile (one lane,
33, 37, 70) sharing launches with other templates, a template past 64
unknowns whose cold operating point needs the dense re-pivoting peel on the
device, and an empty template, which the create call refuses. Tolerance as
in test_gpu_parity: |x - x_ref| <= 1e-6 |x_ref| + 1e-9."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.lanes import LaneError, Lanes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-9


def worst(x, xr):
    return float((np.abs(x - xr) / (RTOL * np.abs(xr) + ATOL)).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ragged_lane_counts_cold_operating_points(oracle, precision):
    nets = [decks.inverter_chain(1), decks.inverter_chain(33), decks.ring_oscillator(70, stages=15),
            decks.ring_oscillator(37, stages=31)]
    opts = abi.newton_opts()
    with Lanes(nets, precision=precision) as L:
        r = L.solve_static(opts)
        xs = [L.get_x(i) for i in range(len(nets))]
    lane0 = 0
    for net, x in zip(nets, xs):
        xo, ro = oracle.op_lanes(net, opts, threads=8)
        rg = r[lane0:lane0 + net.lanes]
        lane0 += net.lanes
        assert x.shape == (net.lanes, net.n)
        ok = (rg[:, 0] & abi.CONVERGED) != 0
        assert (ok | (ro[:, 0] != 1)).all(), (net.name, "a lane the oracle solves did not converge")
        both = ok & (ro[:, 0] == 1)
        assert worst(x[both], xo[both]) <= 1.0, net.name


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_peel_past_64_unknowns(oracle, precision):
    """The 63-stage ring (66 unknowns): from the cold start the replay of the
    lead lane's tape fails on the lanes, which re-pivot densely on the device
    instead of reporting singular. Most of a tile's lanes failing in one
    iteration marks the tape stale, so the solve ends with a tape rebuilt
    from a failing lane's matrix (the reference's retapeFrom); a warm solve
    from the answer runs on it."""
    net = decks.ring_oscillator(32, stages=63)
    assert net.n > 64
    opts = abi.newton_opts()
    xo, ro = oracle.op_lanes(net, opts, threads=8)
    with Lanes([net], precision=precision) as L:
        r = L.solve_static(opts)
        x = L.get_x(0)
        st = L.stats()
        peels, retapes = st.dense_peels, st.retapes
        L.put_x(0, x, False)
        r2 = L.solve_static(abi.newton_opts(init_fix=0))
        x2 = L.get_x(0)
        peels2 = L.stats().dense_peels
    print(f"dense peels: {peels}, retapes: {retapes}, warm solve's dense peels: {peels2}")
    assert (ro[:, 0] == 1).all()
    assert ((r[:, 0] & abi.CONVERGED) != 0).all(), r[:, 0]
    assert ((r[:, 0] & abi.SINGULAR) == 0).all()
    assert worst(x, xo) <= 1.0
    assert retapes >= 1
    assert ((r2[:, 0] & abi.CONVERGED) != 0).all(), r2[:, 0]
    assert worst(x2, xo) <= 1.0


def test_ragged_lane_counts_transient(oracle):
    """Two ring templates of 5 and 37 lanes in one transient launch: the
    same accepted and rejected steps as the oracle, lane by lane (FP64)."""
    nets = [decks.ring_oscillator(5, stages=15), decks.ring_oscillator(37, stages=31)]
    topts = abi.tran_opts(t_stop=0.5e-9, dt=1e-12, dt_max=5e-12, method=1, max_iter=20)
    with Lanes(nets) as L:
        reps = L.run_tran(topts, steps_per_launch=1024)
        xs = [L.get_x(i) for i in range(len(nets))]
    lane0 = 0
    for net, x in zip(nets, xs):
        xo, ro, _, _ = oracle.tran_lanes(net, topts, threads=8)
        mine = reps[lane0:lane0 + net.lanes]
        lane0 += net.lanes
        for a, b in zip(mine, ro):
            assert a.status == 1 and a.steps == b.steps and a.rejects == b.rejects, net.name
        assert worst(x, xo) <= 1.0, net.name


def test_empty_template_is_refused():
    net = decks.inverter_chain(4).subset([])
    assert net.lanes == 0
    with pytest.raises(LaneError):
        Lanes([net])
