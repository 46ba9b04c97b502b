"""The launch plan (espl_set_plan / espl_get_plan) and its autotuner
(espl_autotune) on the GPU: a chosen plan takes effect, FP64 lanes give the
same answer bit for bit under every plan (each plan runs the same
operations on each lane in the same order), and the autotuner returns a plan
no slower than the automatic one from a bounded number of trials, cached
for the process."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.abi import PlanChoice
from egspice_b200.lanes import Lanes, autotune

pytestmark = pytest.mark.gpu


def nets():
    return [decks.ring_oscillator(64, stages=31), decks.ring_oscillator(32, stages=15, base_seed=3),
            decks.ring_oscillator(32, stages=63, base_seed=5)]


def topts(steps):
    return abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=steps, predictor=1)


def run(ns, choices, steps=200):
    with Lanes(ns, precision="fp64", polish=6) as L:
        if choices is not None:
            L.set_plan(choices)
        plan = L.plan()
        L.init_steps(topts(steps))
        reps = L.device_launch(100000)
        xs = [L.get_x(k) for k in range(len(ns))]
    return plan, reps, xs


def test_chosen_plans_take_effect_and_keep_the_answer():
    ns = nets()
    plan0, reps0, x0 = run(ns, None)
    assert all(r.status == 1 and r.steps == 200 for r in reps0)
    variants = [
        [PlanChoice(abi.TILE_WIDE, 0, 0, 0)] * 3,
        [PlanChoice(abi.TILE_NARROW, abi.STAGE_LU_GLOBAL_RECORDS, 0, 0)] * 3,
        [PlanChoice(abi.TILE_NARROW, abi.STAGE_INDEX, 1, 0)] * 3,
        [PlanChoice(0, abi.STAGE_NONE, 2, 0)] * 3,
    ]
    for ch in variants:
        plan, reps, xs = run(ns, ch)
        for p, c in zip(plan, ch):
            if c.tile:
                assert p["tile"] == c.tile
            if c.per_sm:
                assert p["per_sm"] <= c.per_sm
            if c.stage in (abi.STAGE_INDEX, abi.STAGE_NONE):
                assert p["stage"] == c.stage
        assert [(r.steps, r.attempts, r.nr_iters) for r in reps] == [(r.steps, r.attempts, r.nr_iters) for r in reps0]
        for a, b in zip(xs, x0):
            assert np.array_equal(a, b)


def test_autotune_bounded_and_cached():
    ns = nets()
    o = topts(100)
    choices, rep = autotune(ns, o, precision="mixed", polish=6, trial_steps=50, max_trials=6)
    assert len(choices) == len(ns)
    assert 2 <= rep["trials"] <= 6 and rep["cached"] == 0
    assert rep["best_ms"] <= rep["auto_ms"]
    again, rep2 = autotune(ns, o, precision="mixed", polish=6, trial_steps=50, max_trials=6)
    assert rep2["cached"] == 1 and rep2["trials"] == rep["trials"]
    assert [(c.tile, c.stage, c.per_sm) for c in again] == [(c.tile, c.stage, c.per_sm) for c in choices]
    # the chosen plan runs
    with Lanes(ns, precision="mixed", polish=6) as L:
        L.set_plan(choices)
        L.init_steps(o)
        reps = L.device_launch(100000)
    assert all(r.status == 1 and r.steps == 100 for r in reps)
