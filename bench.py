"""Benchmark of the lane-sweep hot path: sweep points per second on B200.

Workload: 16,384 Monte-Carlo lanes of a 31-stage MOS1 ring oscillator plus
32 seeded variants of 15-63 stages (32 lanes each, different patterns in the
same launches), trapezoidal transient with LTE step control, 5,000 accepted
steps per lane, and the oscillation period measured on the device. A "step"
of the benchmark is one complete sweep of all 17,408 points. Three arms, all
with the Newton polish: plain FP64 lanes (linear predictor), mixed-precision
lanes (FP32 LU and solves; FP64 device evaluation, residual, refinement and
step control) and learned + mixed lanes (the bulk template's attempts start
from a step-predictor MLP trained on the device on the run's own first
steps). The metric is points/s of the learned + mixed arm; every lane of
every arm is checked against the polished FP64 oracle (period and final
state).

Launch: `python bench.py --gpus N --steps K --warmup W`; for N > 1 one rank
per GPU under torch.distributed.run (each rank runs its own seeded sweep:
weak scaling, no data-path collective). `--impl reference` times the CPU
FP64 restatement of the reference's CPU path on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sweep points/s on 1 B200: learned+mixed vs plain FP64 lanes at 1e-6 rel err"
RTOL, ATOL = 1e-6, 1e-9


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------
# workloads

def ring_workload(seed: int, lanes: int = 16384, variants: int = 32, lanes_per_variant: int = 32):
    """16,384 Monte-Carlo lanes of a 31-stage MOS1 ring oscillator (20 fF per
    stage, chain-like variation) plus 32 seeded variants of 15-63 stages
    (odd), 32 lanes each; trapezoidal transient with LTE step control, 5,000
    accepted steps per lane; the oscillation period measured on stage 1."""
    from egspice_b200 import abi, decks
    rng = np.random.default_rng(seed)
    nets = [decks.ring_oscillator(lanes, stages=31, base_seed=11 + 1000 * seed)]
    for v in range(variants):
        st = int(rng.integers(7, 32)) * 2 + 1
        nets.append(decks.ring_oscillator(lanes_per_variant, stages=st, base_seed=5000 + 97 * v + 1000 * seed))
    topts = abi.tran_opts(t_stop=1e-6, dt=2e-12, dt_max=10e-12, method=1, max_iter=20, max_steps=5000,
                          predictor=1)
    return nets, topts


# FP64 operations per lane-iteration of k_tran<true> (the mixed arm): the
# FP64 thread instructions of one launch (2 DFMA + DADD + DMUL, ncu
# smsp__sass_thread_inst_executed_op_{dfma,dadd,dmul}_pred_on.sum: 148.5 G
# over 6.34 M lane-iterations of 4,352 ring lanes x 300 polished steps)
# divided by its lane-iterations: device evaluation twice per iteration (the
# instance phase and the limiter pass), the gather, the update, gates and
# LTE. The pipe's activity in the same capture: 4.7 % of peak.
FP64_FLOPS_PER_LANE_ITERATION = 23420.0
FP64_PIPE_ACTIVE_PCT = 4.74
# B200 FP64 peak, nominal: 148 SMs x 64 FP64 FMA per clock x 2 x 1.965 GHz.
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12

# DRAM bytes per lane-step of the bulk k_tran class (31-stage ring lanes, mixed):
# dram__bytes_read.sum + dram__bytes_write.sum from one ncu capture of the
# benchmark's full lane count cut to 200 steps (425.9 GB for 16,704 lanes x 200
# steps), scaled by the run's lane-steps for the roofline's traffic figure.
DRAM_BYTES_PER_LANE_STEP = 127475.0


def algorithmic_bytes(nets, lane_iterations_per_net, s_lu: int):
    """SURVEY 8(d) bytes per lane-iteration, summed: refactor 8 nnz +
    s (nnzL + nnzU + n); solve s (nnzL + nnzU + n) + 16 n; update/gates 40 n;
    assembly 8 (nnz + n) + 16 nnz. Index words are shared by a template's
    lanes and excluded."""
    total = 0.0
    for (net, nl, nu), it in zip(nets, lane_iterations_per_net):
        n, nnz = net.n, net.nnz
        per = (8 * nnz + s_lu * (nl + nu + n)) + (s_lu * (nl + nu + n) + 16 * n) + 40 * n + \
              (8 * (nnz + n) + 16 * nnz)
        total += per * it
    return total


# Every arm and the oracle polish their Newton solves (espl_create_opts.polish,
# orc_set_polish): once the reference's test passes, Newton goes on until its
# step passes the test with the tolerances scaled by 10^-POLISH. The
# converged points then do not depend on where Newton started (the linear or
# the learned predictor, FP32 or FP64 factors) to far below the 1e-6 bar.
POLISH = 6


def run_ring_sweep(nets, topts, precision, learned=None, plan=None):
    """One full sweep through the C ABI from host buffers: create (uploads
    every lane's parameters), operating point, every transient step, final
    states and periods back. With `learned` (a dict: warm, stride, cap,
    epochs, batch, lr, lr_final), the bulk template (net 0) runs `warm`
    attempts with the linear predictor while the recorder samples every
    stride-th lane, a step predictor is trained on the device, and the rest
    of its transient starts each attempt from the network. Time: the CUDA-
    event time of the Newton launches plus that of the training (both device
    time; allocations, as in every arm, outside it). `plan`: the launch
    plan (espl_set_plan choices) the sweep runs with."""
    import copy
    from egspice_b200.lanes import Lanes
    from egspice_b200.learned import Mlp, step_predictor_dims, train_opts
    t0 = time.perf_counter()
    L = Lanes(nets, precision=precision, dt0=topts.dt, polish=POLISH)
    if plan is not None:
        L.set_plan(plan)
    for i, net in enumerate(nets):
        L.set_period_meas(i, net.node("s1"), 0.9, 1e-9)
    o = copy.copy(topts)
    o.predictor = 2 if learned else 1
    if learned:
        L.record_steps(0, learned["stride"], 0, learned["cap"])
    L.init_steps(o)
    dev_ms = L.stats().newton_ms
    classes = None
    m = None
    info = {}

    def launch(steps):
        nonlocal dev_ms, classes
        reps = L.device_launch(steps)
        dev_ms += L.stats().newton_ms
        cl = L.classes()
        if classes is None:
            classes = cl
        else:
            for a, b in zip(classes, cl):
                a["ms"] += b["ms"]
        return reps

    if learned:
        warm = launch(learned["warm"])
        x_ptr, y_ptr, count = L.recorded(0)
        tt = time.perf_counter()
        d_in, d_out = step_predictor_dims(nets[0].n)
        m = Mlp(d_in, d_out, capacity=learned["batch"], seed=7)
        losses = m.train_device(x_ptr, y_ptr, count, train_opts(epochs=learned["epochs"], batch=learned["batch"],
                                                                 lr=learned["lr"], lr_final=learned["lr_final"]))
        t_train = time.perf_counter() - tt
        train_dev = m.train_ms()
        L.record_steps(0, 1, 0, 0)
        L.set_step_predictor(0, m)
        info = dict(samples=count, train_ms=train_dev, train_wall_ms=t_train * 1e3, final_loss=float(losses[-1]),
                    warm_iters=sum(r.nr_iters for r in warm[:nets[0].lanes]),
                    warm_attempts=sum(r.attempts for r in warm[:nets[0].lanes]))
        dev_ms += train_dev
    calls = 0
    while True:
        reps = launch(100000)
        calls += 1
        if all(r.status != 0 for r in reps) or calls > 1000:
            break
    launches = L.stats().launches
    periods = [L.period_meas(i)[0] for i in range(len(nets))]
    xs = [L.get_x(i) for i in range(len(nets))]
    wall = time.perf_counter() - t0
    tapes = []
    for i, net in enumerate(nets):
        t = L.tape(i)
        tapes.append((net, len(t["li"]), len(t["ui"])))
    L.close()
    if m is not None:
        m.close()
    return dict(dev_s=dev_ms / 1e3, wall_s=wall, xs=xs, reps=reps, tapes=tapes, launches=launches, periods=periods,
                classes=classes, learned=info)


def oracle_ring(nets, topts, lanes=None, threads=None):
    """The polished FP64 oracle (linear predictor) on the first `lanes` lanes
    of every template (all when None): (final x, period) per template."""
    import copy
    from oracle import pyoracle as po
    threads = threads or os.cpu_count()
    o = copy.copy(topts)
    o.predictor = 1
    out = []
    with po.polish(POLISH):
        for net in nets:
            cnt = net.lanes if lanes is None else min(lanes, net.lanes)
            xo, reps, _, per = po.tran_lanes(net, o, lane0=0, count=cnt, meas=(net.node("s1"), 0.9, 1e-9),
                                             threads=threads)
            out.append((xo, per, [(r.steps, r.rejects) for r in reps]))
    return out


def ring_errors(res, ref, nets):
    """Worst period and final-state error over the 1e-6 bar against the
    oracle, how many lanes miss the bar (either), and for each such lane its
    accepted and rejected steps beside the oracle's: a lane whose step
    control took one decision differently (an LTE test on the edge of 0.9 dt)
    runs on another time grid from there."""
    wp, wx, bad, checked = 0.0, 0.0, 0, 0
    missed = []
    off = 0
    for t, (x, per, (xo, po_per, oreps)) in enumerate(zip(res["xs"], res["periods"], ref)):
        k = len(xo)
        ep = np.abs(per[:k] - po_per) / (RTOL * np.abs(po_per))
        ep = np.where(np.isfinite(po_per) & np.isfinite(per[:k]), ep, np.where(np.isnan(po_per) & np.isnan(per[:k]),
                                                                               0.0, np.inf))
        ex = (np.abs(x[:k] - xo) / (RTOL * np.abs(xo) + ATOL)).max(axis=1)
        wp, wx = max(wp, float(ep.max())), max(wx, float(ex.max()))
        over = np.nonzero((ep > 1.0) | (ex > 1.0))[0]
        bad += len(over)
        for l in over[:8]:
            r = res["reps"][off + l]
            missed.append({"template": f"{nets[t].name}", "lane": int(l), "period_err_over_tol": float(ep[l]),
                           "final_x_err_over_tol": float(ex[l]), "steps_rejects": [r.steps, r.rejects],
                           "oracle_steps_rejects": list(oreps[l])})
        checked += k
        off += nets[t].lanes
    return dict(period_err_over_tol=wp, final_x_err_over_tol=wx, lanes_over_bar=bad, lanes_checked=checked,
                lanes_over_bar_detail=missed)


def opamp_nominal(net):
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    return x0


def run_learned_dc(points: int = 65536, train_points: int = 8192, epochs: int = 80, seed: int = 0, batch: int = 4096,
                   lr: float = 1e-2, check: bool = True):
    """Config 4: a Monte-Carlo op-amp operating-point sweep (16 varied
    parameters), every solve polished. Plain: every point's Newton (FP64 LU)
    starts from the nominal operating point. Learned + mixed: the first
    `train_points` points are solved that way (FP32 LU), the MLP is trained on
    them on the GPU, and the remaining points start from its predictions; a
    lane that does not converge from its prediction is solved again from the
    nominal start. Time = Newton device time plus the MLP's training and
    inference (wall, synchronized). Every lane of both arms is checked against
    the polished FP64 oracle from the nominal start. Garbage from earlier runs
    is collected before each wall-timed region, so no lane handle is freed
    inside one."""
    import gc
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import Lanes
    from egspice_b200.learned import Mlp, train_opts
    net = decks.miller_opamp(points, base_seed=7 + 1000 * seed)
    x0 = opamp_nominal(net)
    opts = abi.newton_opts(init_fix=0)

    def solve(sub, start, precision, max_iter=None):
        o = opts if max_iter is None else abi.newton_opts(init_fix=0, max_iter=max_iter)
        with Lanes([sub], precision=precision, polish=POLISH) as L:
            L.put_x(0, start, False)
            r = L.solve_static(o)
            return r, L.get_x(0), L.stats().newton_ms

    r_plain, x_plain, dev_plain = solve(net, x0, "fp64")
    r_mixed, x_mixed, dev_mixed = solve(net, x0, "mixed")
    # context: the same points from the cold start through the continuation
    # ladder (what an operating point costs without a start point), wall time
    import torch
    with Lanes([net], precision="fp64", polish=POLISH) as L:
        gc.collect()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r_cold = L.solve_op(abi.newton_opts())
        t_cold = time.perf_counter() - t0
    head = net.subset(list(range(train_points)))
    tail = net.subset(list(range(train_points, points)))
    r_head, x_head, dev_head = solve(head, x0[:train_points], "mixed")
    gc.collect()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with Mlp(net.sweep.shape[1], net.n, capacity=8192, seed=7) as m:
        losses = m.train(net.sweep[:train_points], x_head, train_opts(epochs=epochs, batch=batch, lr=lr,
                                                                      lr_final=1e-4))
        t_train = time.perf_counter() - t0
        guess = m.predict(net.sweep[train_points:])
        predict_dev = m.predict_ms()
        train_dev = m.train_ms()
    t_mlp = time.perf_counter() - t0
    # from a learned start Newton gets three times the plain mean iteration
    # count; a lane that has not converged by then restarts from the nominal
    # point (one slow lane would otherwise hold its whole tile for 100)
    cap = int(max(10, 3 * np.ceil(r_plain[:, 1].mean())))
    r_tail, x_tail, dev_tail = solve(tail, guess, "mixed", max_iter=cap)
    bad = np.nonzero((r_tail[:, 0] & abi.CONVERGED) == 0)[0]
    refallback = len(bad)
    if refallback:
        rb, xb, dev_b = solve(tail.subset(list(bad)), x0[train_points + bad], "mixed")
        r_tail[bad] = rb
        x_tail[bad] = xb
        dev_tail += dev_b
    x_learned = np.concatenate([x_head, x_tail])
    r_learned = np.concatenate([r_head, r_tail])
    conv = lambda r: int(((r[:, 0] & abi.CONVERGED) != 0).sum())  # noqa: E731
    bar = lambda x, xr: float((np.abs(x - xr) / (RTOL * np.abs(xr) + ATOL)).max())  # noqa: E731
    t_plain = dev_plain / 1e3
    t_learned = (dev_head + dev_tail) / 1e3 + t_mlp
    out = {
        "workload": f"miller_opamp_mc_dc ({points:,} points, 16 varied parameters)",
        "polish": POLISH,
        "plain_fp64": {"points_per_s": points / t_plain, "ms": t_plain * 1e3,
                       "mean_newton_iters": float(r_plain[:, 1].mean()), "converged": conv(r_plain)},
        "plain_mixed": {"points_per_s": points / (dev_mixed / 1e3), "ms": dev_mixed,
                        "mean_newton_iters": float(r_mixed[:, 1].mean()), "converged": conv(r_mixed),
                        "fp64_refactor_fallbacks": int(r_mixed[:, 2].sum())},
        "learned_mixed": {"points_per_s": points / t_learned, "ms": t_learned * 1e3,
                          "newton_ms": dev_head + dev_tail, "mlp_train_ms": t_train * 1e3,
                          "mlp_predict_ms": (t_mlp - t_train) * 1e3,
                          "mlp_predict_device_ms": predict_dev, "mlp_train_device_ms": train_dev, "train_points": train_points,
                          "epochs": epochs, "batch": batch, "lr": lr, "final_loss": float(losses[-1]),
                          "mean_newton_iters_predicted": float(r_tail[:, 1].mean()),
                          "mean_newton_iters_all": float(r_learned[:, 1].mean()), "converged": conv(r_learned),
                          "fp64_refactor_fallbacks": int(r_learned[:, 2].sum()),
                          "learned_start_max_iter": cap, "fallbacks_to_nominal": refallback},
        "plain_cold_ladder_fp64": {"points_per_s": points / t_cold, "ms": t_cold * 1e3,
                                   "mean_newton_iters": float(r_cold[:, 1].mean()),
                                   "converged": conv(r_cold)},
        "learned_over_plain": t_plain / t_learned,
        "learned_over_cold_ladder": t_cold / t_learned,
        "learned_vs_plain_err_over_1e-6_bar": bar(x_learned, x_plain),
    }
    if check:
        from oracle import pyoracle as po
        with po.polish(POLISH):
            xo, ro = po.op_lanes(net, opts, x_in=x0, threads=os.cpu_count())
        out["oracle_check"] = {"lanes": points, "oracle_converged": int((ro[:, 0] == 1).sum()),
                               "plain_fp64_err_over_1e-6_bar": bar(x_plain, xo),
                               "learned_mixed_err_over_1e-6_bar": bar(x_learned, xo)}
    return out


def lu_bytes(net, nl, nu, s_lu, iterations, assembly=True):
    """SURVEY 8(d) algorithmic bytes of `iterations` lane-iterations of one
    template (refactor + solve + update/gates + assembly; index words are
    shared by the lanes and excluded)."""
    n, nnz = net.n, net.nnz
    per = (8 * nnz + s_lu * (nl + nu + n)) + (s_lu * (nl + nu + n) + 16 * n) + 40 * n
    if assembly:
        per += 8 * (nnz + n) + 16 * nnz
    return per * iterations


def run_config1(check: bool):
    """Config 1: 1,024 Monte-Carlo operating points of the 16-stage chain,
    FP64, from the cold start through the reference's operating-point path
    (espl_solve_op: the plain rung, then the continuation ladder for a lane
    it leaves), polished; every lane against the oracle's ladder."""
    import torch
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import Lanes
    net = decks.inverter_chain(1024)
    opts = abi.newton_opts()
    with Lanes([net], precision="fp64", polish=POLISH) as L:
        L.solve_op(opts)  # warm-up
    with Lanes([net], precision="fp64", polish=POLISH) as L:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = L.solve_op(opts)
        t = time.perf_counter() - t0
        x = L.get_x(0)
    out = {"workload": "inverter_chain_mc_op (1,024 points, 16 stages, cold start)", "precision": "fp64",
           "points_per_s": 1024 / t, "ms": t * 1e3, "mean_newton_iters": float(r[:, 1].mean()),
           "converged": int(((r[:, 0] & abi.CONVERGED) != 0).sum()), "time": "wall, synchronized"}
    if check:
        from oracle import pyoracle as po
        threads = os.cpu_count() or 1
        with po.polish(POLISH):
            t0 = time.perf_counter()
            xo, ro = po.op_ladder(net, opts, threads=threads)
            tc = time.perf_counter() - t0
        err = np.abs(x - xo) / (RTOL * np.abs(xo) + ATOL)
        out["oracle_check"] = {"lanes": 1024, "err_over_1e-6_bar": float(err.max()),
                               "lanes_over_bar": int((err.max(axis=1) > 1.0).sum()),
                               "oracle_converged": int((ro[:, 0] == 1).sum())}
        out["cpu_oracle"] = {"points_per_s": 1024 / tc, "threads": threads, "polish": POLISH}
    return out


def run_config2(check: bool, steps: int = 2000):
    """Config 2: 4,096 lanes from 64 seeded RC-diode ladders of 200-5,000
    nodes (64 lanes each, uneven patterns in the same launches), 2,000 fixed
    10 ps trapezoidal steps, FP64; lane 0 of eight ladders (the largest
    among them) against the oracle."""
    import torch
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import Lanes
    nets = decks.rc_diode_batch(n_nets=64, lanes_per_net=64)
    topts = abi.tran_opts(t_stop=steps * 10e-12, dt=10e-12, fixed_step=1, method=1, max_iter=50)
    with Lanes(nets, precision="fp64", dt0=topts.dt) as L:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.init_steps(topts)
        dev = L.stats().newton_ms
        reps = L.device_launch(100000)
        dev += L.stats().newton_ms
        t = time.perf_counter() - t0
        xs = [L.get_x(i) for i in range(len(nets))]
        tapes = [(len(L.tape(i)["li"]), len(L.tape(i)["ui"])) for i in range(len(nets))]
        cl = L.classes()
    pts = sum(n.lanes for n in nets)
    by = 0.0
    off = 0
    for net, (nl, nu) in zip(nets, tapes):
        by += lu_bytes(net, nl, nu, 8, sum(r.nr_iters for r in reps[off:off + net.lanes]))
        off += net.lanes
    hbm, kind = peaks()
    out = {"workload": f"rc_diode_ladders (64 nets of {min(n.n for n in nets)}-{max(n.n for n in nets)} unknowns, "
                       f"64 lanes each, {steps} fixed trap steps)", "precision": "fp64",
           "points_per_s": pts / (dev / 1e3), "ms": dev, "wall_ms": t * 1e3,
           "all_done": all(r.status == 1 and r.steps == steps for r in reps),
           "newton_iters": sum(r.nr_iters for r in reps),
           "roofline": {"bound": "hbm", "achieved_gbs": by / (dev / 1e3) / 1e9, "peak": hbm, "peak_kind": kind,
                        "frac": by / (dev / 1e3) / 1e9 / hbm},
           "launch_classes": [[c["tiles"], int(c["wide"]), c["per_sm"], c["smem_bytes"], round(c["ms"], 1)]
                              for c in cl]}
    if check:
        from oracle import pyoracle as po
        order = sorted(range(len(nets)), key=lambda i: nets[i].n)
        pick = order[-4:] + order[:4]
        worst = 0.0
        for i in pick:
            xo, _, _, _ = po.tran_lanes(nets[i], topts, lane0=0, count=1, threads=1)
            worst = max(worst, float((np.abs(xs[i][:1] - xo) / (RTOL * np.abs(xo) + ATOL)).max()))
        out["oracle_check"] = {"lanes": f"lane 0 of {len(pick)} ladders ({nets[pick[0]].n} unknowns the largest)",
                               "err_over_1e-6_bar": worst}
    return out


def run_config3(check: bool, steps: int = 100):
    """Config 3: 256 lanes of the 200 x 200 power-grid mesh (40,005
    unknowns), trapezoidal fixed 10 ps steps, mixed (FP32 LU and solves,
    FP64 residual) and FP64, through the large-template LU (the whole CTA
    refactors by columns and solves by levels); two lanes against the
    oracle. `steps` of the config's 1,000 (the per-step cost is flat)."""
    import torch
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import Lanes
    net = decks.power_grid(256, side=200, loads=400)
    topts = abi.tran_opts(t_stop=steps * 10e-12, dt=10e-12, fixed_step=1, method=1, max_iter=20)
    out = {"workload": f"power_grid_mesh (256 lanes, 200 x 200, {net.n} unknowns, {steps} of 1,000 fixed trap "
                       f"steps)"}
    hbm, kind = peaks()
    for prec in ("mixed", "fp64"):
        with Lanes([net], precision=prec, dt0=topts.dt) as L:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            L.init_steps(topts)
            op_ms = L.stats().newton_ms
            reps = L.device_launch(100000)
            dev = L.stats().newton_ms
            t = time.perf_counter() - t0
            x = L.get_x(0)
            tp = L.tape(0)
        its = sum(r.nr_iters for r in reps)
        s_lu = 4 if prec == "mixed" else 8
        # per Newton iteration of a linear lane the factor is reused: the
        # solve pair's bytes (refactors: three per run, counted apart)
        nl, nu = len(tp["li"]), len(tp["ui"])
        solve_bytes = (s_lu * (nl + nu + net.n) + 16 * net.n) * its
        d = {"points_per_s": 256 / ((op_ms + dev) / 1e3), "ms": op_ms + dev, "transient_ms": dev,
             "operating_point_ms": op_ms, "wall_ms": t * 1e3, "newton_iters_per_lane": its / 256,
             "all_done": all(r.status == 1 and r.steps == steps for r in reps), "nnz_l": nl, "nnz_u": nu,
             "solve_roofline": {"bound": "hbm", "achieved_gbs": solve_bytes / (dev / 1e3) / 1e9, "peak": hbm,
                                "peak_kind": kind, "frac": solve_bytes / (dev / 1e3) / 1e9 / hbm,
                                "note": "the transient's solve bytes over its whole time (refactors included)"}}
        if check:
            from oracle import pyoracle as po
            worst = 0.0
            for l in (0, 255):
                xo, _, _, _ = po.tran_lanes(net, topts, lane0=l, count=1, threads=1)
                worst = max(worst, float((np.abs(x[l:l + 1] - xo) / (RTOL * np.abs(xo) + ATOL)).max()))
            d["oracle_check"] = {"lanes": "0 and 255", "err_over_1e-6_bar": worst}
        out[prec] = d
    return out


def reference_mix(nets, seed: int = 0):
    """The points of the sweep in one fixed shuffled order (the 31-stage bulk
    and the variants in the proportions of the sweep), for the CPU legs."""
    pts = [(i, l) for i, net in enumerate(nets) for l in range(net.lanes)]
    order = np.random.default_rng(seed).permutation(len(pts))
    return [pts[k] for k in order]


def cpu_ring_reference(nets, topts, budget_s: float, threads: int, mix=None, start: int = 0):
    """The oracle (the reference's CPU path restated: linear predictor, no
    polish) on a bounded sample of the sweep: points of `mix` from `start`
    on, `threads` at a time (one point per thread), until `budget_s` is
    spent. Returns (points/s, points, wall s, next start)."""
    import copy
    from oracle import pyoracle as po
    mix = mix or reference_mix(nets)
    o = copy.copy(topts)
    o.predictor = 1
    t0 = time.perf_counter()
    points = 0
    k = start
    while time.perf_counter() - t0 < budget_s:
        sel = [mix[(k + j) % len(mix)] for j in range(threads)]
        jobs = [threading.Thread(target=po.tran_lanes, args=(nets[i], o), kwargs=dict(lane0=l, count=1, threads=1))
                for i, l in sel]
        for th in jobs:
            th.start()
        for th in jobs:
            th.join()
        k += threads
        points += threads
    wall = time.perf_counter() - t0
    return points / wall, points, wall, k


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # smaller cases of the same workload (profiling); the defaults are the benchmark
    ap.add_argument("--lanes", type=int, default=16384, help="lanes of the 31-stage template")
    ap.add_argument("--variants", type=int, default=32, help="seeded 15-63-stage variants, 32 lanes each")
    ap.add_argument("--max-steps", type=int, default=5000, help="accepted steps per lane")
    ap.add_argument("--modes", default="fp64,mixed,learned",
                    help="arms to run, comma-separated: fp64, mixed, learned (learned + mixed)")
    ap.add_argument("--check", default="all", choices=["all", "sample", "none"],
                    help="lanes checked against the polished oracle")
    ap.add_argument("--no-learned-dc", action="store_true", help="skip the learned warm-start DC measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the runs of configs 1-3")
    ap.add_argument("--config3-steps", type=int, default=100, help="steps of the config-3 mesh run (of 1,000)")
    # the learned arm's step predictor
    ap.add_argument("--no-autotune", action="store_true", help="run the automatic launch plan, no search")
    ap.add_argument("--polish-chord", action="store_true",
                    help="polish iterations reuse the previous factor (espl_tran_opts.polish_chord), every arm")
    ap.add_argument("--tune-steps", type=int, default=200, help="transient attempts per autotuner trial")
    ap.add_argument("--tune-trials", type=int, default=10, help="autotuner trials per precision")
    ap.add_argument("--learn-warm", type=int, default=500, help="attempts with the linear predictor and recorder")
    ap.add_argument("--learn-stride", type=int, default=32, help="the recorder samples every stride-th bulk lane")
    ap.add_argument("--learn-epochs", type=int, default=5)
    ap.add_argument("--learn-batch", type=int, default=8192)
    ap.add_argument("--learn-lr", type=float, default=3e-3)
    args = ap.parse_args()
    modes = [m for m in args.modes.split(",") if m]
    if not modes or any(m not in ("fp64", "mixed", "learned") for m in modes):
        ap.error("--modes takes fp64, mixed and/or learned")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    nets, topts = ring_workload(seed=rank, lanes=args.lanes, variants=args.variants)
    topts.polish_chord = 1 if args.polish_chord else 0
    topts.max_steps = args.max_steps
    n_points = sum(n.lanes for n in nets)
    full = (args.lanes, args.variants, args.max_steps) == (16384, 32, 5000)
    config = {"workload": "ring_oscillator_mc_uneven" + ("" if full else " (reduced)"), "templates": len(nets),
              "lanes": n_points,
              "stages": f"31 ({args.lanes:,} lanes) + {args.variants} variants of 15-63 (32 lanes each)",
              "steps_per_lane": args.max_steps,
              "method": "trap, LTE step control",
              "predictor": "learned (MLP on the last 3 solutions and the step) vs linear (SPICE xfact)",
              "newton_polish": f"10^-{POLISH} of the Newton tolerances, every arm and the oracle",
              "meas": "oscillation period of stage 1 (rising 0.9 V)",
              "l2": "inputs larger than L2 (per-sweep working set > 126 MB)", "parallelism": f"lanes x{world} GPUs"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        mix = reference_mix(nets)
        budget = max(1.0, args.cpu_budget / max(1, args.steps))
        k = 0
        for _ in range(args.warmup and 1):
            _, _, _, k = cpu_ring_reference(nets, topts, min(budget, 2.0), threads, mix, k)
        pts_total, wall_total, walls = 0, 0.0, []
        for _ in range(max(1, args.steps)):
            _, pts, wall, k = cpu_ring_reference(nets, topts, budget, threads, mix, k)
            pts_total += pts
            wall_total += wall
            walls.append(wall)
        v = pts_total / wall_total
        sample = (f"{pts_total} points of the sweep's template mix (31-stage bulk and 15-63-stage variants in "
                  f"proportion, 5,000 steps each), {threads} threads, one point per thread; a step is one bounded "
                  f"sample of ~{budget:.1f} s; scalar C restatement (-O3, x86-64-v3, no FP contraction), not the "
                  f"reference's @Vector(W) lanes")
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(walls),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded MC ring oscillators)", "config": config,
                "cpu_baseline": {"value": v, "unit": "points/s", "cores": threads, "kind": "port", "sample": sample},
                "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist_mod
        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import torch
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    learn = dict(warm=args.learn_warm, stride=args.learn_stride,
                 cap=(args.lanes // args.learn_stride + 1) * args.learn_warm, epochs=args.learn_epochs,
                 batch=args.learn_batch, lr=args.learn_lr, lr_final=args.learn_lr / 10)
    # the launch plan of each precision, searched by timing short
    # transients (espl_autotune), before any arm; once per process
    plans, tuned = {}, {}
    for prec in dict.fromkeys("fp64" if m == "fp64" else "mixed" for m in modes):
        if args.no_autotune:
            plans[prec] = None
            continue
        from egspice_b200.lanes import autotune
        tt = time.perf_counter()
        plans[prec], rep = autotune(nets, topts, precision=prec, dt0=topts.dt, polish=POLISH,
                                    trial_steps=args.tune_steps, max_trials=args.tune_trials)
        rep["wall_s"] = time.perf_counter() - tt
        rep["trial_steps"] = args.tune_steps
        rep["plan"] = [[c.tile, c.stage, c.per_sm] for c in plans[prec]]
        rep["plan_fields"] = "per template: tile (0 auto, 1 narrow, 2 wide), stage (0 auto, 1 LU chain and records, " \
                             "2 LU chain, records global, 3 index words, 4 none), resident tiles per SM cap (0 none)"
        tuned[prec] = rep
    results = {}
    for k, mode in enumerate(modes):
        prec = "fp64" if mode == "fp64" else "mixed"
        lk = learn if mode == "learned" else None
        # W warm-up sweeps before the first arm; later arms (the same
        # kernels, the device already warm) one each
        for _ in range(args.warmup if k == 0 else min(args.warmup, 1)):
            run_ring_sweep(nets, topts, prec, lk, plans[prec])
        runs = []
        barrier()
        with ClockSampler(dev) as clk:
            for _ in range(args.steps):
                barrier()
                runs.append(run_ring_sweep(nets, topts, prec, lk, plans[prec]))
                barrier()
        r = runs[-1]
        dmax = max(x["dev_s"] for x in runs)
        wmax = max(x["wall_s"] for x in runs)
        if dist:
            t = torch.tensor([dmax, wmax], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dmax, wmax = float(t[0]), float(t[1])
        r.update(dev_s=dmax, wall_s=wmax, clocks=clk.summary())
        results[mode] = r

    head = "learned" if "learned" in results else "mixed" if "mixed" in results else "fp64"
    best = results[head]
    plain = results.get("fp64")
    points_all = n_points * world
    value = points_all / best["dev_s"]
    e2e = points_all / best["wall_s"]
    errs = {}
    check_s = None
    if rank == 0 and args.check != "none":
        tc = time.perf_counter()
        ref = oracle_ring(nets, topts, lanes=None if args.check == "all" else 2)
        check_s = time.perf_counter() - tc
        errs = {m: ring_errors(results[m], ref, nets) for m in results}
    mix_run = results.get("mixed") or best
    per_net_iters = []
    off = 0
    for net in nets:
        per_net_iters.append(sum(r.nr_iters for r in mix_run["reps"][off:off + net.lanes]))
        off += net.lanes
    s_lu = 8 if mix_run is plain else 4
    mix_run_iters = sum(r.nr_iters for r in mix_run["reps"])
    bytes_alg = algorithmic_bytes(mix_run["tapes"], per_net_iters, s_lu)
    hbm, kind = peaks()
    achieved = bytes_alg / mix_run["dev_s"] / 1e9
    h2d = sum(sum(b.param.nbytes + b.term.nbytes for b in n.batches) + n.col_ptr.nbytes + n.row_idx.nbytes
              for n in nets)
    d2h = sum(n.lanes * n.n * 8 + n.lanes * 8 for n in nets)

    def arm(m):
        r = results[m]
        it = sum(x.nr_iters for x in r["reps"])
        at = sum(x.attempts for x in r["reps"])
        d = {"points_per_s": points_all / r["dev_s"], "ms_per_sweep": r["dev_s"] * 1e3,
             "newton_iters": it, "attempts": at, "iters_per_attempt": it / max(at, 1),
             "rejects": sum(x.rejects for x in r["reps"]), "gpu_launches": int(r["launches"]),
             "launch_classes": [[c["tiles"], int(c["wide"]), c["per_sm"], c["smem_bytes"], round(c["ms"], 1)]
                                for c in (r["classes"] or [])],
             "launch_classes_fields": "tiles, wide, resident tiles per SM, dynamic shared bytes per tile, ms",
             "clocks": r["clocks"]}
        d.update(errs.get(m, {}))
        if m == "learned":
            bulk = r["reps"][:nets[0].lanes]
            info = r["learned"]
            it_b = sum(x.nr_iters for x in bulk) - info["warm_iters"]
            at_b = sum(x.attempts for x in bulk) - info["warm_attempts"]
            d["step_predictor"] = dict(info, template="31-stage ring (bulk)", warm_attempts_per_lane=args.learn_warm,
                                       recorder_stride=args.learn_stride, epochs=args.learn_epochs,
                                       batch=args.learn_batch, lr=args.learn_lr,
                                       bulk_iters_per_attempt_after_warm=it_b / max(at_b, 1),
                                       learned_retries=sum(x.learned_retries for x in bulk))
        return d

    modes_out = {m: arm(m) for m in results}
    if plain and "mixed" in results:
        p = results["mixed"]
        bulk_p = p["reps"][:nets[0].lanes]
        modes_out["mixed"]["bulk_iters_per_attempt"] = (sum(x.nr_iters for x in bulk_p) /
                                                        max(1, sum(x.attempts for x in bulk_p)))
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": best["dev_s"] * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (eval, residual, step control); f32 LU in mixed; bf16 MLP (f32 accumulation)",
        "data": "synthetic (seeded Monte-Carlo MOS1 ring oscillators)", "config": config,
        "headline_arm": head,
        "modes": dict(modes_out,
                      learned_mixed_over_fp64=(plain["dev_s"] / results["learned"]["dev_s"])
                      if (plain and "learned" in results) else None,
                      mixed_over_fp64=(plain["dev_s"] / results["mixed"]["dev_s"])
                      if (plain and "mixed" in results) else None,
                      learned_predictor=head == "learned",
                      autotune=tuned or None,
                      oracle_check={"lanes": "all" if args.check == "all" else "2 per template",
                                    "polish": POLISH, "seconds": check_s} if errs else None),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": kind,
                     "traffic": (DRAM_BYTES_PER_LANE_STEP * sum(r.steps for r in mix_run["reps"]) / 1e9
                                 if mix_run is not plain else None),
                     "traffic_unit": "GB per sweep (ncu capture scaled by lane-steps)",
                     "traffic_per_lane_step": DRAM_BYTES_PER_LANE_STEP if mix_run is not plain else None,
                     "algorithmic_per_sweep_gb": bytes_alg / 1e9,
                     "kernel": ("k_tran<true>" if mix_run is not plain else "k_tran<false>") +
                               ": per-tile eval + gather + shared-memory LU + gates, fused (the mixed arm)"},
        "roofline_fp64": ({"bound": "fp64", "kernel": "k_tran<true> (the mixed arm): device evaluation and the rest "
                                                    "of the step in FP64",
                           "flops_per_lane_iteration": FP64_FLOPS_PER_LANE_ITERATION,
                           "achieved": FP64_FLOPS_PER_LANE_ITERATION * mix_run_iters / mix_run["dev_s"] / 1e12,
                           "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                           "frac": FP64_FLOPS_PER_LANE_ITERATION * mix_run_iters / mix_run["dev_s"] / 1e12 /
                                   FP64_PEAK_TFLOPS,
                           "peak_kind": "nominal (148 SMs x 64 FP64 FMA per clock x 2 x 1.965 GHz)",
                           "pipe_active_pct_ncu": FP64_PIPE_ACTIVE_PCT}
                          if mix_run is not plain else None),
        "e2e": {"value": e2e, "unit": "points/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(best["launches"]),
        "clocks": best["clocks"],
    }
    if not args.no_learned_dc:
        line["modes"]["learned_dc"] = run_learned_dc(seed=rank, check=rank == 0 and args.check != "none")
    if not args.no_configs:
        chk = rank == 0 and args.check != "none"
        line["modes"]["configs"] = {"config1": run_config1(chk), "config2": run_config2(chk),
                                    "config3": run_config3(chk, steps=args.config3_steps),
                                    "note": "one run each, outside the headline's timed sweeps"}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        v, pts, wall, _ = cpu_ring_reference(nets, topts, args.cpu_budget, threads)
        line["cpu_baseline"] = {"value": v, "unit": "points/s", "cores": threads, "kind": "port",
                                "sample": f"{pts} points of the sweep's template mix (5,000 steps each, the "
                                          f"reference's linear predictor, no polish) in {wall:.1f} s on {threads} "
                                          f"threads"}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
