"""Benchmark of the lane-sweep hot path: sweep points per second on B200.

Workload: 16,384 Monte-Carlo lanes of a 31-stage MOS1 ring oscillator plus
32 seeded variants of 15-63 stages (32 lanes each, different patterns in the
same launches), trapezoidal transient with LTE step control, 5,000 accepted
steps per lane, and the oscillation period measured on the device. A "step"
of the benchmark is one complete sweep of all 17,408 points. The metric is
points/s of the mixed-precision lanes (FP32 LU and solves; FP64 device
evaluation, residual, refinement and step control) next to the plain FP64
lanes of the same build; a sample of lanes is checked against the FP64
oracle (period and final state).

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


def ring_check(nets, topts, xs, per_gpu, lanes_per_net=2, threads=None):
    """Worst error of the GPU lanes against the FP64 oracle on a sample:
    the oscillation period (.meas) and the final state."""
    from oracle import pyoracle as po
    threads = threads or os.cpu_count()
    worst_p, worst_x = 0.0, 0.0
    for k, (net, x) in enumerate(zip(nets, xs)):
        row = net.node("s1")
        xo, _, _, po_per = po.tran_lanes(net, topts, lane0=0, count=lanes_per_net, meas=(row, 0.9, 1e-9),
                                         threads=threads)
        pg = per_gpu[k][:lanes_per_net]
        ok = np.isfinite(po_per) & np.isfinite(pg)
        if ok.any():
            worst_p = max(worst_p, float((np.abs(pg[ok] - po_per[ok]) / (RTOL * np.abs(po_per[ok]))).max()))
        worst_x = max(worst_x, float((np.abs(x[:lanes_per_net] - xo) / (RTOL * np.abs(xo) + ATOL)).max()))
    return worst_p, worst_x


def run_ring_sweep(nets, topts, precision, steps_per_launch=5000):
    from egspice_b200.lanes import Lanes
    t0 = time.perf_counter()
    L = Lanes(nets, precision=precision, dt0=topts.dt)
    for i, net in enumerate(nets):
        L.set_period_meas(i, net.node("s1"), 0.9, 1e-9)
    L.init_steps(topts)
    dev_ms = L.stats().newton_ms
    calls = 0
    classes = None
    while True:
        reps = L.device_launch(steps_per_launch)
        calls += 1
        dev_ms += L.stats().newton_ms
        cl = L.classes()
        if classes is None:
            classes = cl
        else:
            for a, b in zip(classes, cl):
                a["ms"] += b["ms"]
        if all(r.status != 0 for r in reps) or calls > 1000:
            break
    launches = L.stats().launches  # Newton kernels: one per launch class per call
    periods = [L.period_meas(i)[0] for i in range(len(nets))]
    xs = [L.get_x(i) for i in range(len(nets))]
    wall = time.perf_counter() - t0
    tapes = []
    for i, net in enumerate(nets):
        t = L.tape(i)
        tapes.append((net, len(t["li"]), len(t["ui"])))
    L.close()
    return dev_ms, wall, xs, reps, tapes, launches, periods, classes


def opamp_nominal(net):
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    return x0


def run_learned_dc(points: int = 65536, train_points: int = 8192, epochs: int = 80, seed: int = 0, batch: int = 4096,
                   lr: float = 1e-2):
    """Config 4: a Monte-Carlo op-amp operating-point sweep (16 varied
    parameters). Plain: every point's Newton (FP64 LU) starts from the
    nominal operating point. Learned + mixed: the first `train_points` points
    are solved that way (FP32 LU), the MLP is trained on them on the GPU, and
    the remaining points start from its predictions. Time = Newton device time
    plus the MLP's training and inference (wall, synchronized). Garbage from
    earlier runs is collected before each wall-timed region, so no lane
    handle is freed inside one."""
    import gc
    from egspice_b200 import abi, decks
    from egspice_b200.lanes import Lanes
    from egspice_b200.learned import Mlp, train_opts
    net = decks.miller_opamp(points, base_seed=7 + 1000 * seed)
    x0 = opamp_nominal(net)
    opts = abi.newton_opts(init_fix=0)

    def solve(sub, start, precision):
        with Lanes([sub], precision=precision) as L:
            L.put_x(0, start, False)
            r = L.solve_static(opts)
            return r, L.get_x(0), L.stats().newton_ms

    r_plain, x_plain, dev_plain = solve(net, x0, "fp64")
    # context: the same points from the cold start through the continuation
    # ladder (what an operating point costs without a start point), wall time
    import torch
    with Lanes([net], precision="fp64") as L:
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
    t_mlp = time.perf_counter() - t0
    r_tail, x_tail, dev_tail = solve(tail, guess, "mixed")
    # plain Newton stays the fallback: a lane that does not converge from its
    # predicted start is solved again from the nominal one
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
    cur = np.asarray(net.current_rows, dtype=bool)
    newton_tol = opts.reltol * np.maximum(np.abs(x_plain), np.abs(x_learned)) + np.where(cur, opts.abstol, opts.vntol)
    err_newton = float((np.abs(x_learned - x_plain) / newton_tol).max())
    err_bar = float((np.abs(x_learned - x_plain) / (RTOL * np.abs(x_plain) + ATOL)).max())
    t_plain = dev_plain / 1e3
    t_learned = (dev_head + dev_tail) / 1e3 + t_mlp
    return {
        "workload": f"miller_opamp_mc_dc ({points:,} points, 16 varied parameters)",
        "plain_fp64": {"points_per_s": points / t_plain, "ms": t_plain * 1e3,
                       "mean_newton_iters": float(r_plain[:, 1].mean()), "converged": conv(r_plain)},
        "learned_mixed": {"points_per_s": points / t_learned, "ms": t_learned * 1e3,
                          "newton_ms": dev_head + dev_tail, "mlp_train_ms": t_train * 1e3,
                          "mlp_predict_ms": (t_mlp - t_train) * 1e3, "train_points": train_points,
                          "epochs": epochs, "batch": batch, "lr": lr, "final_loss": float(losses[-1]),
                          "mean_newton_iters_predicted": float(r_tail[:, 1].mean()),
                          "mean_newton_iters_all": float(r_learned[:, 1].mean()), "converged": conv(r_learned),
                          "fallbacks_to_nominal": refallback},
        "plain_cold_ladder_fp64": {"points_per_s": points / t_cold, "ms": t_cold * 1e3,
                                   "mean_newton_iters": float(r_cold[:, 1].mean()),
                                   "converged": conv(r_cold)},
        "learned_over_plain": t_plain / t_learned,
        "learned_over_cold_ladder": t_cold / t_learned,
        "max_err_over_newton_tol": err_newton,
        "max_err_over_1e-6_bar": err_bar,
        "note": "learned and plain runs stop at the same Newton test, so they agree to the Newton tolerance "
                "(reltol|x| + vntol), not bit for bit",
    }


def cpu_ring_reference(nets, topts, budget_s: float, threads: int):
    """The oracle on a bounded sample of the ring workload: lanes of the
    31-stage template (the workload's bulk), `threads` at a time, until the
    budget is spent."""
    from oracle import pyoracle as po
    t0 = time.perf_counter()
    points = 0
    lane = 0
    while time.perf_counter() - t0 < budget_s and lane < nets[0].lanes:
        po.tran_lanes(nets[0], topts, lane0=lane, count=threads, threads=threads)
        lane += threads
        points += threads
    wall = time.perf_counter() - t0
    return points / wall, points, wall


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
    ap.add_argument("--modes", default="fp64,mixed", help="precisions to run, comma-separated")
    ap.add_argument("--no-check", action="store_true", help="skip the oracle check of sampled lanes")
    ap.add_argument("--no-learned-dc", action="store_true", help="skip the learned warm-start DC measurement")
    args = ap.parse_args()
    modes = [m for m in args.modes.split(",") if m]
    if not modes or any(m not in ("fp64", "mixed") for m in modes):
        ap.error("--modes takes fp64 and/or mixed")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist_mod
        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    nets, topts = ring_workload(seed=rank, lanes=args.lanes, variants=args.variants)
    topts.max_steps = args.max_steps
    n_points = sum(n.lanes for n in nets)
    full = (args.lanes, args.variants, args.max_steps) == (16384, 32, 5000)
    config = {"workload": "ring_oscillator_mc_uneven" + ("" if full else " (reduced)"), "templates": len(nets),
              "lanes": n_points,
              "stages": f"31 ({args.lanes:,} lanes) + {args.variants} variants of 15-63 (32 lanes each)",
              "steps_per_lane": args.max_steps,
              "method": "trap, LTE step control", "predictor": "linear (SPICE xfact)",
              "meas": "oscillation period of stage 1 (rising 0.9 V)",
              "l2": "inputs larger than L2 (per-sweep working set > 126 MB)", "parallelism": f"lanes x{world} GPUs"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        vals = []
        pts_total = 0
        for _ in range(max(1, args.steps)):
            v, pts, wall = cpu_ring_reference(nets, topts, args.cpu_budget / max(1, args.steps), threads)
            vals.append(v)
            pts_total += pts
        v = statistics.median(vals)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * n_points / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded MC ring oscillators)", "config": config,
                "cpu_baseline": {"value": v, "unit": "points/s", "cores": threads, "kind": "port",
                                 "sample": f"{pts_total} lanes of the 31-stage template, 5,000 steps each, "
                                           f"{threads} threads"},
                "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    results = {}
    for prec in modes:
        for _ in range(args.warmup):
            run_ring_sweep(nets, topts, prec)
        dev_ms, walls = [], []
        barrier()
        with ClockSampler(dev) as clk:
            for _ in range(args.steps):
                barrier()
                d, w, xs, reps, tapes, launches, periods, classes = run_ring_sweep(nets, topts, prec)
                barrier()
                dev_ms.append(d)
                walls.append(w)
        dmax = max(dev_ms) / 1000.0
        wmax = max(walls)
        if dist:
            t = torch.tensor([dmax, wmax], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dmax, wmax = float(t[0]), float(t[1])
        results[prec] = dict(dev_s=dmax, wall_s=wmax, xs=xs, reps=reps, tapes=tapes, clocks=clk.summary(),
                             iters=sum(r.nr_iters for r in reps), rejects=sum(r.rejects for r in reps),
                             launches=launches, periods=periods, classes=classes)

    best = results.get("mixed") or results["fp64"]
    plain = results.get("fp64")
    points_all = n_points * world
    value = points_all / best["dev_s"]
    e2e = points_all / best["wall_s"]
    err = {}
    if rank == 0 and not args.no_check:
        sample = [0] + list(range(1, len(nets), 8))
        for prec in modes:
            r = results[prec]
            err[prec] = ring_check([nets[i] for i in sample], topts, [r["xs"][i] for i in sample],
                                   [r["periods"][i] for i in sample])
    per_net_iters = []
    off = 0
    for net in nets:
        per_net_iters.append(sum(r.nr_iters for r in best["reps"][off:off + net.lanes]))
        off += net.lanes
    bytes_alg = algorithmic_bytes(best["tapes"], per_net_iters, 4)
    hbm, kind = peaks()
    achieved = bytes_alg / best["dev_s"] / 1e9
    h2d = sum(sum(b.param.nbytes + b.term.nbytes for b in n.batches) + n.col_ptr.nbytes + n.row_idx.nbytes
              for n in nets)
    d2h = sum(n.lanes * n.n * 8 + n.lanes * 8 for n in nets)
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": best["dev_s"] * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (eval, residual, step control); f32 LU in mixed",
        "data": "synthetic (seeded Monte-Carlo MOS1 ring oscillators)", "config": config,
        "modes": dict(
            {m: {"points_per_s": points_all / results[m]["dev_s"], "ms_per_sweep": results[m]["dev_s"] * 1e3,
                 "newton_iters": results[m]["iters"], "rejects": results[m]["rejects"],
                 "period_err_over_tol": err.get(m, (None,))[0],
                 "final_x_err_over_tol": err.get(m, (None, None))[1],
                 "launch_classes": [[c["tiles"], int(c["wide"]), c["per_sm"], round(c["ms"], 1)]
                                    for c in results[m]["classes"]]} for m in modes},
            mixed_over_fp64=(plain["dev_s"] / best["dev_s"]) if (plain and "mixed" in results) else None,
            learned=False),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": kind,
                     "traffic": (DRAM_BYTES_PER_LANE_STEP * sum(r.steps for r in best["reps"]) / 1e9
                                 if "mixed" in results else None),
                     "traffic_unit": "GB per sweep (ncu capture scaled by lane-steps)",
                     "traffic_per_lane_step": DRAM_BYTES_PER_LANE_STEP if "mixed" in results else None,
                     "algorithmic_per_sweep_gb": bytes_alg / 1e9,
                     "kernel": ("k_tran<true>" if "mixed" in results else "k_tran<false>") +
                               ": per-tile eval + gather + shared-memory LU + gates, fused"},
        "e2e": {"value": e2e, "unit": "points/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(best["launches"]),
        "clocks": best["clocks"],
    }
    if not args.no_learned_dc:
        line["modes"]["learned_dc"] = run_learned_dc(seed=rank)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        v, pts, wall = cpu_ring_reference(nets, topts, args.cpu_budget, threads)
        line["cpu_baseline"] = {"value": v, "unit": "points/s", "cores": threads, "kind": "port",
                                "sample": f"{pts} lanes of the 31-stage template (5,000 steps each) in "
                                          f"{wall:.1f} s on {threads} threads"}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
