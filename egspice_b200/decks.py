"""Seeded synthetic decks for the lane sweeps, built directly as MNA netlists.

The reference reads SPICE decks through its front end (src/frontend/) and
freezes them into a CSC pattern plus device batches (src/device/Circuit.zig
`freeze`). Here the generators write that frozen form themselves: unknown 0
is the ground row, then the circuit nodes, then one branch-current unknown
per voltage source. A device terminal on the datum node is ESPL_GROUND.

Monte-Carlo draws follow the reference's counter-based sampler
(src/frontend/variants.zig:1680-1745): the uniform of trial `trial` at
`site` is ((siteKey(siteKey(seed, trial), site) >> 11) + 0.5) * 2^-53
(siteKey is src/frontend/netlist.zig:683-688), mapped through Acklam's
inverse normal (src/core/numerics.zig:416-432). Each point draws with
seed = base_seed + point index and trial 1, so a point's values depend only
on its own index.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

GROUND = 0xFFFFFFFF
RES, CAP, VSRC, ISRC, DIODE, MOS1 = 1, 2, 3, 4, 5, 6
TERMS = {RES: 2, CAP: 2, VSRC: 3, ISRC: 2, DIODE: 2, MOS1: 4}
PARAMS = {RES: 1, CAP: 1, VSRC: 9, ISRC: 9, DIODE: 7, MOS1: 9}
# Which (row terminal, column terminal) Jacobian entries each kind stamps.
_STAMPS = {
    RES: [(r, c) for r in range(2) for c in range(2)],
    CAP: [(r, c) for r in range(2) for c in range(2)],
    DIODE: [(r, c) for r in range(2) for c in range(2)],
    VSRC: [(0, 2), (1, 2), (2, 0), (2, 1)],
    ISRC: [],
    MOS1: [(r, c) for r in (0, 2, 3) for c in range(4)],
}

_M64 = (1 << 64) - 1


def site_key(owner: np.ndarray, salt: np.ndarray) -> np.ndarray:
    """splitmix64's finalizer over owner ^ (salt + golden): netlist.zig:683-688."""
    owner = np.asarray(owner, dtype=np.uint64)
    salt = np.asarray(salt, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = owner ^ (salt + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed: np.ndarray, trial: int, site: int) -> np.ndarray:
    """Sampler.uniform without Latin hypercube (variants.zig:1710-1716)."""
    bits = site_key(site_key(seed, np.uint64(trial)), np.uint64(site))
    return ((bits >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


_A = (-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
      1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00)
_B = (-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
      6.680131188771972e+01, -1.328068155288572e+01)
_C = (-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
      -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00)
_D = (7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
      3.754408661907416e+00)


def normal_quantile(u: np.ndarray) -> np.ndarray:
    """Acklam's rational approximation, numerics.zig:416-432, vectorized."""
    u = np.asarray(u, dtype=np.float64)
    low = 0.02425
    out = np.empty_like(u)
    tail = (u < low) | (u > 1 - low)
    if np.any(tail):
        ut = u[tail]
        q = np.sqrt(-2 * np.log(np.where(ut < low, ut, 1 - ut)))
        x = (((((_C[0] * q + _C[1]) * q + _C[2]) * q + _C[3]) * q + _C[4]) * q + _C[5]) / \
            ((((_D[0] * q + _D[1]) * q + _D[2]) * q + _D[3]) * q + 1)
        out[tail] = np.where(ut < low, x, -x)
    mid = ~tail
    if np.any(mid):
        q = u[mid] - 0.5
        r = q * q
        out[mid] = (((((_A[0] * r + _A[1]) * r + _A[2]) * r + _A[3]) * r + _A[4]) * r + _A[5]) * q / \
            (((((_B[0] * r + _B[1]) * r + _B[2]) * r + _B[3]) * r + _B[4]) * r + 1)
    return out


def mc_normal(seeds: np.ndarray, site: int) -> np.ndarray:
    return normal_quantile(uniform(seeds, 1, site))


@dataclasses.dataclass
class Batch:
    kind: int
    term: np.ndarray   # [count, terms] uint32
    param: np.ndarray  # [count, params, lanes] float64 (C order = lane-major rows)


@dataclasses.dataclass
class Netlist:
    """A frozen template: CSC pattern, device batches, lanes."""
    name: str
    n: int
    col_ptr: np.ndarray
    row_idx: np.ndarray
    batches: List[Batch]
    lanes: int
    node_names: Dict[str, int]
    current_rows: np.ndarray  # uint8 [n]
    # Sweep parameters per lane (the MLP's inputs), [lanes, k]; may be empty.
    sweep: Optional[np.ndarray] = None
    # The branch-current unknown of each named voltage source.
    branch_names: Dict[str, int] = dataclasses.field(default_factory=dict)
    # Small-signal sources: ("v", branch row, mag, phase in degrees) or
    # ("i", from row, to row, mag, phase), rows GROUND where grounded.
    ac_sources: List[tuple] = dataclasses.field(default_factory=list)

    @property
    def nnz(self) -> int:
        return int(self.col_ptr[-1])

    def node(self, name: str) -> int:
        return self.node_names[name]

    def subset(self, lanes: Sequence[int]) -> "Netlist":
        idx = np.asarray(lanes, dtype=np.int64)
        bs = [Batch(b.kind, b.term, np.ascontiguousarray(b.param[:, :, idx])) for b in self.batches]
        sw = None if self.sweep is None else np.ascontiguousarray(self.sweep[idx])
        return dataclasses.replace(self, batches=bs, lanes=len(idx), sweep=sw)


class Builder:
    """Collects devices by node name and freezes them into a Netlist."""

    def __init__(self, name: str, lanes: int):
        self.name = name
        self.lanes = lanes
        self.nodes: Dict[str, int] = {}
        self.devs: Dict[int, List[Tuple[List[str], np.ndarray]]] = {k: [] for k in TERMS}
        self.vsrc_names: List[str] = []
        self.vsrc_labels: Dict[str, str] = {}
        self.ac: List[tuple] = []  # ("v", branch name, mag, ph) or ("i", p, n, mag, ph)

    def _lane(self, v) -> np.ndarray:
        a = np.asarray(v, dtype=np.float64)
        if a.ndim == 0:
            a = np.full(self.lanes, float(a))
        assert a.shape == (self.lanes,)
        return a

    def _node(self, name: str) -> None:
        if name != "0" and name not in self.nodes:
            self.nodes[name] = -1

    def add(self, kind: int, terms: List[str], params: Sequence) -> None:
        for t in terms:
            self._node(t)
        p = np.stack([self._lane(v) for v in params])
        assert p.shape[0] == PARAMS[kind], (kind, p.shape)
        self.devs[kind].append((terms, p))

    def r(self, a, b, r):
        self.add(RES, [a, b], [r])

    def c(self, a, b, c):
        self.add(CAP, [a, b], [c])

    def d(self, a, c, is_=1e-14, n=1.0, cjo=0.0, vj=1.0, m=0.5, fc=0.5, tt=0.0):
        self.add(DIODE, [a, c], [is_, n, cjo, vj, m, fc, tt])

    def m(self, d, g, s, b, typ, vto, kp, w, l, gamma=0.0, phi=0.6, lam=0.0, is_=1e-14):
        self.add(MOS1, [d, g, s, b], [typ, vto, kp, gamma, phi, lam, is_, w, l])

    def v(self, p, n, dc=0.0, pulse=None, label=None, ac=None):
        """pulse = (v1, v2, td, tr, tf, pw, per); `label` names the source
        (its branch current is then Netlist.branch_names[label]); `ac` =
        (magnitude, phase in degrees) of its small-signal value."""
        name = f"#br{len(self.vsrc_names)}"
        self.vsrc_names.append(name)
        if ac is not None:
            self.ac.append(("v", name, float(ac[0]), float(ac[1])))
        if label is not None:
            self.vsrc_labels[label] = name
        self.add(VSRC, [p, n, name], _src_params(dc, pulse))

    def i(self, p, n, dc=0.0, pulse=None, ac=None):
        if ac is not None:
            self.ac.append(("i", p, n, float(ac[0]), float(ac[1])))
        self.add(ISRC, [p, n], _src_params(dc, pulse))

    def freeze(self, sweep: Optional[np.ndarray] = None) -> Netlist:
        # Unknown order: ground row 0, nodes in first-use order, branches.
        names = [k for k in self.nodes if not k.startswith("#br")]
        idx = {"0": GROUND}
        for i, k in enumerate(names):
            idx[k] = i + 1
        for j, k in enumerate(self.vsrc_names):
            idx[k] = len(names) + 1 + j
        n = len(names) + 1 + len(self.vsrc_names)
        cols: List[set] = [set([i]) for i in range(n)]
        batches = []
        cur = np.zeros(n, dtype=np.uint8)
        for kind in (RES, CAP, VSRC, ISRC, DIODE, MOS1):
            lst = self.devs[kind]
            if not lst:
                continue
            term = np.array([[idx[t] for t in ts] for ts, _ in lst], dtype=np.uint32)
            param = np.ascontiguousarray(np.stack([p for _, p in lst]))
            for row in term:
                for (rt, ct) in _STAMPS[kind]:
                    r, c = int(row[rt]), int(row[ct])
                    if r != GROUND and c != GROUND:
                        cols[c].add(r)
                if kind == VSRC:
                    cur[int(row[2])] = 1
            batches.append(Batch(kind, term, param))
        col_ptr = np.zeros(n + 1, dtype=np.uint32)
        rows: List[int] = []
        for c in range(n):
            rr = sorted(cols[c])
            rows.extend(rr)
            col_ptr[c + 1] = len(rows)
        node_names = {k: v for k, v in idx.items() if k != "0"}
        branches = {label: idx[br] for label, br in self.vsrc_labels.items()}
        acs = [("v", idx[a[1]], a[2], a[3]) if a[0] == "v" else ("i", idx[a[1]], idx[a[2]], a[3], a[4])
               for a in self.ac]
        return Netlist(self.name, n, col_ptr, np.array(rows, dtype=np.uint32), batches, self.lanes,
                       node_names, cur, sweep, branches, acs)


def _src_params(dc, pulse):
    if pulse is None:
        return [dc, 0.0, 0, 0, 0, 0, 0, 0, 0]
    v1, v2, td, tr, tf, pw, per = pulse
    return [dc, 1.0, v1, v2, td, tr, tf, pw, per]


# --------------------------------------------------------------------------
# Configurations

NMOS_KP, PMOS_KP = 200e-6, 80e-6
L_CH = 0.18e-6


def inverter_chain(points: int, stages: int = 16, base_seed: int = 1, vin: float = 0.9,
                   vdd: float = 1.8, cload: float = 10e-15, first_point: int = 0,
                   lam: float = 0.0) -> Netlist:
    """16-stage CMOS inverter chain, MOS level 1, Monte Carlo per point:
    VTO +-0.45 V + N(0, 20 mV) and KP x (1 + N(0, 5 %)) per device, NMOS W/L
    2/0.18 um, PMOS 4/0.18 um, 10 fF per stage, input at 0.9 V DC."""
    seeds = np.uint64(base_seed) + np.arange(first_point, first_point + points, dtype=np.uint64)
    b = Builder(f"inv_chain{stages}", points)
    b.v("vdd", "0", dc=vdd)
    b.v("in", "0", dc=vin)
    prev = "in"
    sweep = []
    for s in range(stages):
        out = f"s{s + 1}"
        dvn = 0.020 * mc_normal(seeds, 4 * s + 0)
        dkn = 0.05 * mc_normal(seeds, 4 * s + 1)
        dvp = 0.020 * mc_normal(seeds, 4 * s + 2)
        dkp = 0.05 * mc_normal(seeds, 4 * s + 3)
        b.m(out, prev, "0", "0", 1.0, 0.45 + dvn, NMOS_KP * (1 + dkn), 2e-6, L_CH, lam=lam)
        b.m(out, prev, "vdd", "vdd", -1.0, -0.45 + dvp, PMOS_KP * (1 + dkp), 4e-6, L_CH, lam=lam)
        b.c(out, "0", cload)
        sweep += [dvn, dkn, dvp, dkp]
        prev = out
    return b.freeze(np.stack(sweep, axis=1))


def miller_opamp(points: int, base_seed: int = 7, first_point: int = 0, vdd: float = 1.8,
                 vcm: float = 0.9, lam: float = 0.02) -> Netlist:
    """Two-stage Miller op-amp (8 MOS1, Cc = 1 pF) in unity-gain feedback,
    with 16 varied parameters: VTO ~ N(0, 15 mV) on all 8 devices, and on
    4 matched groups (input pair, mirror load, tail/sink/bias, second-stage
    PMOS) KP ~ N(0, 4 %) and W ~ N(0, 2 %)."""
    seeds = np.uint64(base_seed) + np.arange(first_point, first_point + points, dtype=np.uint64)
    b = Builder("miller_opamp", points)
    dv = [0.015 * mc_normal(seeds, k) for k in range(8)]
    dk = [0.04 * mc_normal(seeds, 8 + k) for k in range(4)]
    dw = [0.02 * mc_normal(seeds, 12 + k) for k in range(4)]
    b.v("vdd", "0", dc=vdd)
    b.v("inp", "0", dc=vcm)
    b.i("vdd", "vb", dc=20e-6)
    w_in, w_ld, w_t, w_2 = 4e-6, 4e-6, 4e-6, 16e-6
    L = 0.36e-6
    grp = [0, 0, 1, 1, 2, 3, 2, 2]  # device -> matched group
    def kp(i, base):
        return base * (1 + dk[grp[i]])
    def w(i, base):
        return base * (1 + dw[grp[i]])
    # input pair
    b.m("n1", "out", "tail", "0", 1.0, 0.45 + dv[0], kp(0, NMOS_KP), w(0, w_in), L, lam=lam)
    b.m("n2", "inp", "tail", "0", 1.0, 0.45 + dv[1], kp(1, NMOS_KP), w(1, w_in), L, lam=lam)
    # PMOS mirror load
    b.m("n1", "n1", "vdd", "vdd", -1.0, -0.45 + dv[2], kp(2, PMOS_KP), w(2, w_ld), L, lam=lam)
    b.m("n2", "n1", "vdd", "vdd", -1.0, -0.45 + dv[3], kp(3, PMOS_KP), w(3, w_ld), L, lam=lam)
    # tail source
    b.m("tail", "vb", "0", "0", 1.0, 0.45 + dv[4], kp(4, NMOS_KP), w(4, w_t), L, lam=lam)
    # second stage
    b.m("out", "n2", "vdd", "vdd", -1.0, -0.45 + dv[5], kp(5, PMOS_KP), w(5, w_2), L, lam=lam)
    b.m("out", "vb", "0", "0", 1.0, 0.45 + dv[6], kp(6, NMOS_KP), w(6, 2 * w_t), L, lam=lam)
    # bias diode
    b.m("vb", "vb", "0", "0", 1.0, 0.45 + dv[7], kp(7, NMOS_KP), w(7, w_t), L, lam=lam)
    b.c("n2", "out", 1e-12)
    b.c("out", "0", 1e-12)
    sweep = np.stack(dv + dk + dw, axis=1)
    return b.freeze(sweep)


def rc_diode_ladder(nodes: int, lanes: int, seed: int, jitter: float = 0.05, t_rise: float = 1e-9,
                    lane_seed0: int = 0) -> Netlist:
    """An RC-diode ladder of `nodes` nodes: R to the next node (log-uniform
    1 k - 100 k), C to ground (log-uniform 1 fF - 1 pF), and with
    probability 0.2 a diode to ground (IS 1e-14, N 1); a 0 -> 1 V PULSE with
    1 ns rise drives node 1 through the first resistor. Lanes share the
    pattern; each lane scales every R and C by a uniform factor in
    [1 - jitter, 1 + jitter] (seeded per lane)."""
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(math.log(1e3), math.log(1e5), nodes))
    c = np.exp(rng.uniform(math.log(1e-15), math.log(1e-12), nodes))
    has_d = rng.uniform(size=nodes) < 0.2
    lrng = np.random.default_rng(seed * 7919 + 17 + lane_seed0)
    jr = 1 + jitter * (2 * lrng.uniform(size=(nodes, lanes)) - 1)
    jc = 1 + jitter * (2 * lrng.uniform(size=(nodes, lanes)) - 1)
    b = Builder(f"rcd{nodes}_{seed}", lanes)
    b.v("src", "0", dc=0.0, pulse=(0.0, 1.0, 0.0, t_rise, t_rise, 1e-3, 2.1e-3))
    prev = "src"
    for k in range(nodes):
        nd = f"n{k + 1}"
        b.r(prev, nd, r[k] * jr[k])
        b.c(nd, "0", c[k] * jc[k])
        if has_d[k]:
            b.d(nd, "0")
        prev = nd
    return b.freeze()


def rc_diode_batch(n_nets: int = 64, lanes_per_net: int = 64, seed: int = 2024, min_nodes: int = 200,
                   max_nodes: int = 5000) -> List[Netlist]:
    """64 seeded ladders of 200-5,000 nodes (log-uniform), 64 lanes each."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(min_nodes), math.log(max_nodes), n_nets)).astype(int)
    return [rc_diode_ladder(int(sz), lanes_per_net, seed=seed * 1000 + i) for i, sz in enumerate(sizes)]


def ring_oscillator(points: int, stages: int = 31, base_seed: int = 11, first_point: int = 0,
                    vdd: float = 1.8, cload: float = 20e-15, kick: float = 100e-6) -> Netlist:
    """A ring of `stages` (odd) MOS1 inverters with chain-like Monte Carlo
    and 20 fF per stage. The ring starts from its DC operating point (all
    stages at the trip point); a 50 ps current pulse into stage 1 at
    t = 20 ps kicks it into oscillation (GPU lanes refuse uic and .ic, so the
    kick is a source)."""
    seeds = np.uint64(base_seed) + np.arange(first_point, first_point + points, dtype=np.uint64)
    b = Builder(f"ring{stages}", points)
    b.v("vdd", "0", dc=vdd)
    sweep = []
    for s in range(stages):
        inp = f"s{s}"
        out = f"s{(s + 1) % stages}"
        dvn = 0.020 * mc_normal(seeds, 4 * s + 0)
        dkn = 0.05 * mc_normal(seeds, 4 * s + 1)
        dvp = 0.020 * mc_normal(seeds, 4 * s + 2)
        dkp = 0.05 * mc_normal(seeds, 4 * s + 3)
        b.m(out, inp, "0", "0", 1.0, 0.45 + dvn, NMOS_KP * (1 + dkn), 2e-6, L_CH)
        b.m(out, inp, "vdd", "vdd", -1.0, -0.45 + dvp, PMOS_KP * (1 + dkp), 4e-6, L_CH)
        b.c(out, "0", cload)
        sweep += [dvn, dkn, dvp, dkp]
    b.i("0", "s1", dc=0.0, pulse=(0.0, kick, 20e-12, 10e-12, 10e-12, 50e-12, 1.0))
    return b.freeze(np.stack(sweep, axis=1))


def power_grid(lanes: int, side: int = 200, loads: int = 400, seed: int = 3, r_seg: float = 0.1,
               c_node: float = 10e-12) -> Netlist:
    """side x side resistive mesh (0.1 ohm x U(0.9, 1.1) per segment, per
    lane), 10 pF decap per node, 1 V pads at the four corners, and `loads`
    seeded current pulses (peak log-uniform 1-10 mA, width U(50, 500) ps)."""
    rng = np.random.default_rng(seed)
    b = Builder(f"grid{side}", lanes)
    def nm(i, j):
        return f"g{i}_{j}"
    for (i, j) in ((0, 0), (0, side - 1), (side - 1, 0), (side - 1, side - 1)):
        b.v(nm(i, j), "0", dc=1.0)
    lr = np.random.default_rng(seed + 101)
    for i in range(side):
        for j in range(side):
            if j + 1 < side:
                b.r(nm(i, j), nm(i, j + 1), r_seg * lr.uniform(0.9, 1.1, lanes))
            if i + 1 < side:
                b.r(nm(i, j), nm(i + 1, j), r_seg * lr.uniform(0.9, 1.1, lanes))
            b.c(nm(i, j), "0", c_node)
    pos = rng.choice(side * side, size=loads, replace=False)
    for k, p in enumerate(pos):
        i, j = divmod(int(p), side)
        peak = float(np.exp(rng.uniform(math.log(1e-3), math.log(1e-2))))
        width = float(rng.uniform(50e-12, 500e-12))
        td = float(rng.uniform(0, 500e-12))
        b.i(nm(i, j), "0", dc=0.0, pulse=(0.0, peak, td, 10e-12, 10e-12, width, 1.0))
    return b.freeze()


def inverter_pair(points: int, widths: Optional[Sequence[float]] = None) -> Netlist:
    """Two inverters in series with a .step over the NMOS W, the reference's
    GPU-vs-CPU tolerance deck shape (src/tests/espice.zig:3353-3389)."""
    if widths is None:
        widths = np.linspace(1e-6, 4e-6, points)
    w = np.asarray(widths, dtype=np.float64)
    b = Builder("inv_pair", points)
    b.v("vdd", "0", dc=1.8)
    b.v("in", "0", dc=0.7)
    b.m("mid", "in", "0", "0", 1.0, 0.45, NMOS_KP, w, L_CH, lam=0.02)
    b.m("mid", "in", "vdd", "vdd", -1.0, -0.45, PMOS_KP, 4e-6, L_CH, lam=0.02)
    b.m("out", "mid", "0", "0", 1.0, 0.45, NMOS_KP, w, L_CH, lam=0.02)
    b.m("out", "mid", "vdd", "vdd", -1.0, -0.45, PMOS_KP, 4e-6, L_CH, lam=0.02)
    return b.freeze(w[:, None])


def rc_points(points: int, r: Sequence[float], c: Sequence[float], tr: float = 1e-12) -> Netlist:
    """An RC low-pass driven by a pulse: the analytic-delay deck of the C
    API tests (src/tests/c_api.zig:795-821)."""
    b = Builder("rc", points)
    b.v("in", "0", dc=0.0, pulse=(0.0, 1.0, 0.0, tr, tr, 1.0, 2.0))
    b.r("in", "out", np.asarray(r, dtype=np.float64))
    b.c("out", "0", np.asarray(c, dtype=np.float64))
    return b.freeze()
