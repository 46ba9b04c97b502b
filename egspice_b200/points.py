"""The reference's points API (include/espice.h :244-362:
espice_append_points, espice_copy_point_measures, espice_release_points,
espice_lane_width) over the GPU lanes: one SPICE deck as a template, run at
many rows of its live parameters, each row a point whose `.meas tran`
measures and reason are copied back by query id.

Points run as lanes of one template per batch (at most `lane_width()` lanes,
the reference's GPU lane cap), in the order they were appended; a point's
measures depend only on the deck and its values up to the lanes' numerics,
not on which batch carried it. The deck's `.tran tstep tstop [tstart [tmax]]`
card sets the transient (tstart must be 0: the lanes record from t = 0);
every point has one query, its transient, so point k of an append has id
first_id + k. Errors raise PointsError carrying the reference's status code
and diagnostic name."""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Mapping, Optional, Sequence

import numpy as np

from . import abi
from .decks import RES
from .netlist import (DeckError, _logical_lines, _split, measure_passes, param_defaults, parse_number,
                      point_measures, read_deck, read_measures)

# espice_status (include/espice.h :33-37)
OK, INVALID_ARGUMENT, INVALID_QUERY, RESULT_UNAVAILABLE, FAILED = 0, 1, 4, 5, 6
# espice_reason (include/espice.h :260-284) for a point refused as appended
REASON_TOPOLOGY_CHANGED = 8
REASON_INVALID_PARAMETER = 9
LANE_WIDTH = 16384  # espice_lane_width under GPU lanes


class PointsError(RuntimeError):
    def __init__(self, status: int, name: str):
        super().__init__(f"{name} (status {status})")
        self.status, self.name = status, name


def _tran_card(text: str, allow_none: bool = False):
    """(tstep, tstop, tmax) of the deck's one .tran card, or None for a deck
    whose analyses are .op (or, with allow_none, .ac)."""
    found = None
    has_op = False
    for ln, card in _logical_lines(text):
        toks = _split(card)
        if toks[0] in (".step", ".data", ".alter"):
            raise PointsError(INVALID_ARGUMENT, "SweptTemplate")
        has_op |= toks[0] == ".op"
        if toks[0] != ".tran":
            continue
        if found is not None:
            raise DeckError(f"line {ln}: a second .tran card")
        nums = [t for t in toks[1:] if t != "uic"]
        if "uic" in toks[1:]:
            raise DeckError(f"line {ln}: UIC is refused on the lanes (as the reference's GPU lanes do)")
        vals = [parse_number(t) for t in nums]
        if len(vals) < 2 or any(v is None for v in vals):
            raise DeckError(f"line {ln}: .tran needs tstep and tstop as numbers")
        if len(vals) > 2 and vals[2] != 0:
            raise DeckError(f"line {ln}: a nonzero tstart is outside what the lanes carry")
        tmax = vals[3] if len(vals) > 3 else None
        found = (vals[0], vals[1], tmax)
    if found is None and not has_op and not allow_none:
        raise DeckError("the deck has neither a .tran nor an .op card")
    return found


def ac_frequencies(text: str) -> Optional[np.ndarray]:
    """The frequencies (Hz) of the deck's `.ac dec|oct|lin n fstart fstop`
    card as ngspice steps them (dec/oct: fstart times 10^(1/n) or 2^(1/n)
    repeatedly while at most fstop; lin: n points from fstart to fstop), or
    None without one."""
    found = None
    for ln, card in _logical_lines(text):
        toks = _split(card)
        if toks[0] != ".ac":
            continue
        if found is not None:
            raise DeckError(f"line {ln}: a second .ac card")
        vals = [parse_number(t) for t in toks[2:5]]
        if len(toks) != 5 or toks[1] not in ("dec", "oct", "lin") or any(v is None for v in vals):
            raise DeckError(f"line {ln}: .ac needs dec|oct|lin, a count, fstart and fstop")
        n, f0, f1 = int(vals[0]), vals[1], vals[2]
        if n < 1 or not (0 < f0 <= f1):
            raise DeckError(f"line {ln}: .ac needs a count from 1 and 0 < fstart <= fstop")
        if toks[1] == "lin":
            found = np.linspace(f0, f1, n)
        else:
            step = (10.0 if toks[1] == "dec" else 2.0) ** (1.0 / n)
            fs = [f0]
            while fs[-1] * step <= f1 * (1 + 1e-12):
                fs.append(fs[-1] * step)
            found = np.array(fs)
    return found


def ac_rhs(net) -> np.ndarray:
    """The small-signal excitation b of the deck's AC sources: a voltage
    source's branch row gets mag e^{j ph}; a current source from p to n adds
    -mag e^{j ph} at p and +mag e^{j ph} at n (it leaves p)."""
    from .decks import GROUND
    b = np.zeros(net.n, dtype=complex)
    for a in net.ac_sources:
        if a[0] == "v":
            b[a[1]] += a[2] * np.exp(1j * np.deg2rad(a[3]))
        else:
            v = a[3] * np.exp(1j * np.deg2rad(a[4]))
            if a[1] != GROUND:
                b[a[1]] -= v
            if a[2] != GROUND:
                b[a[2]] += v
    return b


def ac_measure_values(measures: Sequence, freqs: np.ndarray, z: np.ndarray) -> Dict[str, np.ndarray]:
    """Each `.meas ac` card's value per lane from the AC solution z
    [lanes, F, n] at `freqs`: its columns (magnitude, dB, phase, real or
    imaginary part of an unknown) over frequency through the lanes' measure
    passes on the host (espl_meas_table)."""
    from .lanes import meas_table
    out: Dict[str, np.ndarray] = {}
    forms = {"m": np.abs, "db": lambda v: 20.0 * np.log10(np.abs(v)), "p": np.angle, "r": np.real, "i": np.imag}
    for m in measures:
        if m.analysis != "ac":
            continue
        vals = np.full(z.shape[0], np.nan)
        with np.errstate(divide="ignore", invalid="ignore"):
            table = np.stack([forms[f](z[:, :, row]) for f, row in m.columns], axis=2)  # [lanes, F, cols]
        for l in range(z.shape[0]):
            v, _ = meas_table(m.passes, freqs, table[l])
            vals[l] = v[0] - v[1] if m.pp else v[-1]
        out[m.name] = vals
    return out


class Points:
    """A deck `text` as a points template over `live_params` (names of the
    deck's parameters each point gives values for; the others keep their
    .param values). `precision` as Lanes takes it; `tran` overrides fields
    of the transient options (abi.tran_opts keywords). TMAX defaults to
    ngspice's min(TSTEP, TSTOP / 50). A measure may read parameters, but no
    live one: a template's measure passes are the same on every lane.
    `early_stop` (espice_points_options.early_stop) ends each point's
    transient once all its measure passes have resolved. A
    deck with .op and no .tran runs operating points (the continuation
    ladder), which `.meas op ... find` cards read; in a .tran deck they read
    the operating point solved the same way before the transient."""

    def __init__(self, text: str, live_params: Sequence[str], precision: str = "fp64",
                 tran: Optional[Mapping[str, float]] = None, early_stop: bool = False, device: Optional[int] = None):
        self.text = text
        # the GPU this process runs its points on (default: LOCAL_RANK under torchrun, else 0)
        self.device = int(os.environ.get("LOCAL_RANK", "0")) if device is None else device
        self.early_stop = early_stop
        self.live = [p.lower() for p in live_params]
        self.precision = precision
        self.freqs = ac_frequencies(text)
        card = _tran_card(text, allow_none=self.freqs is not None)
        self.topts = None
        if card is not None:
            tstep, tstop, tmax = card
            kw = dict(t_stop=tstop, dt=tstep, dt_max=tmax if tmax else min(tstep, tstop / 50))
            kw.update(tran or {})
            self.topts = abi.tran_opts(**kw)
        # the measures are read once on a two-lane instance of the template
        # whose live values differ, so a card that names no vector, or reads
        # a live parameter, fails here
        probe_params = {p: np.array([0.0, 1.0]) for p in self.live}
        probe = read_deck(text, lanes=2, params=probe_params)
        self.measures = read_measures(text, probe, params=probe_params)
        if self.topts is None and measure_passes(self.measures):
            raise DeckError("a .meas tran card needs the deck's .tran card")
        if any(m.analysis == "ac" for m in self.measures) and self.freqs is None:
            raise DeckError("a .meas ac card needs the deck's .ac card")
        if self.freqs is not None and not probe.ac_sources:
            raise DeckError("the .ac analysis needs a source with an AC value")
        self.need_op = (self.topts is None or self.freqs is not None
                        or any(m.op_row is not None for m in self.measures))
        # The lead lane of every batch, whose matrix gives the batch's pivot
        # tape: the deck's own .param values of the live parameters when it
        # gives them all. Each batch then replays the same tape, and a lane's
        # arithmetic reads only its own values, so a point's results are
        # bitwise the same in any order, batch or rank split (the points
        # API's promise, include/espice.h:246-250). Without them the first
        # point of each batch leads, and results agree to roundoff only.
        d = param_defaults(text, self.live)
        self.lead = None if d is None else np.array([d[p] for p in self.live])
        self.rows: List[np.ndarray] = []     # each point's values
        self.state: List[int] = []           # 0 pending, 1 complete, 2 released
        self.values: Dict[int, np.ndarray] = {}
        self.reasons: Dict[int, int] = {}

    @staticmethod
    def lane_width() -> int:
        return LANE_WIDTH

    def append_points(self, values) -> int:
        """Appends count points (values [count][len(live_params)]); returns
        point 0's query id. A point with a non-finite value is appended
        already failed (INVALID_PARAMETER), as is one whose values short a
        resistor (TOPOLOGY_CHANGED: a zero resistance collapses two nodes,
        which the template's pattern cannot)."""
        if not self.live:
            raise PointsError(INVALID_ARGUMENT, "NoLiveParameters")
        v = np.asarray(values, dtype=np.float64)
        if v.ndim != 2 or v.shape[0] == 0 or v.shape[1] != len(self.live):
            raise PointsError(INVALID_ARGUMENT, "InvalidArgument")
        first = len(self.rows)
        finite = np.isfinite(v).all(axis=1)
        shorted = np.zeros(len(v), dtype=bool)
        if finite.any():
            net = read_deck(self.text, lanes=len(v), params={p: np.where(finite, v[:, j], 1.0)
                                                             for j, p in enumerate(self.live)})
            for b in net.batches:
                if b.kind == RES:
                    shorted |= (b.param[:, 0, :] == 0).any(axis=0)
        for i, row in enumerate(v):
            self.rows.append(row.copy())
            reason = REASON_INVALID_PARAMETER if not finite[i] else REASON_TOPOLOGY_CHANGED if shorted[i] else None
            if reason is None:
                self.state.append(0)
            else:
                k = len(self.rows) - 1
                self.state.append(1)
                self.values[k] = np.full(len(self.measures), np.nan)
                self.reasons[k] = reason
        return first

    def batches(self, ids: Sequence[int]) -> List[List[int]]:
        """The lane batches of the points `ids` as one process runs them:
        consecutive runs of lane_width() lanes, one of them the lead lane
        when the deck gives the live parameters' values."""
        per = LANE_WIDTH - (1 if self.lead is not None else 0)
        return [list(ids[b0:b0 + per]) for b0 in range(0, len(ids), per)]

    def rank_batches(self, pending: Sequence[int], rank: int, world: int) -> List[List[int]]:
        """Rank `rank`'s share of the one-process batches: contiguous whole
        batches, so every batch keeps its members (and lead) at any world
        size."""
        bs = self.batches(pending)
        per = -(-len(bs) // world) if bs else 0
        return bs[rank * per:(rank + 1) * per]

    def run(self, group=None) -> None:
        """Runs every pending point on the GPU lanes, lane_width() at a time.
        Under torch.distributed (one process per GPU), the one-process lane
        batches split into contiguous runs of whole batches, one per rank of
        `group`, each rank runs its batches on its own GPU, and every rank
        receives every result (no collective touches the lanes: the exchange
        is of finished results)."""
        pending = [k for k, s in enumerate(self.state) if s == 0]
        rank, world, dist = 0, 1, None
        td = sys.modules.get("torch.distributed")  # a process group needs torch imported already
        if td is not None and td.is_available() and td.is_initialized():
            dist, rank, world = td, td.get_rank(group), td.get_world_size(group)
            if rank < 0:
                raise PointsError(INVALID_ARGUMENT, "NotInProcessGroup")
        results = {}
        for batch in self.rank_batches(pending, rank, world):
            results.update(self._run_ids(batch))
        parts = [results]
        if world > 1:
            if td.get_backend(group) == "nccl":
                # all_gather_object stages its tensors on the current device
                import torch
                torch.cuda.set_device(self.device)
            parts = [None] * world
            dist.all_gather_object(parts, results, group=group)
        for part in parts:
            for k, (values, reason) in part.items():
                self.values[k] = np.asarray(values, dtype=np.float64)
                self.reasons[k] = int(reason)
                self.state[k] = 1

    def _run_ids(self, ids: Sequence[int]) -> Dict[int, tuple]:
        """{id: (measure values in card order, reason)} of the points `ids`,
        run as lane batches of at most lane_width() on this process's GPU."""
        from .lanes import Lanes
        names = [m.name for m in self.measures]
        done: Dict[int, tuple] = {}
        lead = 1 if self.lead is not None else 0
        for batch in self.batches(ids):
            block = np.stack(([self.lead] if lead else []) + [self.rows[k] for k in batch])
            params = {p: block[:, j] for j, p in enumerate(self.live)}
            net = read_deck(self.text, lanes=len(block), params=params)
            ms = read_measures(self.text, net, params=params)
            op = x_op = reps = ac = None
            value = np.zeros((len(block), 0))
            with Lanes([net], precision=self.precision, device=self.device) as L:
                if self.need_op:
                    op = L.solve_op(abi.newton_opts())
                    x_op = L.get_x(0)
                if self.topts is not None:
                    passes = measure_passes(ms)
                    L.set_meas(0, passes)
                    if self.early_stop and passes:
                        reps = self._run_early_stop(L)
                    else:
                        reps = L.run_tran(self.topts, steps_per_launch=2048)
                    value, _ = L.get_meas(0)
                if self.freqs is not None:
                    # the AC sweep at the operating point solve_op left in x
                    L.put_x(0, x_op, False)
                    z = L.ac_solve(0, 2 * np.pi * self.freqs, ac_rhs(net)[None, :], np.arange(net.n))[:, :, 0, :]
                    ac = ac_measure_values(ms, self.freqs, z)
            out, reasons = point_measures(ms, value, names, reports=reps, op=op, x_op=x_op,
                                          stopped_ok=self.early_stop, ac=ac)
            for i, k in enumerate(batch):
                done[k] = (out[lead + i], int(reasons[lead + i]))
        return done

    def _run_early_stop(self, L, steps_per_launch: int = 512, max_launches: int = 100000):
        """The transient in launches of `steps_per_launch` steps; between
        launches every lane whose passes have all resolved is stopped."""
        L.init_steps(self.topts)
        reps = None
        for _ in range(max_launches):
            reps = L.device_launch(steps_per_launch)
            if all(r.status != 0 for r in reps):
                break
            done = L.meas_done(0).all(axis=1)
            if done.any():
                L.request_stop(0, done)
        return reps

    def copy_point_measures(self, first_id: int, count: int, names: Sequence[str]):
        """(values [count][len(names)], reasons [count]) of the points from
        first_id; names case-insensitive."""
        if count < 1 or first_id < 0 or first_id + count > len(self.rows):
            raise PointsError(INVALID_QUERY, "InvalidQuery")
        keys = {m.name.lower(): j for j, m in enumerate(self.measures)}
        cols = []
        for nm in names:
            if nm.lower() not in keys:
                raise PointsError(INVALID_ARGUMENT, "UnknownMeasure")
            cols.append(keys[nm.lower()])
        ids = range(first_id, first_id + count)
        if any(self.state[k] != 1 for k in ids):
            raise PointsError(RESULT_UNAVAILABLE, "ResultUnavailable")
        out = np.stack([self.values[k][cols] for k in ids])
        reasons = np.array([self.reasons[k] for k in ids], dtype=np.uint32)
        return out, reasons

    def release_points(self, first_id: int, count: int) -> None:
        """Frees the results of count points from first_id; copying them
        afterwards is RESULT_UNAVAILABLE."""
        if count < 1 or first_id < 0 or first_id + count > len(self.rows):
            raise PointsError(INVALID_QUERY, "InvalidQuery")
        for k in range(first_id, first_id + count):
            if self.state[k] == 1:
                self.state[k] = 2
                self.values.pop(k, None)
                self.reasons.pop(k, None)
