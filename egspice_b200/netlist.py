"""A reader for the SPICE decks the lane sweep runs (ngspice syntax).

The front end on the input side of the path: deck text in, the frozen MNA
pattern and per-kind device batches out (what the reference gets from
src/frontend/netlist.zig `parse` and `Circuit.freeze`), as an
`egspice_b200.decks.Netlist` that `Lanes` takes directly. It reads the subset
the lanes carry:

* R, C            ``Rname n1 n2 value``
* V, I            ``Vname n+ n- [DC] value [PULSE(v1 v2 td tr tf pw per)] [AC mag [phase]]``
* D               ``Dname anode cathode model``
* M (level 1)     ``Mname d g s b model [W=value] [L=value]``
* ``.model name nmos|pmos|d (params)`` — MOS: LEVEL=1, VTO, KP, GAMMA, PHI,
  LAMBDA, IS (TOX, RD, RS must be absent or zero: the lanes carry no Meyer
  capacitances and no series resistances); diode: IS, N, CJO, VJ, M, FC, TT
  (RS absent or zero)
* ``.param name=value``; values anywhere may be numbers with SPICE scale
  suffixes (t g meg k m u n p f a mil), parameter names, or ``{expression}``
  over numbers, parameters, + - * / ** and parentheses
* ``+`` continuation lines, ``*`` comment lines, ``;`` and ``$ `` inline
  comments; the first line is the title; ``.end`` ends the deck; analysis
  cards (.op .tran .ac .dc .option .options .temp .print .save .probe) are
  accepted and ignored (the caller runs the analysis through the API;
  egspice_b200.points reads .op, .tran and .ac); ``.meas tran``, ``.meas
  ac`` and ``.meas op`` cards are read by `read_measures`.

Per-lane values: `params` maps parameter names to a scalar or to an array of
one value per lane (a Monte Carlo draw or a sweep); they override `.param`
cards, and any expression that reads one becomes per-lane. The arrays also
form the netlist's sweep matrix (the learned warm start's inputs), in the
order given. Numbers read as ngspice's INPevaluate reads them (every digit
into one mantissa, then times a correctly rounded power of ten), so a value
is bit for bit the value the reference parses from the same text. Anything
outside the subset raises `DeckError` naming the line.
"""
from __future__ import annotations

import ast
import dataclasses
import math
import operator
import re
from typing import Dict, List, Mapping, Optional, Sequence, Union

import numpy as np

from . import abi
from .decks import Builder, Netlist

Value = Union[float, np.ndarray]


class DeckError(ValueError):
    pass


_SCALE = {"t": 12, "g": 9, "k": 3, "m": -3, "u": -6, "n": -9, "p": -12, "f": -15, "a": -18}
_NUM = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][+-]?\d+)?")


def _pow10(e: int) -> float:
    """10**e as the C library's pow(10, e) gives it to ngspice: correctly
    rounded except at e = 23 and 210, which it rounds up; 0 below 1e-330 and
    inf past 1e308."""
    if e < -330:
        return 0.0
    if e > 308:
        return float("inf")
    v = float(f"1e{e}")
    return math.nextafter(v, math.inf) if e in (23, 210) else v


def parse_number(text: str) -> Optional[float]:
    """A SPICE number with its scale suffix (``10meg``, ``2.5u``, ``1mil``),
    or None when `text` does not start with a number. The digits go into one
    mantissa and the value is sign * mantissa * 10**exponent, as ngspice's
    INPevaluate computes it (so ``0.1n`` is 1e-10 exactly as ngspice reads
    it, not 0.1 * 1e-9)."""
    t = text.strip().lower()
    m = _NUM.match(t)
    if not m:
        return None
    lit, rest = m.group(0), t[m.end():]
    if rest.startswith("meg"):
        scale, mil = 6, False
    elif rest.startswith("mil"):
        scale, mil = -6, True
    else:
        scale, mil = (_SCALE.get(rest[0], 0) if rest else 0), False
    sign = -1.0 if lit.startswith("-") else 1.0
    body = lit.lstrip("+-")
    mant, exp = body, 0
    for sep in "ed":
        if sep in mant:
            mant, ex = mant.split(sep)
            exp = int(ex)
    e = scale + exp
    digits = mant
    if "." in mant:
        a, b = mant.split(".")
        digits = a + b
        e -= len(b)
    mantissa = 0.0
    for ch in digits:
        mantissa = 10.0 * mantissa + float(ord(ch) - 48)
    if mil:
        mantissa *= 25.4
    if mantissa == 0.0:
        return sign * 0.0
    return sign * mantissa * _pow10(e)


_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.Pow: operator.pow}


class _Env:
    def __init__(self, lanes: int, params: Mapping[str, Value]):
        self.lanes = lanes
        self.vals: Dict[str, Value] = {}
        for k, v in params.items():
            a = np.asarray(v, dtype=np.float64)
            if a.ndim == 0:
                self.vals[k.lower()] = float(a)
            elif a.shape == (lanes,):
                self.vals[k.lower()] = a
            else:
                raise DeckError(f"parameter {k}: {a.shape[0]} values for {lanes} lanes")
        self.given = set(self.vals)

    def value(self, text: str, where: str) -> Value:
        t = text.strip()
        if t.startswith("{") and t.endswith("}"):
            return self.expr(t[1:-1], where)
        if t.startswith("'") and t.endswith("'"):
            return self.expr(t[1:-1], where)
        m = _NUM.match(t.lower())
        if m and re.fullmatch(r"[a-z]*", t.lower()[m.end():]):
            return parse_number(t)
        name = t.lower()
        if name in self.vals:
            return self.vals[name]
        raise DeckError(f"{where}: cannot read the value {text!r}")

    def expr(self, text: str, where: str) -> Value:
        # every number literal (with its scale suffix) reads as parse_number reads it
        src = re.sub(r"(?<![\w.])(?:\d+\.?\d*|\.\d+)(?:e[+-]?\d+)?(?:meg|mil|[tgkmunpfa](?![a-z_0-9]))?",
                     lambda m: repr(parse_number(m.group(0))), text.lower())
        try:
            tree = ast.parse(src, mode="eval")
        except SyntaxError:
            raise DeckError(f"{where}: cannot parse the expression {{{text}}}") from None

        def ev(n):
            if isinstance(n, ast.Expression):
                return ev(n.body)
            if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
                return float(n.value)
            if isinstance(n, ast.Name):
                if n.id in self.vals:
                    return self.vals[n.id]
                raise DeckError(f"{where}: unknown parameter {n.id!r}")
            if isinstance(n, ast.BinOp) and type(n.op) in _BINOPS:
                return _BINOPS[type(n.op)](ev(n.left), ev(n.right))
            if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
                v = ev(n.operand)
                return -v if isinstance(n.op, ast.USub) else v
            raise DeckError(f"{where}: unsupported expression {{{text}}}")

        return ev(tree)


def _logical_lines(text: str) -> List[tuple]:
    """(line number, text) of each card: continuations joined, comments cut,
    lower case; the title line dropped."""
    raw = text.splitlines()
    out: List[list] = []
    for k, line in enumerate(raw[1:], start=2):
        s = line.strip()
        if not s or s.startswith("*"):
            continue
        for cut in (";", "$ "):
            i = s.find(cut)
            if i >= 0:
                s = s[:i].rstrip()
        if not s:
            continue
        if s.startswith("+"):
            if not out:
                raise DeckError(f"line {k}: continuation with nothing to continue")
            out[-1][1] += " " + s[1:].strip().lower()
        else:
            out.append([k, s.lower()])
    return [tuple(x) for x in out]


def _split(card: str) -> List[str]:
    """Tokens of a card: spaces separate, `=` binds, braces, parentheses
    and single quotes keep their contents together."""
    card = re.sub(r"\s*=\s*", "=", card)
    toks, cur, depth, quoted = [], "", 0, False
    for ch in card:
        if ch == "'":
            quoted = not quoted
        elif ch in "{(":
            depth += 1
        elif ch in "})":
            depth -= 1
        if (ch.isspace() or ch == ",") and depth == 0 and not quoted:
            if cur:
                toks.append(cur)
            cur = ""
        else:
            cur += ch
    if cur:
        toks.append(cur)
    return toks


_IGNORED = {".op", ".tran", ".ac", ".dc", ".option", ".options", ".temp", ".meas", ".measure", ".print", ".save",
            ".probe", ".plot", ".control", ".endc", ".title"}
_MOS_DEFAULTS = dict(level=1.0, vto=0.0, kp=2e-5, gamma=0.0, phi=0.6, lambda_=0.0, is_=1e-14, tox=0.0, rd=0.0,
                     rs=0.0)
_DIODE_DEFAULTS = dict(is_=1e-14, n=1.0, cjo=0.0, vj=1.0, m=0.5, fc=0.5, tt=0.0, rs=0.0)


def _kv(tokens: Sequence[str], where: str) -> Dict[str, str]:
    out = {}
    flat: List[str] = []
    for t in tokens:
        if t.startswith("(") and t.endswith(")"):
            flat += _split(t[1:-1])  # a parenthesized parameter list
        else:
            flat.append(t)
    for t in flat:
        t = t.strip("()")
        if not t:
            continue
        if "=" not in t:
            raise DeckError(f"{where}: expected name=value, got {t!r}")
        k, v = t.split("=", 1)
        out[k] = v
    return out


_NODE_TOKENS = {"r": 2, "c": 2, "d": 2, "v": 2, "i": 2, "m": 4}


def _expand_subckts(cards: List[tuple]) -> List[tuple]:
    """Flattens `.subckt name ports ... .ends` definitions and their `x`
    instances (nested to any depth): an instance's cards get its ports for
    the definition's port names, `inst.node` for the definition's own nodes
    (ngspice's naming, so v(x1.y) reads an internal node) and `head.inst`
    for element names; the ground stays global. Subcircuit parameters are
    outside what the lanes carry."""
    defs: Dict[str, tuple] = {}
    top: List[tuple] = []
    stack: List[list] = []
    for ln, card in cards:
        toks = _split(card)
        if toks[0] == ".subckt":
            if len(toks) < 2:
                raise DeckError(f"line {ln}: .subckt needs a name")
            if any("=" in t or t == "params:" for t in toks[2:]):
                raise DeckError(f"line {ln}: subcircuit parameters are outside what the lanes carry")
            stack.append([toks[1], toks[2:], [], ln])
        elif toks[0] == ".ends":
            if not stack:
                raise DeckError(f"line {ln}: .ends without .subckt")
            name, ports, body, _ = stack.pop()
            defs[name] = (ports, body)
        elif stack:
            stack[-1][2].append((ln, card))
        else:
            top.append((ln, card))
    if stack:
        raise DeckError(f"line {stack[-1][3]}: .subckt {stack[-1][0]} has no .ends")

    def expand(body: List[tuple], inst: str, nodes: Dict[str, str], depth: int) -> List[tuple]:
        if depth > 32:
            raise DeckError("subcircuits nest deeper than 32 (a recursive definition?)")
        out: List[tuple] = []
        for ln, card in body:
            toks = _split(card)
            head = toks[0]
            rename = (lambda t: t if t in ("0", "gnd") else nodes.get(t, f"{inst}.{t}")) if inst else (lambda t: t)
            if head.startswith("."):
                if inst:
                    raise DeckError(f"line {ln}: the card {head} inside a subcircuit is outside what the lanes carry")
                out.append((ln, card))
                continue
            if head[0] == "x":
                args = [t for t in toks[1:] if "=" not in t]
                if len(args) < 1 or len(args) < len(toks) - 1:
                    raise DeckError(f"line {ln}: instance parameters of a subcircuit are outside what the lanes carry")
                sub = args[-1]
                if sub not in defs:
                    raise DeckError(f"line {ln}: unknown subcircuit {sub!r}")
                ports, sbody = defs[sub]
                conn = [rename(t) for t in args[:-1]]
                if len(conn) != len(ports):
                    raise DeckError(f"line {ln}: {sub} takes {len(ports)} nodes, given {len(conn)}")
                path = f"{inst}.{head}" if inst else head  # x1.x2: x2 inside x1
                out += expand(sbody, path, dict(zip(ports, conn)), depth + 1)
                continue
            k = _NODE_TOKENS.get(head[0])
            if k is None or not inst:
                out.append((ln, card))
                continue
            toks = [f"{head}.{inst}"] + [rename(t) for t in toks[1:1 + k]] + toks[1 + k:]
            out.append((ln, " ".join(toks)))
        return out

    return expand(top, "", {}, 0) if defs or any(_split(c)[0][0] == "x" for _, c in top) else top


def _read_params(cards: Sequence[tuple], env: _Env) -> None:
    """The .param cards into `env`, values given by the caller kept."""
    for ln, card in cards:
        toks = _split(card)
        if toks[0] == ".param":
            where = f"line {ln}"
            for k, v in _kv(toks[1:], where).items():
                if k not in env.given:
                    env.vals[k] = env.value(v, where)


def param_defaults(text: str, names: Sequence[str]) -> Optional[Dict[str, float]]:
    """The deck's own `.param` values of `names` (lower-cased keys), or
    None when the deck does not give every one of them a single value."""
    env = _Env(1, {})
    _read_params(_expand_subckts(_logical_lines(text)), env)
    out = {}
    for k in names:
        v = env.vals.get(k.lower())
        if v is None or np.ndim(v) != 0 or not np.isfinite(v):
            return None
        out[k.lower()] = float(v)
    return out


def read_deck(text: str, lanes: int = 1, params: Optional[Mapping[str, Value]] = None,
              name: Optional[str] = None) -> Netlist:
    """The deck `text` as a Netlist of `lanes` lanes; `params` gives
    parameter values (scalars or one per lane) that override `.param`."""
    if lanes < 1:
        raise DeckError("a deck needs at least one lane")
    params = dict(params or {})
    env = _Env(lanes, params)
    cards = _expand_subckts(_logical_lines(text))
    title = text.splitlines()[0].strip() if text.strip() else "deck"
    _read_params(cards, env)
    # .model next (SPICE cards are order-free)
    models: Dict[str, tuple] = {}
    for ln, card in cards:
        toks = _split(card)
        where = f"line {ln}"
        if toks[0] == ".model":
            if len(toks) < 3:
                raise DeckError(f"{where}: .model needs a name and a type")
            mtype = toks[2].split("(")[0]
            rest = [toks[2][len(mtype):]] + toks[3:]
            models[toks[1]] = (mtype, rest, where)
    b = Builder(name or title, lanes)
    node = lambda t: "0" if t in ("0", "gnd") else t  # noqa: E731

    def model_vals(mname: str, kinds: Sequence[str], defaults: dict, where: str) -> tuple:
        if mname not in models:
            raise DeckError(f"{where}: unknown model {mname!r}")
        mtype, rest, mwhere = models[mname]
        if mtype not in kinds:
            raise DeckError(f"{where}: model {mname!r} is a {mtype}, not a {'/'.join(kinds)}")
        vals = dict(defaults)
        for k, v in _kv(rest, mwhere).items():
            key = {"lambda": "lambda_", "is": "is_"}.get(k, k)
            if key not in vals:
                raise DeckError(f"{mwhere}: model parameter {k!r} is outside what the lanes carry")
            vals[key] = env.value(v, mwhere)
        return mtype, vals

    def source(toks: List[str], where: str) -> tuple:
        dc, pulse, ac = 0.0, None, None
        i = 0
        while i < len(toks):
            t = toks[i]
            if t == "dc":
                dc = env.value(toks[i + 1], where)
                i += 2
            elif t == "ac":
                # AC magnitude [phase in degrees], the same on every lane
                vals = []
                for u in toks[i + 1:i + 3]:
                    if parse_number(u) is None and u not in env.vals and not u.startswith(("{", "'")):
                        break
                    vals.append(_scalar(env, u, where))
                ac = (vals[0] if vals else 1.0, vals[1] if len(vals) > 1 else 0.0)
                i += 1 + len(vals)
            elif t.startswith("pulse"):
                body = t[len("pulse"):].strip()
                if not body.startswith("("):
                    body = " ".join(toks[i + 1:])
                    i = len(toks)
                else:
                    i += 1
                vals = [env.value(v, where) for v in _split(body.strip("()"))]
                if len(vals) != 7:
                    raise DeckError(f"{where}: PULSE needs all seven values (v1 v2 td tr tf pw per)")
                pulse = tuple(vals)
            elif t.startswith(("sin", "exp", "pwl", "sffm", "am")):
                raise DeckError(f"{where}: only DC and PULSE sources (and an AC value) ride the lanes")
            else:
                dc = env.value(t, where)
                i += 1
        return dc, pulse, ac

    for ln, card in cards:
        toks = _split(card)
        where = f"line {ln}"
        head = toks[0]
        if head.startswith("."):
            if head in (".param", ".model") or head in _IGNORED:
                continue
            if head == ".end":
                break
            raise DeckError(f"{where}: the card {head} is outside what the lanes carry")
        kind = head[0]
        if kind == "r":
            if len(toks) != 4:
                raise DeckError(f"{where}: R needs two nodes and a value")
            b.r(node(toks[1]), node(toks[2]), env.value(toks[3], where))
        elif kind == "c":
            if len(toks) != 4:
                raise DeckError(f"{where}: C needs two nodes and a value")
            b.c(node(toks[1]), node(toks[2]), env.value(toks[3], where))
        elif kind in "vi":
            if len(toks) < 3:
                raise DeckError(f"{where}: a source needs two nodes")
            dc, pulse, ac = source(toks[3:], where)
            if kind == "v":
                b.v(node(toks[1]), node(toks[2]), dc=dc, pulse=pulse, label=head, ac=ac)
            else:
                b.i(node(toks[1]), node(toks[2]), dc=dc, pulse=pulse, ac=ac)
        elif kind == "d":
            if len(toks) != 4:
                raise DeckError(f"{where}: D needs two nodes and a model")
            _, m = model_vals(toks[3], ("d",), _DIODE_DEFAULTS, where)
            if np.any(np.asarray(m["rs"]) != 0):
                raise DeckError(f"{where}: diode series resistance is outside what the lanes carry")
            b.d(node(toks[1]), node(toks[2]), is_=m["is_"], n=m["n"], cjo=m["cjo"], vj=m["vj"], m=m["m"],
                fc=m["fc"], tt=m["tt"])
        elif kind == "m":
            if len(toks) < 6:
                raise DeckError(f"{where}: M needs four nodes and a model")
            mtype, m = model_vals(toks[5], ("nmos", "pmos"), _MOS_DEFAULTS, where)
            if np.any(np.asarray(m["level"]) != 1):
                raise DeckError(f"{where}: only level-1 MOS models ride the lanes")
            for k in ("tox", "rd", "rs"):
                if np.any(np.asarray(m[k]) != 0):
                    raise DeckError(f"{where}: MOS {k.upper()} is outside what the lanes carry")
            inst = _kv(toks[6:], where)
            w = env.value(inst.pop("w"), where) if "w" in inst else 1e-4
            l_ = env.value(inst.pop("l"), where) if "l" in inst else 1e-4
            if inst:
                raise DeckError(f"{where}: instance parameters {sorted(inst)} are outside what the lanes carry")
            typ = 1.0 if mtype == "nmos" else -1.0
            b.m(node(toks[1]), node(toks[2]), node(toks[3]), node(toks[4]), typ, m["vto"], m["kp"], w, l_,
                gamma=m["gamma"], phi=m["phi"], lam=m["lambda_"], is_=m["is_"])
        else:
            raise DeckError(f"{where}: the element {head!r} is outside what the lanes carry")
    arrays = [np.asarray(v, dtype=np.float64) for k, v in params.items() if np.ndim(v) == 1]
    sweep = np.stack(arrays, axis=1) if arrays else None
    return b.freeze(sweep)


# ---------------------------------------------------------------------------
# .meas tran cards -> the lanes' streaming measure passes (espl_meas)


@dataclasses.dataclass
class Measure:
    """One `.meas` card: its name, the consecutive passes that compute it
    (`.meas tran`), and how its value comes out of them: the last pass's
    value, or (PP) the first pass's (MAX) minus the second's (MIN). A
    `.meas op ... find vec` card has no passes and reads unknown `op_row`
    of the operating point; a `.meas tran name param='expr'` card has none
    either and evaluates `expr` over the parameters (`params`, as read with
    the deck) and the measures before it."""
    name: str
    passes: List[abi.MeasPass]
    pp: bool = False
    op_row: Optional[int] = None
    expr: Optional[str] = None
    params: Optional[Dict[str, Value]] = None
    # `.meas ac`: its passes read `columns`, each (form, unknown) with form
    # m (magnitude), db (20 log10 |.|), p (phase, radians), r or i (real or
    # imaginary part) of the AC solution over frequency.
    analysis: str = "tran"
    columns: Optional[List[tuple]] = None


_COUNTS = ("rise", "fall", "cross")


def _vector(tok: str, net: Netlist, where: str) -> int:
    """The unknown a waveform token reads: v(node) or i(vsource)."""
    m = re.fullmatch(r"([vi])\(([^(),]+)\)", tok)
    if not m:
        raise DeckError(f"{where}: the measure reads {tok!r}; only v(node) and i(vsource) ride the lanes")
    kind, name = m.group(1), m.group(2).strip()
    if kind == "v":
        if name in ("0", "gnd"):
            raise DeckError(f"{where}: v(0) is the ground")
        if name not in net.node_names:
            raise DeckError(f"{where}: no node {name!r}")
        return net.node_names[name]
    if name not in net.branch_names:
        raise DeckError(f"{where}: no voltage source {name!r} for i({name})")
    return net.branch_names[name]


def _scalar(env: _Env, text: str, where: str) -> float:
    v = env.value(text, where)
    if np.ndim(v) != 0:
        raise DeckError(f"{where}: a measure's {text!r} must be the same on every lane")
    return float(v)


def _clause(toks: List[str], net: Netlist, env: _Env, where: str, opts_ok: Sequence[str]) -> Dict[str, object]:
    """Options name=value of one clause (rise/fall/cross as counts or LAST,
    the others as scalars); a bare `last` is RISE/FALL/CROSS=LAST's shorthand
    for CROSS."""
    out: Dict[str, object] = {}
    for t in toks:
        if t == "last":
            out["cross"] = abi.MEAS_LAST
            continue
        if "=" not in t:
            raise DeckError(f"{where}: unexpected {t!r} in a .meas card")
        k, v = t.split("=", 1)
        if k not in opts_ok:
            raise DeckError(f"{where}: the .meas option {k.upper()} is outside what the lanes carry")
        if k in _COUNTS:
            if v == "last":
                out[k] = abi.MEAS_LAST
            else:
                c = _scalar(env, v, where)
                if c != int(c) or c < 1:
                    raise DeckError(f"{where}: {k.upper()}={v} must be a count from 1 or LAST")
                out[k] = int(c)
        else:
            out["from_" if k == "from" else k] = _scalar(env, v, where)
    if sum(k in out for k in _COUNTS) > 1:
        raise DeckError(f"{where}: give one of RISE, FALL, CROSS")
    return out


def _when(test: str, net: Netlist, env: _Env, where: str, vec=None) -> Dict[str, object]:
    """`vec=value` or `vec=vec2` of a WHEN: the pass's row and its level;
    `vec` resolves a vector token (default: an unknown of `net`)."""
    vec = vec or (lambda t: _vector(t, net, where))
    if "=" not in test:
        raise DeckError(f"{where}: WHEN needs vector=value")
    lhs, rhs = test.split("=", 1)
    row = vec(lhs)
    if re.fullmatch(r"[a-z]+\([^()]*\)", rhs):
        return {"row": row, "level_row": vec(rhs)}
    return {"row": row, "val": _scalar(env, rhs, where)}


def _measure(name: str, func: str, rest: List[str], net: Netlist, env: _Env, where: str, vec=None) -> Measure:
    vec = vec or (lambda t: _vector(t, net, where))
    M = abi.meas_pass
    window = ("from", "to")
    counts_td = _COUNTS + ("td",)
    if func == "when":
        if not rest:
            raise DeckError(f"{where}: WHEN needs vector=value")
        w = _when(rest[0], net, env, where, vec)
        o = _clause(rest[1:], net, env, where, counts_td + window)
        return Measure(name, [M(abi.MEAS_WHEN, w.pop("row"), **w, **o)])
    if func in ("find", "deriv"):
        if len(rest) < 2:
            raise DeckError(f"{where}: {func.upper()} needs a vector and AT= or WHEN")
        row = vec(rest[0])
        if rest[1].startswith("at="):
            if len(rest) > 2:
                raise DeckError(f"{where}: {func.upper()} ... AT takes no other option")
            kind = abi.MEAS_FIND_AT if func == "find" else abi.MEAS_DERIV_AT
            return Measure(name, [M(kind, row, at=_scalar(env, rest[1][3:], where))])
        if rest[1] != "when" or len(rest) < 3:
            raise DeckError(f"{where}: {func.upper()} needs AT= or WHEN vector=value")
        w = _when(rest[2], net, env, where, vec)
        o = _clause(rest[3:], net, env, where, counts_td + window)
        kind = abi.MEAS_FIND_WHEN if func == "find" else abi.MEAS_DERIV_WHEN
        return Measure(name, [M(abi.MEAS_WHEN, w.pop("row"), **w, **o), M(kind, row)])
    if func == "trig":
        if "targ" not in rest:
            raise DeckError(f"{where}: TRIG needs its TARG")
        k = rest.index("targ")
        trig, targ = rest[:k], rest[k + 1:]
        passes = []
        for part, kind in ((trig, abi.MEAS_WHEN), (targ, abi.MEAS_TARG)):
            if not part or part[0].startswith("at="):
                raise DeckError(f"{where}: TRIG/TARG AT= is outside what the lanes carry; give a vector and VAL=")
            row = vec(part[0])
            o = _clause(part[1:], net, env, where, ("val",) + counts_td + window)
            if kind == abi.MEAS_TARG:
                o.pop("td", None)  # the TARG counts from the TRIG event
            passes.append(M(kind, row, **o))
        return Measure(name, passes)
    stats = {"max": abi.MEAS_MAX, "min": abi.MEAS_MIN, "avg": abi.MEAS_AVG, "rms": abi.MEAS_RMS,
             "integ": abi.MEAS_INTEG, "integral": abi.MEAS_INTEG}
    if func in stats or func == "pp":
        if not rest:
            raise DeckError(f"{where}: {func.upper()} needs a vector")
        row = vec(rest[0])
        o = _clause(rest[1:], net, env, where, window)
        if func == "pp":
            return Measure(name, [M(abi.MEAS_MAX, row, **o), M(abi.MEAS_MIN, row, **o)], pp=True)
        return Measure(name, [M(stats[func], row, **o)])
    raise DeckError(f"{where}: the measure {func.upper()} is outside what the lanes carry")


def read_measures(text: str, net: Netlist, params: Optional[Mapping[str, Value]] = None) -> List[Measure]:
    """The deck's `.meas tran` cards as measures on `net` (the deck read by
    `read_deck`, with the same `params`): WHEN (against a value or a second
    vector; RISE/FALL/CROSS counts or LAST, TD, FROM, TO), FIND and DERIV at
    a time or at a WHEN, TRIG ... TARG (VAL and counts per clause; the TARG
    counts from the TRIG event, as the reference's measure stream does),
    MAX, MIN, AVG, RMS, INTEG, PP over a window, and PARAM='expr' over the
    parameters and the measures before it; `.meas op ... find vec` reads the
    operating point. Vectors are v(node) and i(vsource); values are numbers
    or parameters the same on every lane.
    Anything else raises DeckError naming the line."""
    env = _Env(net.lanes, dict(params or {}))
    cards = _expand_subckts(_logical_lines(text))
    _read_params(cards, env)
    out: List[Measure] = []
    for ln, card in cards:
        toks = _split(card)
        if toks[0] not in (".meas", ".measure"):
            continue
        where = f"line {ln}"
        if len(toks) < 4:
            raise DeckError(f"{where}: .meas needs an analysis, a name and a measure")
        name = toks[2]
        if any(m.name == name for m in out):
            raise DeckError(f"{where}: a second measure named {name!r}")
        if toks[1] == "op":
            if toks[3] != "find" or len(toks) != 5:
                raise DeckError(f"{where}: .meas op takes FIND vector")
            out.append(Measure(name, [], op_row=_vector(toks[4], net, where)))
            continue
        if toks[1] == "ac":
            columns: List[tuple] = []

            def acvec(tok, where=where, columns=columns):
                m = re.fullmatch(r"(v|vm|vdb|vp|vr|vi|i|im|idb|ip|ir|ii)\(([^(),]+)\)", tok)
                if not m:
                    raise DeckError(f"{where}: the AC measure reads {tok!r}; only v/vm/vdb/vp/vr/vi(node) and "
                                    "i/im/idb/ip/ir/ii(vsource) ride the lanes")
                f, nm = m.group(1), m.group(2).strip()
                row = _vector(f[0] + "(" + nm + ")", net, where)
                key = ("m" if len(f) == 1 else f[1:], row)
                if key not in columns:
                    columns.append(key)
                return columns.index(key)

            mm = _measure(name, toks[3], toks[4:], net, env, where, vec=acvec)
            mm.analysis, mm.columns = "ac", columns
            out.append(mm)
            continue
        if toks[1] != "tran":
            raise DeckError(f"{where}: only .meas tran, ac and op ride the lanes")
        if toks[3].startswith("param="):
            if len(toks) != 4:
                raise DeckError(f"{where}: PARAM takes one expression")
            text = toks[3][len("param="):].strip("'{}")
            trial = _Env(net.lanes, {})
            trial.vals = dict(env.vals)
            trial.vals.update({m.name: np.zeros(net.lanes) for m in out})
            trial.expr(text, where)  # names only parameters and earlier measures
            out.append(Measure(name, [], expr=text, params=dict(env.vals)))
            continue
        out.append(_measure(name, toks[3], toks[4:], net, env, where))
    return out


def measure_passes(measures: Sequence[Measure]) -> List[abi.MeasPass]:
    """Every measure's passes, in order, for Lanes.set_meas."""
    passes = [p for m in measures if m.analysis == "tran" for p in m.passes]
    if len(passes) > abi.MEAS_MAX_PASSES:
        raise DeckError(f"the measures need {len(passes)} passes; a template takes {abi.MEAS_MAX_PASSES}")
    return passes


def measure_values(measures: Sequence[Measure], value: np.ndarray, x_op: Optional[np.ndarray] = None,
                   ac: Optional[Mapping[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
    """Each measure's value per lane from Lanes.get_meas's `value` [lanes,
    passes] (NaN where it has none); `.meas op` cards read the operating
    points x_op [lanes, n], `.meas ac` cards their values in `ac` (NaN
    without them)."""
    out: Dict[str, np.ndarray] = {}
    k = 0
    lanes = value.shape[0]
    for m in measures:
        if m.expr is not None:
            ev = _Env(lanes, {})
            ev.vals = dict(m.params or {})
            ev.vals.update(out)
            with np.errstate(all="ignore"):
                out[m.name] = np.broadcast_to(np.asarray(ev.expr(m.expr, m.name), dtype=np.float64),
                                              (lanes,)).copy()
            continue
        if m.op_row is not None:
            out[m.name] = x_op[:, m.op_row].copy() if x_op is not None else np.full(value.shape[0], np.nan)
            continue
        if m.analysis == "ac":
            out[m.name] = np.asarray(ac[m.name]) if ac and m.name in ac else np.full(lanes, np.nan)
            continue
        if m.pp:
            out[m.name] = value[:, k] - value[:, k + 1]
        else:
            out[m.name] = value[:, k + len(m.passes) - 1]
        k += len(m.passes)
    return out


# The reasons a point has no value, or not all of them (include/espice.h
# espice_reason :260-284).
REASON_OK = 0
REASON_NO_CONVERGENCE = 1
REASON_TIMESTEP_TOO_SMALL = 2
REASON_SINGULAR_MATRIX = 3
REASON_MEASURE_UNRESOLVED = 5
REASON_OTHER = 255


def point_measures(measures: Sequence[Measure], value: np.ndarray, names: Optional[Sequence[str]] = None,
                   reports: Optional[Sequence] = None, op: Optional[np.ndarray] = None,
                   x_op: Optional[np.ndarray] = None, stopped_ok: bool = False,
                   ac: Optional[Mapping[str, np.ndarray]] = None):
    """Each lane's measures and reason as the reference's points API copies
    them (include/espice.h espice_copy_point_measures :324-338): values
    [lanes][len(names)] (names case-insensitive, default every measure in
    card order) and reasons [lanes]. A failed lane reads NaN throughout: its
    operating point (`op`, the espl_lane_newton rows [lanes, 4]) did not
    converge (SINGULAR_MATRIX when it was singular, else NO_CONVERGENCE), or
    its transient (`reports`, espl_step_report per lane) ended otherwise than
    done (TIMESTEP_TOO_SMALL on a step underflow, else OTHER). Otherwise NaN
    marks a measure with no value and the reason is MEASURE_UNRESOLVED.
    `.meas op` cards read x_op, the operating points [lanes, n]. With
    `stopped_ok` a transient stopped on request (status 4, an early stop
    once its measures resolved) counts as done."""
    allv = measure_values(measures, value, x_op, ac)
    keys = {k.lower(): k for k in allv}
    if names is None:
        names = list(allv)
    cols = []
    for nm in names:
        if nm.lower() not in keys:
            raise DeckError(f"UnknownMeasure: no .meas card named {nm!r}")
        cols.append(allv[keys[nm.lower()]])
    lanes = value.shape[0]
    out = np.stack(cols, axis=1) if cols else np.zeros((lanes, 0))
    reasons = np.zeros(lanes, dtype=np.uint32)
    failed = np.zeros(lanes, dtype=bool)
    if op is not None:
        bits = np.asarray(op)[:, 0]
        bad = (bits & abi.CONVERGED) == 0
        reasons[bad] = np.where((bits[bad] & abi.SINGULAR) != 0, REASON_SINGULAR_MATRIX, REASON_NO_CONVERGENCE)
        failed |= bad
    if reports is not None:
        status = np.array([r.status for r in reports], dtype=np.uint32)
        bad = (status != 1) & ~(stopped_ok & (status == 4)) & ~failed
        reasons[bad] = np.where(status[bad] == 2, REASON_TIMESTEP_TOO_SMALL, REASON_OTHER)
        failed |= bad
    out[failed] = np.nan
    unresolved = ~failed & np.isnan(out).any(axis=1)
    reasons[unresolved] = REASON_MEASURE_UNRESOLVED
    return out, reasons
