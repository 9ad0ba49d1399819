"""Payoff scripts on the device: the reference's payoff language parsed and compiled here into register bytecode that
the engine's script kernel (csrc/script.cu, ob_script_price) runs on every path while it simulates them.

The language is the reference's (packages/structured/src/optlab/structured/script/parser.py:3-16 for the grammar,
lexer.py for the tokens, validate.py for the static rules): `underlying`, `param` and `state` declarations, then
events at dates or times, each with assignments, `if ... then ... else ... end`, `pay EXPR as TAG`, `terminate`;
expressions with arithmetic, comparisons, `and`/`or`/`not`, min, max, abs, exp, log, sqrt, worst, best, and windows
(`lowest`, `highest`, `variance`) over an underlying's fixings. Its evaluation (evaluator.py) reads conditions as masks
on every path: inside an `if`, `x = e` becomes `x = m e + (1 - m) x`, `pay e` adds `m alive e` to the flows and
`terminate` multiplies `alive` by 1 - m; with smoothing eps a comparison a >= b is the ramp
clip((a - b) / (eps |b|) + 1/2, 0, 1). The device keeps that reading, so every path runs the same instructions
(no divergence), and accumulates the present value of the flows (discount factors of the payment dates).

The issuer's call (`call pay`) runs in one of three modes: never called (the script's flows as written, the
reference's policy NEVER), recording a pilot (each event's flows before and after its call, and at the call its mask,
the alive mass, the amount and the state: what optlab_b200.exercise fits a Longstaff-Schwartz policy on), or applying
a fitted policy (the issuer calls where the regression's continuation is above the amount). Not on the device:
variance corridors whose bounds are not constants, fixings before the valuation date, calls decided on more than
four state variables; `compile_script` refuses them with a `ScriptError`.
"""

from __future__ import annotations

import ctypes as C
import datetime as dt
import math
import re
from dataclasses import dataclass, field

import numpy as np

from ._abi import OB_MODEL_HESTON_QE, OB_RULE_STRIDE, ObScriptRequest, ObScriptResult, check, load
from .engine import precision_code

try:  # the reference's error class, so that callers catching it catch ours
    from optlab.structured.script.lexer import ScriptError as _Base  # type: ignore
except Exception:  # noqa: BLE001
    _Base = ValueError


class ScriptError(_Base):
    """Syntax, validation or evaluation error, located in the script text (line and column when known)."""

    def __init__(self, message: str, line: int = 0, col: int = 0):
        self.message, self.line, self.col = message, line, col
        where = f"line {line}, col {col}: " if line else ""
        ValueError.__init__(self, where + message)


# ----------------------------------------------------------------------------------------------------------- tokens

KEYWORDS = {"underlying", "param", "event", "pay", "as", "end", "if", "then", "else", "terminate", "and", "or", "not"}
FUNCTIONS = {"min": 2, "max": 2, "abs": 1, "exp": 1, "log": 1, "sqrt": 1, "worst": None, "best": None}
WINDOWS = ("lowest", "highest", "variance")
TAGS = ("coupon", "upside", "redemption")
COMPARISONS = ("<", "<=", ">", ">=", "==")
MAX_UNDERLYINGS = 5
MAX_NESTING = 40
ANNUAL = 252.0  # realised variance: fixings a year (packages/structured/src/optlab/structured/varswap.py:24)


@dataclass(frozen=True)
class Token:
    kind: str  # NUMBER, DATE, NAME, KEYWORD, OP, NEWLINE, EOF
    text: str
    line: int
    col: int


_LEX = re.compile(
    r"(?P<SPACE>[ \t\r]+)|(?P<COMMENT>\#[^\n]*)|(?P<NEWLINE>\n)|(?P<DATE>\d{4}-\d{2}-\d{2}(?![\w.]))"
    r"|(?P<NUMBER>(\d+\.\d*|\.\d+|\d+)([eE][+-]?\d+)?)|(?P<NAME>[A-Za-z_][A-Za-z0-9_]*)|(?P<OP><=|>=|==|[-+*/()<>=,])"
)


def tokenize(text: str) -> list[Token]:
    out, line, start, pos = [], 1, 0, 0
    while pos < len(text):
        m = _LEX.match(text, pos)
        col = pos - start + 1
        if m is None:
            raise ScriptError(f"unexpected character {text[pos]!r}", line, col)
        kind, value = m.lastgroup, m.group()
        if kind == "NEWLINE":
            out.append(Token("NEWLINE", "\n", line, col))
            line, start = line + 1, m.end()
        elif kind == "NAME" and value in KEYWORDS:
            out.append(Token("KEYWORD", value, line, col))
        elif kind not in ("SPACE", "COMMENT"):
            out.append(Token(kind, value, line, col))
        pos = m.end()
    out.append(Token("NEWLINE", "\n", line, pos - start + 1))
    out.append(Token("EOF", "", line, pos - start + 1))
    return out


# -------------------------------------------------------------------------------------------------------------- AST


@dataclass(frozen=True)
class When:
    """An observation: a calendar date (ISO string) or a time in years."""

    value: object
    is_date: bool


@dataclass(eq=False)
class Num:
    value: float
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Name:
    id: str
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Unary:
    op: str  # "-" or "not"
    operand: object
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Binary:
    op: str
    left: object
    right: object
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Call:
    func: str
    args: tuple
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Window:
    func: str  # lowest, highest or variance
    underlying: str
    start: When
    end: When
    n: int | None = None
    lower: object = None
    upper: object = None
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Assign:
    name: str
    expr: object
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class If:
    cond: object
    body: tuple
    orelse: tuple = ()
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Pay:
    expr: object
    tag: str
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Terminate:
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class IssuerCall:
    expr: object
    line: int = 0
    col: int = 0


@dataclass(eq=False)
class Event:
    when: When
    pay: When | None
    body: tuple
    line: int = 0
    col: int = 0


@dataclass
class Program:
    underlyings: list
    params: dict
    events: list
    states: list = field(default_factory=list)


# ----------------------------------------------------------------------------------------------------------- parser


class _Parser:
    """Recursive descent over the token list; one statement a line, blocks closed by `end`."""

    def __init__(self, text: str):
        self.t = tokenize(text)
        self.i = 0
        self.depth = 0

    @property
    def tok(self) -> Token:
        return self.t[self.i]

    def err(self, msg, tok=None):
        tok = tok or self.tok
        return ScriptError(msg, tok.line, tok.col)

    def is_(self, kind, text=None):
        return self.tok.kind == kind and (text is None or self.tok.text == text)

    def take(self, kind, text=None):
        if self.is_(kind, text):
            self.i += 1
            return self.t[self.i - 1]
        return None

    def need(self, kind, text=None, what=None):
        tok = self.take(kind, text)
        if tok is None:
            found = {"NEWLINE": "end of line", "EOF": "end of script"}.get(self.tok.kind, repr(self.tok.text))
            raise self.err(f"expected {what or text or kind.lower()}, found {found}")
        return tok

    def peek(self, kind, text=None):
        nxt = self.t[min(self.i + 1, len(self.t) - 1)]
        return nxt.kind == kind and (text is None or nxt.text == text)

    def deeper(self, fn, tok):
        self.depth += 1
        if self.depth > MAX_NESTING:
            raise self.err(f"nested more than {MAX_NESTING} levels deep: split it into assignments", tok)
        try:
            return fn()
        finally:
            self.depth -= 1

    def eol(self):
        if not (self.take("NEWLINE") or self.is_("EOF")):
            raise self.err(f"unexpected {self.tok.text!r} at end of statement")
        while self.take("NEWLINE"):
            pass

    def program(self) -> Program:
        unds, params, events, states = [], {}, [], []
        while self.take("NEWLINE"):
            pass
        while not self.is_("EOF"):
            if self.is_("NAME", "state") and self.peek("NAME"):
                self.i += 1
                states.append(self.need("NAME", what="state variable").text)
                while self.take("OP", ","):
                    states.append(self.need("NAME", what="state variable").text)
            elif tok := self.take("KEYWORD", "underlying"):
                name = self.need("NAME", what="underlying name")
                unds.append((name.text, tok.line, tok.col))
            elif tok := self.take("KEYWORD", "param"):
                name = self.need("NAME", what="parameter name")
                self.need("OP", "=")
                sign = -1.0 if self.take("OP", "-") else 1.0
                value = sign * float(self.need("NUMBER", what="number").text)
                if name.text in params:
                    raise ScriptError(f"name {name.text!r} declared twice", tok.line, tok.col)
                params[name.text] = (value, tok.line, tok.col)
            elif self.is_("KEYWORD", "event"):
                events.append(self.event())
                continue
            else:
                raise self.err(f"expected underlying, param, state or event, found {self.tok.text!r}")
            self.eol()
        return Program(unds, params, events, states)

    def when(self) -> When:
        tok = self.tok
        if self.take("DATE"):
            return When(tok.text, True)
        if self.is_("NAME", "t"):
            self.i += 1
            self.need("OP", "=")
            return When(float(self.need("NUMBER", what="time in years").text), False)
        raise self.err(f"expected a date (YYYY-MM-DD) or t=<years>, found {tok.text!r}")

    def event(self) -> Event:
        tok = self.need("KEYWORD", "event")
        when = self.when()
        pay = self.when() if self.take("KEYWORD", "pay") else None
        self.eol()
        body = self.block(("end",))
        self.need("KEYWORD", "end", "'end' closing the event")
        self.eol()
        return Event(when, pay, body, tok.line, tok.col)

    def block(self, closers) -> tuple:
        out = []
        while not any(self.is_("KEYWORD", c) for c in closers):
            if self.is_("EOF"):
                raise self.err("unexpected end of script, missing 'end'")
            out.append(self.statement())
        return tuple(out)

    def statement(self):
        tok = self.tok
        if self.take("KEYWORD", "if"):
            cond = self.expr()
            self.need("KEYWORD", "then")
            self.eol()
            body = self.deeper(lambda: self.block(("else", "end")), tok)
            orelse = ()
            if self.take("KEYWORD", "else"):
                self.eol()
                orelse = self.deeper(lambda: self.block(("end",)), tok)
            self.need("KEYWORD", "end", "'end' closing the if")
            self.eol()
            return If(cond, body, orelse, tok.line, tok.col)
        if self.take("KEYWORD", "pay"):
            e = self.expr()
            self.need("KEYWORD", "as")
            tag = self.need("NAME", what="a flow tag").text
            self.eol()
            return Pay(e, tag, tok.line, tok.col)
        if self.take("KEYWORD", "terminate"):
            self.eol()
            return Terminate(tok.line, tok.col)
        if self.is_("NAME", "call") and self.peek("KEYWORD", "pay"):
            self.i += 2
            e = self.expr()
            self.eol()
            return IssuerCall(e, tok.line, tok.col)
        if self.take("NAME"):
            self.need("OP", "=", "'=' (assignment)")
            e = self.expr()
            self.eol()
            return Assign(tok.text, e, tok.line, tok.col)
        raise self.err(f"expected a statement, found {tok.text!r}")

    def expr(self):
        left = self.conj()
        while tok := self.take("KEYWORD", "or"):
            left = Binary("or", left, self.conj(), tok.line, tok.col)
        return left

    def conj(self):
        left = self.negation()
        while tok := self.take("KEYWORD", "and"):
            left = Binary("and", left, self.negation(), tok.line, tok.col)
        return left

    def negation(self):
        if tok := self.take("KEYWORD", "not"):
            return Unary("not", self.deeper(self.negation, tok), tok.line, tok.col)
        return self.comparison()

    def comparison(self):
        left = self.sum()
        if self.tok.kind == "OP" and self.tok.text in COMPARISONS:
            tok = self.tok
            self.i += 1
            left = Binary(tok.text, left, self.sum(), tok.line, tok.col)
            if self.tok.kind == "OP" and self.tok.text in COMPARISONS:
                raise self.err("chained comparisons are not allowed, use 'and'")
        return left

    def sum(self):
        left = self.product()
        while self.tok.kind == "OP" and self.tok.text in "+-":
            tok = self.tok
            self.i += 1
            left = Binary(tok.text, left, self.product(), tok.line, tok.col)
        return left

    def product(self):
        left = self.sign()
        while self.tok.kind == "OP" and self.tok.text in "*/":
            tok = self.tok
            self.i += 1
            left = Binary(tok.text, left, self.sign(), tok.line, tok.col)
        return left

    def sign(self):
        if tok := self.take("OP", "-"):
            return Unary("-", self.deeper(self.sign, tok), tok.line, tok.col)
        return self.atom()

    def atom(self):
        tok = self.tok
        if self.take("NUMBER"):
            return Num(float(tok.text), tok.line, tok.col)
        if self.take("OP", "("):
            e = self.deeper(self.expr, tok)
            self.need("OP", ")")
            return e
        if self.take("NAME"):
            if not self.take("OP", "("):
                return Name(tok.text, tok.line, tok.col)
            if tok.text in WINDOWS:
                return self.window(tok)
            if tok.text not in FUNCTIONS:
                raise self.err(f"unknown function {tok.text!r}", tok)
            args = [self.deeper(self.expr, tok)]
            while self.take("OP", ","):
                args.append(self.deeper(self.expr, tok))
            self.need("OP", ")")
            arity = FUNCTIONS[tok.text]
            if (arity is None and len(args) < 2) or (arity is not None and len(args) != arity):
                raise self.err(f"{tok.text} takes {'at least 2' if arity is None else arity} argument(s), "
                               f"got {len(args)}", tok)
            return Call(tok.text, tuple(args), tok.line, tok.col)
        raise self.err(f"expected an expression, found {tok.text!r}" if tok.text else "expected an expression")

    def window(self, tok):
        und = self.need("NAME", what="underlying name").text
        self.need("OP", ",")
        start = self.when()
        self.need("OP", ",")
        end = self.when()
        n = lower = upper = None
        while self.take("OP", ","):
            if n is None and lower is None and self.is_("NAME", "n") and self.peek("OP", "="):
                self.i += 2
                num = self.need("NUMBER", what="number of fixings")
                if not num.text.isdigit() or int(num.text) < 1:
                    raise self.err("n must be a positive integer", num)
                n = int(num.text)
                continue
            if lower is not None:
                raise self.err("a window takes at most two bounds (its corridor)")
            lower = self.deeper(self.expr, tok)
            self.need("OP", ",")
            upper = self.deeper(self.expr, tok)
        self.need("OP", ")")
        return Window(tok.text, und, start, end, n, lower, upper, tok.line, tok.col)


def parse(text: str) -> Program:
    """The script's Program; ScriptError with the line and column of the first syntax error."""
    return _Parser(text).program()


# -------------------------------------------------------------------------------------------------------- validation


def _reserved(name, line, what):
    if name in KEYWORDS or name in FUNCTIONS or name in WINDOWS:
        raise ScriptError(f"{what} name {name!r} is reserved", line)


def _key(w: When):
    return w.value


def validate(p: Program) -> Program:
    """The reference's static rules (validate.py:46-167): declarations, increasing events, payment dates, tags,
    variables assigned before use, windows inside their event and of the script's date mode."""
    if not p.underlyings:
        raise ScriptError("no underlying declared (add 'underlying NAME')", 1)
    unds = set()
    for name, line, col in p.underlyings:
        _reserved(name, line, "underlying")
        if name in unds:
            raise ScriptError(f"underlying {name!r} declared twice", line, col)
        unds.add(name)
    if len(p.underlyings) > MAX_UNDERLYINGS:
        raise ScriptError(f"at most {MAX_UNDERLYINGS} underlyings are supported, found {len(p.underlyings)}",
                          p.underlyings[MAX_UNDERLYINGS][1])
    for name, (_, line, col) in p.params.items():
        _reserved(name, line, "parameter")
        if name in unds:
            raise ScriptError(f"name {name!r} declared twice", line, col)
    if not p.events:
        raise ScriptError("the script has no event", 1)
    if len(set(p.states)) != len(p.states):
        raise ScriptError("a state is declared twice", 1)
    mode = p.events[0].when.is_date
    defined: set = set()
    prev = None
    for ev in p.events:
        for w in (ev.when, ev.pay):
            if w is not None and w.is_date != mode:
                raise ScriptError("dates and times (t=...) cannot be mixed in one script", ev.line, ev.col)
        if prev is not None and _key(ev.when) <= _key(prev.when):
            raise ScriptError(f"event dates must be strictly increasing ({ev.when.value} after {prev.when.value})",
                              ev.line, ev.col)
        if ev.pay is not None and _key(ev.pay) < _key(ev.when):
            raise ScriptError("the payment date is before the observation date", ev.line, ev.col)
        defined = _check_block(p, ev, mode, ev.body, defined, unds)
        prev = ev
    return p


def _check_block(p, ev, mode, body, defined, unds):
    defined = set(defined)
    calls = 0
    for s in body:
        if isinstance(s, Assign):
            _reserved(s.name, s.line, "variable")
            if s.name in p.params or s.name in unds:
                raise ScriptError(f"cannot assign to {s.name!r}, it is a parameter or an underlying", s.line, s.col)
            _check_expr(p, ev, mode, s.expr, defined, unds)
            defined.add(s.name)
        elif isinstance(s, Pay):
            if ev.pay is None:
                raise ScriptError("'pay' in an event without a payment date (write 'event DATE pay DATE')",
                                  s.line, s.col)
            if s.tag not in TAGS:
                raise ScriptError(f"unknown flow tag {s.tag!r}, expected one of {', '.join(TAGS)}", s.line, s.col)
            _check_expr(p, ev, mode, s.expr, defined, unds)
        elif isinstance(s, IssuerCall):
            if ev.pay is None:
                raise ScriptError("'call pay' in an event without a payment date (write 'event DATE pay DATE')",
                                  s.line, s.col)
            calls += 1
            if calls > 1:
                raise ScriptError("one call per event: the issuer redeems at most once on a date", s.line, s.col)
            _check_expr(p, ev, mode, s.expr, defined, unds)
        elif isinstance(s, If):
            _check_expr(p, ev, mode, s.cond, defined, unds)
            defined = (_check_block(p, ev, mode, s.body, defined, unds)
                       & _check_block(p, ev, mode, s.orelse, defined, unds))
    return defined


def _check_expr(p, ev, mode, e, defined, unds):
    if isinstance(e, Num):
        return
    if isinstance(e, Name):
        if e.id not in defined and e.id not in p.params and e.id not in unds:
            raise ScriptError(f"{e.id!r} is used before it is assigned", e.line, e.col)
    elif isinstance(e, Unary):
        _check_expr(p, ev, mode, e.operand, defined, unds)
    elif isinstance(e, Binary):
        _check_expr(p, ev, mode, e.left, defined, unds)
        _check_expr(p, ev, mode, e.right, defined, unds)
    elif isinstance(e, Call):
        for a in e.args:
            _check_expr(p, ev, mode, a, defined, unds)
    elif isinstance(e, Window):
        if e.underlying not in unds:
            raise ScriptError(f"{e.underlying!r} is not a declared underlying", e.line, e.col)
        for d in (e.start, e.end):
            if d.is_date != mode:
                raise ScriptError("dates and times (t=...) cannot be mixed in one script", e.line, e.col)
        if _key(e.end) <= _key(e.start):
            raise ScriptError(f"{e.func} window ends before it starts", e.line, e.col)
        if _key(e.end) > _key(ev.when):
            raise ScriptError(f"{e.func} window ends after the event date (it would read future fixings)",
                              e.line, e.col)
        if mode and e.n is not None:
            raise ScriptError("n= is only for time windows; date windows use every business day", e.line, e.col)
        if not mode and e.n is None:
            raise ScriptError("a time window needs the number of fixings, e.g. n=252", e.line, e.col)
        if e.lower is not None and e.func != "variance":
            raise ScriptError(f"{e.func} takes no corridor: only variance does", e.line, e.col)
        for b in (e.lower, e.upper):
            if b is not None:
                _check_expr(p, ev, mode, b, defined, unds)
    else:
        raise ScriptError(f"unexpected expression {e!r}", getattr(e, "line", 0))


# ---------------------------------------------------------------------------------------------------------- timeline


def _date(s) -> dt.date:
    return dt.date.fromisoformat(str(s))


def year_fraction(start, end) -> float:
    """ACT/365F between two dates."""
    return (_date(end) - _date(start)).days / 365.0


def business_days(start, end) -> list:
    """Monday to Friday from start to end, both included (the reference's weekend calendar)."""
    a, b = _date(start), _date(end)
    out, d = [], a
    while d <= b:
        if d.weekday() < 5:
            out.append(d)
        d += dt.timedelta(days=1)
    return out


@dataclass
class Timeline:
    event_times: np.ndarray
    pay_times: list
    windows: list  # Window nodes in order of first appearance
    window_times: list  # their fixing times
    sim_times: np.ndarray  # sorted positive times to simulate


def _walk_windows(node, out):
    if isinstance(node, Window):
        if all(node is not w for w in out):
            out.append(node)
        for b in (node.lower, node.upper):
            if b is not None:
                _walk_windows(b, out)
    elif isinstance(node, Unary):
        _walk_windows(node.operand, out)
    elif isinstance(node, Binary):
        _walk_windows(node.left, out)
        _walk_windows(node.right, out)
    elif isinstance(node, Call):
        for a in node.args:
            _walk_windows(a, out)
    elif isinstance(node, If):
        _walk_windows(node.cond, out)
        for s in node.body + node.orelse:
            _walk_windows(s, out)
    elif isinstance(node, (Assign, Pay, IssuerCall)):
        _walk_windows(node.expr, out)


def build_timeline(p: Program, valuation=None) -> Timeline:
    """Times in years of the events, payments and window fixings (timeline.py:84-103): dates by ACT/365F from the
    valuation date, time windows on n equal steps in (start, end], date windows on every business day."""

    def t_of(w: When) -> float:
        if not w.is_date:
            return float(w.value)
        if valuation is None:
            raise ValueError("the script uses calendar dates: give a valuation date")
        return year_fraction(valuation, w.value)

    events = np.array([t_of(ev.when) for ev in p.events])
    pays = [t_of(ev.pay) if ev.pay is not None else None for ev in p.events]
    found: list = []
    for ev in p.events:
        for s in ev.body:
            _walk_windows(s, found)
    times = []
    for w in found:
        if not w.start.is_date:
            a, b = float(w.start.value), float(w.end.value)
            times.append(np.linspace(a + (b - a) / w.n, b, w.n))
        else:
            if valuation is None:
                raise ValueError("the script uses calendar dates: give a valuation date")
            times.append(np.array([year_fraction(valuation, d) for d in business_days(w.start.value, w.end.value)]))
    every = np.concatenate([events, *times]) if times else events
    return Timeline(events, pays, found, times, np.unique(every[every > 0]))


# ---------------------------------------------------------------------------------------------------------- compiler

# Opcodes of the device program (csrc/script.cu). An instruction is four ints: op, d, a, b (registers or indices).
OP = {name: k for k, name in enumerate((
    "spot", "win", "mov", "add", "sub", "mul", "div", "neg", "min", "max", "abs", "exp", "log", "sqrt",
    "ge", "gt", "le", "lt", "eq", "and", "or", "not", "assign", "pay", "term", "cond", "call"))}
_ARITH = {"+": "add", "-": "sub", "*": "mul", "/": "div"}
_CMP = {">=": "ge", ">": "gt", "<=": "le", "<": "lt", "==": "eq"}
WIN_FUNC = {"lowest": 0, "highest": 1, "variance": 2}
MAX_REGS = 128
MAX_WINDOWS = 8
MAX_STATE = 4  # variables an issuer's call is decided on (the regression's state)


@dataclass
class Compiled:
    """A script ready for the device: registers 0..n_const-1 hold the constants (register 0 is 1.0, the top-level
    mask), then the variables, then temporaries; `code` is (n, 4) int32, each event a slice `event_code[k]:[k+1]`."""

    program: Program
    timeline: Timeline
    names: list
    consts: np.ndarray
    n_regs: int
    code: np.ndarray
    event_code: np.ndarray
    event_times: np.ndarray
    pay_times: list
    windows: list  # (name index, func, fixing times, lower, upper)
    smoothing: float
    params: dict
    calls: list = field(default_factory=list)  # per `call pay`: (event index, registers of its state)


class _Emitter:
    def __init__(self, p: Program, params: dict, names: list, windows: list, smoothing: float):
        self.p, self.params, self.names, self.windows = p, params, names, windows
        self.consts: list = [1.0]
        self.const_reg: dict = {1.0: 0}
        self.vars: dict = {}
        self.code: list = []
        self.n_fixed = None  # registers below it are constants and variables; temporaries above
        self.top = 0
        self.max_top = 0
        self.smooth = smoothing
        self.calls: list = []
        self.event = 0

    def const(self, v: float) -> int:
        v = float(v)
        key = v if not math.isnan(v) else "nan"
        if key not in self.const_reg:
            self.const_reg[key] = len(self.consts)
            self.consts.append(v)
        return self.const_reg[key]

    def temp(self) -> int:
        r = self.top
        self.top += 1
        self.max_top = max(self.max_top, self.top)
        return r

    def emit(self, op, d=0, a=0, b=0):
        self.code.append((OP[op], d, a, b))

    # constants and variables get their registers in a first pass, so that temporaries can sit above them
    def collect(self, node):
        if isinstance(node, Num):
            self.const(node.value)
        elif isinstance(node, Name):
            if node.id in self.params:
                self.const(self.params[node.id])
        elif isinstance(node, Assign):
            self.vars.setdefault(node.name, None)
            self.collect(node.expr)
        elif isinstance(node, (Pay, IssuerCall)):
            self.collect(node.expr)
            if isinstance(node, IssuerCall):
                for n in self.p.states:
                    if n in self.params:
                        self.const(self.params[n])
        elif isinstance(node, If):
            self.collect(node.cond)
            for s in node.body + node.orelse:
                self.collect(s)
        elif isinstance(node, Unary):
            self.const(1.0)
            self.collect(node.operand)
        elif isinstance(node, Binary):
            self.collect(node.left)
            self.collect(node.right)
        elif isinstance(node, Call):
            for a in node.args:
                self.collect(a)
        elif isinstance(node, Window):
            for b in (node.lower, node.upper):
                if b is not None:
                    self.collect(b)

    def layout(self):
        n_const = len(self.consts)
        for k, name in enumerate(self.vars):
            self.vars[name] = n_const + k
        self.n_fixed = n_const + len(self.vars)
        self.top = self.max_top = self.n_fixed

    def expr(self, e) -> int:
        """Registers of e's value (a constant's or a variable's own register, or a new temporary)."""
        if isinstance(e, Num):
            return self.const_reg[float(e.value) if not math.isnan(e.value) else "nan"]
        if isinstance(e, Name):
            if e.id in self.vars and self.vars[e.id] is not None and e.id not in self.params:
                return self.vars[e.id]
            if e.id in self.params:
                return self.const_reg[float(self.params[e.id])]
            d = self.temp()
            self.emit("spot", d, self.names.index(e.id))
            return d
        if isinstance(e, Unary):
            a = self.expr(e.operand)
            d = self.temp()
            self.emit("neg" if e.op == "-" else "not", d, a)
            return d
        if isinstance(e, Binary):
            a = self.expr(e.left)
            b = self.expr(e.right)
            d = self.temp()
            op = _ARITH.get(e.op) or _CMP.get(e.op) or e.op  # and / or
            self.emit(op, d, a, b)
            return d
        if isinstance(e, Call):
            regs = [self.expr(a) for a in e.args]
            if e.func in ("worst", "best"):
                acc = regs[0]
                for r in regs[1:]:
                    d = self.temp()
                    self.emit("min" if e.func == "worst" else "max", d, acc, r)
                    acc = d
                return acc
            d = self.temp()
            self.emit(e.func, d, *regs)
            return d
        if isinstance(e, Window):
            d = self.temp()
            self.emit("win", d, next(k for k, w in enumerate(self.windows) if w is e))
            return d
        raise ScriptError(f"unexpected expression {e!r}", getattr(e, "line", 0))

    def block(self, body, mask: int, tag_of: dict):
        for s in body:
            mark = self.top
            if isinstance(s, Assign):
                e = self.expr(s.expr)
                self.emit("assign", self.vars[s.name], e, mask)
            elif isinstance(s, Pay):
                e = self.expr(s.expr)
                self.emit("pay", TAGS.index(s.tag), e, mask)
            elif isinstance(s, Terminate):
                self.emit("term", 0, mask)
            elif isinstance(s, IssuerCall):
                e = self.expr(s.expr)
                names = self.p.states or [u[0] for u in self.p.underlyings]
                if len(names) > MAX_STATE:
                    raise ScriptError(f"the issuer's call is decided on at most {MAX_STATE} state variables on the "
                                      f"device, found {len(names)}", s.line, s.col)
                regs = [self.expr(Name(n, s.line, s.col)) for n in names]
                self.emit("call", len(self.calls), e, mask)
                self.calls.append((self.event, regs))
            elif isinstance(s, If):
                c = self.expr(s.cond)
                cd = self.temp()
                self.emit("cond", cd, c, mask)
                m_body = self.temp()
                self.emit("mul", m_body, mask, cd)
                inner = self.top
                self.block(s.body, m_body, tag_of)
                self.top = inner
                if s.orelse:
                    inv = self.temp()
                    self.emit("not", inv, cd)
                    m_else = self.temp()
                    self.emit("mul", m_else, mask, inv)
                    self.block(s.orelse, m_else, tag_of)
            self.top = mark
            if self.max_top > MAX_REGS:
                raise ScriptError(f"the script needs more than {MAX_REGS} registers: split its expressions",
                                  getattr(s, "line", 0))


def _constant(e, params):
    """The value of an expression made of numbers and parameters only, else None."""
    if isinstance(e, Num):
        return e.value
    if isinstance(e, Name) and e.id in params:
        return params[e.id]
    if isinstance(e, Unary) and e.op == "-":
        v = _constant(e.operand, params)
        return None if v is None else -v
    if isinstance(e, Binary) and e.op in _ARITH:
        a, b = _constant(e.left, params), _constant(e.right, params)
        if a is None or b is None:
            return None
        return {"+": a + b, "-": a - b, "*": a * b, "/": a / b if b != 0 else math.nan}[e.op]
    return None


def compile_script(text: str, params: dict | None = None, smoothing: float = 0.0, valuation=None) -> Compiled:
    """Parse, validate and compile a script for the device; `params` override the script's `param` values."""
    p = validate(parse(text))
    values = {k: v[0] for k, v in p.params.items()}
    unknown = set(params or {}) - set(values)
    if unknown:
        raise KeyError(f"unknown parameter(s): {', '.join(sorted(unknown))}")
    values.update({k: float(v) for k, v in (params or {}).items()})
    tl = build_timeline(p, valuation)
    if np.any(tl.event_times < 0) or any(np.any(t < 0) for t in tl.window_times):
        raise ScriptError("an observation before the valuation date reads history: not evaluated on the device")
    names = [u[0] for u in p.underlyings]
    if len(tl.windows) > MAX_WINDOWS:
        raise ScriptError(f"at most {MAX_WINDOWS} windows on the device, found {len(tl.windows)}")
    windows = []
    for w, times in zip(tl.windows, tl.window_times):
        lo = hi = math.nan
        if w.func == "variance":
            if len(times) < 2:
                raise ScriptError("a variance window needs at least two fixings", w.line, w.col)
            if w.lower is not None:
                lo, hi = _constant(w.lower, values), _constant(w.upper, values)
                if lo is None or hi is None:
                    raise ScriptError("a variance corridor on the device has bounds made of numbers and parameters",
                                      w.line, w.col)
        windows.append((names.index(w.underlying), WIN_FUNC[w.func], np.asarray(times, float), lo, hi))
    em = _Emitter(p, values, names, tl.windows, smoothing)
    for ev in p.events:
        for s in ev.body:
            em.collect(s)
    em.layout()
    starts = []
    for k, ev in enumerate(p.events):
        starts.append(len(em.code))
        em.event = k
        em.block(ev.body, 0, {})
    starts.append(len(em.code))
    code = np.array(em.code, dtype=np.int32).reshape(-1, 4) if em.code else np.zeros((0, 4), np.int32)
    return Compiled(p, tl, names, np.array(em.consts, float), em.max_top, code, np.array(starts, np.int32),
                    tl.event_times, tl.pay_times, windows, float(smoothing), values, em.calls)


# ----------------------------------------------------------------------------------------------------------- device


def _step_of(times, t_end, what):
    """Index of each time among the grid's step ends (0: the valuation date)."""
    idx = np.searchsorted(t_end, np.asarray(times, float) - 1e-9)
    idx = np.clip(idx, 0, len(t_end) - 1)
    bad = np.abs(t_end[idx] - times) > 1e-9
    if np.any(bad):
        raise ValueError(f"the simulation grid has no step ending at the {what} time(s) {np.asarray(times)[bad][:3]}")
    return idx.astype(np.int32)


@dataclass
class ScriptHeld:
    struct: ObScriptRequest
    keep: list
    compiled: Compiled


def script_request(compiled: Compiled, sim, discount, call_mode: int = 0, rules=None, pair_values: bool = False,
                   branch=None) -> ScriptHeld:
    """The device request of a compiled script on a simulation: `sim` is an mc_request (Held) whose model part
    (model, names in the script's underlying order, grid, tables, spots, log-forwards) is simulated, its product part
    ignored; `discount(t)` gives the discount factor of a payment at t. Every observation time must be a step end.
    call_mode: 0 the issuer never calls, 1 record a pilot (the held `record` array, filled by `run`), 2 apply
    `rules` ((n_calls, OB_RULE_STRIDE), optlab_b200.exercise.Policy.pack). pair_values: keep each pair's average
    present value (the held `pair_value` array). branch = (step, outer_pairs, pairs_per_outer, outer_seed): the
    pairs continue the paths of an outer simulation of outer_pairs pairs on outer_seed after step end `step`
    (pairs_per_outer pairs a path, path o < outer_pairs being leg 0 of outer pair o, the others leg 1)."""
    s = sim.struct
    S = s.n_steps
    if s.n_names != len(compiled.names):
        raise ValueError(f"the script has {len(compiled.names)} underlyings, the simulation {s.n_names} names")
    if s.model == OB_MODEL_HESTON_QE and len(compiled.names) != 1:
        raise ValueError("the QE model has one name")
    dts = np.ctypeslib.as_array(s.dt, shape=(S,))
    t0 = np.ctypeslib.as_array(s.t0, shape=(S,))
    t_end = np.concatenate([[0.0], t0 + dts])
    ev_step = _step_of(compiled.event_times, t_end, "event")
    disc = np.array([float(discount(t)) if (t is not None and t > 0) else 0.0 for t in compiled.pay_times])
    win_name, win_func, win_fix0, fix_step, lo, hi = [], [], [0], [], [], []
    for name, func, times, a, b in compiled.windows:
        win_name.append(name), win_func.append(func)
        fix_step.extend(_step_of(times, t_end, "window fixing").tolist())
        win_fix0.append(len(fix_step))
        lo.append(a), hi.append(b)
    arrays = dict(
        code=np.ascontiguousarray(compiled.code.ravel(), np.int32),
        consts=np.ascontiguousarray(compiled.consts, np.float64),
        event_step=np.ascontiguousarray(ev_step, np.int32),
        event_code=np.ascontiguousarray(compiled.event_code, np.int32),
        event_discount=np.ascontiguousarray(disc, np.float64),
        win_name=np.array(win_name, np.int32), win_func=np.array(win_func, np.int32),
        win_fix0=np.array(win_fix0, np.int32), fix_step=np.array(fix_step, np.int32),
        win_lower=np.array(lo, np.float64), win_upper=np.array(hi, np.float64),
    )
    n_calls = len(compiled.calls)
    n_state = len(compiled.calls[0][1]) if n_calls else 0
    cs = np.full((max(n_calls, 1), 4), 0, np.int32)
    for c, (_, regs) in enumerate(compiled.calls):
        cs[c, : len(regs)] = regs
    arrays["call_state"] = np.ascontiguousarray(cs.ravel() if n_calls else np.zeros(0, np.int32))
    if call_mode == 2:
        rules = np.ascontiguousarray(rules, np.float64)
        if rules.shape != (n_calls, OB_RULE_STRIDE):
            raise ValueError(f"rules must be ({n_calls}, {OB_RULE_STRIDE})")
        arrays["rules"] = rules.ravel()
    if call_mode == 1:
        arrays["record"] = np.zeros((2 * s.n_pairs, 2 * len(ev_step) + n_calls * (3 + n_state)))
    if pair_values or branch is not None:
        arrays["pair_value"] = np.zeros(s.n_pairs)
    r = ObScriptRequest()
    r.model = s
    r.n_code = compiled.code.shape[0]
    r.n_const = len(compiled.consts)
    r.n_regs = compiled.n_regs
    r.n_events = len(ev_step)
    r.n_windows = len(win_name)
    r.smoothing = compiled.smoothing
    r.n_calls, r.n_state, r.call_mode = n_calls, n_state, int(call_mode)
    if branch is not None:
        step, outer, per, seed = branch
        r.branch, r.branch_step, r.branch_outer, r.branch_pairs, r.branch_seed = 1, int(step), int(outer), int(per), \
            int(seed) & (2**64 - 1)
    for k, a in arrays.items():
        ctype = C.c_int if a.dtype == np.int32 else C.c_double
        setattr(r, k, a.ctypes.data_as(C.POINTER(ctype)) if a.size else None)
    return ScriptHeld(r, [sim, arrays], compiled)


def run(held: ScriptHeld, precision="fp64") -> ObScriptResult:
    """Simulate and evaluate on the device: the price (mean of the pair-averaged present values), its SE, and the
    paths where the script was undefined (counts), raised as ScriptError like the reference's evaluator."""
    res = ObScriptResult()
    check(load().ob_script_price(C.byref(held.struct), precision_code(precision), C.byref(res)))
    return check_result(held, res)


def check_result(held: ScriptHeld, res: ObScriptResult) -> ObScriptResult:
    """Raise ScriptError for the paths where a run's script was undefined (the counts of res), as the reference's
    evaluator raises; else res."""
    if res.bad_pay:
        raise ScriptError(f"an amount paid is not finite on {res.bad_pay} paths it reaches")
    if res.bad_cond:
        raise ScriptError(f"a condition is undefined (NaN) on {res.bad_cond} paths it reaches")
    if res.bad_redemption and held.compiled.smoothing == 0.0:
        raise ScriptError(f"the redemption is not paid exactly once on {res.bad_redemption} paths "
                          "(a valid product pays one 'redemption' per path)")
    return res
