"""NMODL source -> syntax tree, for the mechanism subset MIND.jl's runtime executes.

MIND.jl reads MOD files with its own front end (src/compiler/frontend.jl:15-110, syntax
types in src/compiler/ir.jl:1-120).  This module is this project's reader for the same
language subset: the NEURON, PARAMETER, STATE, ASSIGNED, DEFINE, INITIAL, BREAKPOINT,
DERIVATIVE, PROCEDURE, FUNCTION and NET_RECEIVE blocks; declarations with units, limits,
defaults and fixed array extents; assignments (including derivatives `x'`), calls,
if/else, while, LOCAL and SOLVE statements; and the expression grammar with NMODL's
operator precedence (`^` binds tighter than unary minus and is right-associative).
TITLE, COMMENT, UNITS, INDEPENDENT, UNITSON/UNITSOFF and TABLE statements carry nothing
the step loop needs and are skipped.  VERBATIM, KINETIC, LINEAR and NONLINEAR blocks are
rejected with a ModError naming the line.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple, Union


class ModError(Exception):
    """A MOD source error, with file:line."""

    def __init__(self, filename: str, line: int, message: str):
        super().__init__(f"{filename}:{line}: {message}")
        self.filename, self.line, self.message = filename, line, message


# ---------------------------------------------------------------- tokens

@dataclass(frozen=True)
class Token:
    kind: str      # "name", "number", "op", "eof"
    text: str
    line: int


_TOKEN = re.compile(r"""
    (?P<ws>[ \t\r\f\v]+)
  | (?P<nl>\n)
  | (?P<number>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)
  | (?P<name>[A-Za-z_][A-Za-z_0-9]*'?)
  | (?P<op>==|!=|<=|>=|&&|\|\||[-+*/^<>=(){}\[\],!~:?'@.])
""", re.VERBOSE)


def tokenize(source: str, filename: str = "<string>") -> List[Token]:
    """Tokens of a MOD source with comments, TITLE lines and COMMENT blocks removed."""
    out: List[Token] = []
    lines = source.split("\n")
    i, in_comment = 0, False
    for number, text in enumerate(lines, start=1):
        stripped = text.strip()
        if in_comment:
            if stripped.startswith("ENDCOMMENT"):
                in_comment = False
            continue
        if stripped.startswith("COMMENT"):
            in_comment = True
            continue
        if stripped.startswith("TITLE"):
            continue
        pos = 0
        while pos < len(text):
            m = _TOKEN.match(text, pos)
            if m is None:
                raise ModError(filename, number, f"unexpected character {text[pos]!r}")
            kind = m.lastgroup
            value = m.group(kind)
            pos = m.end()
            if kind in ("ws", "nl"):
                continue
            if kind == "op" and value in (":", "?"):
                break   # comment to the end of the line
            out.append(Token(kind, value, number))
        i += 1
    if in_comment:
        raise ModError(filename, len(lines), "COMMENT without ENDCOMMENT")
    out.append(Token("eof", "", len(lines)))
    return out


# ---------------------------------------------------------------- syntax tree

@dataclass
class Num:
    value: float
    text: str


@dataclass
class Name:
    name: str


@dataclass
class Index:          # array element a[i]
    name: str
    index: "Expr"


@dataclass
class Call:
    name: str
    args: List["Expr"]


@dataclass
class Unary:
    op: str           # "-", "+", "!"
    arg: "Expr"


@dataclass
class Binary:
    op: str           # + - * / ^ < > <= >= == != && ||
    left: "Expr"
    right: "Expr"


Expr = Union[Num, Name, Index, Call, Unary, Binary]


@dataclass
class Assign:
    target: Union[Name, Index]
    value: Expr
    derivative: bool
    line: int


@dataclass
class CallStmt:
    call: Call
    line: int


@dataclass
class If:
    cond: Expr
    then: List["Stmt"]
    orelse: List["Stmt"]
    line: int


@dataclass
class While:
    cond: Expr
    body: List["Stmt"]
    line: int


@dataclass
class Local:
    names: List[Tuple[str, int]]   # (name, extent; 0 = scalar)
    line: int


@dataclass
class Solve:
    block: str
    method: str
    line: int


@dataclass
class EventInitial:     # INITIAL inside NET_RECEIVE
    body: List["Stmt"]
    line: int


Stmt = Union[Assign, CallStmt, If, While, Local, Solve, EventInitial]


@dataclass
class Decl:
    name: str
    extent: int = 0
    default: Optional[float] = None
    units: str = ""
    limits: Optional[Tuple[float, float]] = None
    line: int = 0


@dataclass
class Ion:
    name: str
    reads: List[str]
    writes: List[str]
    valence: Optional[float] = None


@dataclass
class Block:
    kind: str                      # initial, breakpoint, derivative, procedure, function, net_receive
    name: str
    args: List[str]
    body: List[Stmt]
    line: int


@dataclass
class ModFile:
    filename: str
    name: str = ""
    kind: str = ""                 # "density" (SUFFIX), "point" (POINT_PROCESS), "artificial"
    ranges: List[str] = field(default_factory=list)
    globals_: List[str] = field(default_factory=list)
    nonspecific: List[str] = field(default_factory=list)
    electrode: List[str] = field(default_factory=list)
    ions: List[Ion] = field(default_factory=list)
    randoms: List[str] = field(default_factory=list)
    defines: Dict[str, float] = field(default_factory=dict)
    parameters: List[Decl] = field(default_factory=list)
    states: List[Decl] = field(default_factory=list)
    assigned: List[Decl] = field(default_factory=list)
    blocks: Dict[str, Block] = field(default_factory=dict)   # by lower-case name (initial, breakpoint, ...)


# ---------------------------------------------------------------- parser

_SKIPPED_BLOCKS = {"UNITS", "INDEPENDENT", "CONSTANT"}
_REJECTED = {"VERBATIM", "KINETIC", "LINEAR", "NONLINEAR", "PARTIAL", "DISCRETE", "FUNCTION_TABLE",
             "BEFORE", "AFTER", "CONSERVE", "LAG", "SENS", "MATCH"}


class _Parser:
    def __init__(self, tokens: List[Token], filename: str):
        self.toks, self.pos, self.filename = tokens, 0, filename

    # -- token helpers
    def peek(self, k: int = 0) -> Token:
        return self.toks[min(self.pos + k, len(self.toks) - 1)]

    def next(self) -> Token:
        t = self.peek()
        self.pos += 1
        return t

    def error(self, message: str, tok: Optional[Token] = None):
        raise ModError(self.filename, (tok or self.peek()).line, message)

    def accept(self, text: str) -> bool:
        if self.peek().text == text and self.peek().kind != "eof":
            self.pos += 1
            return True
        return False

    def expect(self, text: str) -> Token:
        t = self.next()
        if t.text != text:
            self.error(f"expected {text!r}, found {t.text or 'end of file'!r}", t)
        return t

    def name(self) -> str:
        t = self.next()
        if t.kind != "name":
            self.error(f"expected a name, found {t.text!r}", t)
        return t.text

    def skip_braces(self):
        self.expect("{")
        depth = 1
        while depth:
            t = self.next()
            if t.kind == "eof":
                self.error("unbalanced braces", t)
            depth += (t.text == "{") - (t.text == "}")

    def units(self) -> str:
        """A parenthesised unit annotation, returned as text."""
        self.expect("(")
        parts, depth = [], 1
        while True:
            t = self.next()
            if t.kind == "eof":
                self.error("unterminated unit annotation", t)
            if t.text == "(":
                depth += 1
            elif t.text == ")":
                depth -= 1
                if depth == 0:
                    return "".join(parts)
            parts.append(t.text)

    def number(self) -> float:
        sign = -1.0 if self.accept("-") else (self.accept("+") and 1.0) or 1.0
        t = self.next()
        if t.kind == "number":
            return sign * float(t.text)
        if t.kind == "name" and t.text in self.mod.defines:
            return sign * self.mod.defines[t.text]
        self.error(f"expected a number, found {t.text!r}", t)

    # -- file
    def parse(self) -> ModFile:
        self.mod = ModFile(self.filename)
        while self.peek().kind != "eof":
            t = self.next()
            word = t.text
            if word in ("UNITSOFF", "UNITSON", "THREADSAFE"):
                continue
            if word in _REJECTED:
                self.error(f"{word} is not supported by this runtime", t)
            if word in _SKIPPED_BLOCKS:
                self.skip_braces()
            elif word == "DEFINE":
                name = self.name()
                self.mod.defines[name] = self.number()
            elif word == "NEURON":
                self.neuron_block()
            elif word in ("PARAMETER", "STATE", "ASSIGNED"):
                decls = self.declarations(word)
                {"PARAMETER": self.mod.parameters, "STATE": self.mod.states,
                 "ASSIGNED": self.mod.assigned}[word].extend(decls)
            elif word in ("INITIAL", "BREAKPOINT"):
                self.add_block(Block(word.lower(), word.lower(), [], self.statements(), t.line))
            elif word == "DERIVATIVE":
                name = self.name()
                self.add_block(Block("derivative", name, [], self.statements(), t.line))
            elif word in ("PROCEDURE", "FUNCTION"):
                name = self.name()
                args = self.arguments()
                if word == "FUNCTION" and self.peek().text == "(":
                    self.units()
                self.add_block(Block(word.lower(), name, args, self.statements(), t.line))
            elif word == "NET_RECEIVE":
                args = self.arguments()
                self.add_block(Block("net_receive", "net_receive", args, self.statements(True), t.line))
            else:
                self.error(f"unexpected {word!r} at the top level", t)
        if not self.mod.name:
            self.error("the NEURON block names no SUFFIX, POINT_PROCESS or ARTIFICIAL_CELL")
        return self.mod

    def add_block(self, block: Block):
        key = block.name if block.kind in ("derivative", "procedure", "function") else block.kind
        if key in self.mod.blocks:
            raise ModError(self.filename, block.line, f"{key} is defined twice")
        self.mod.blocks[key] = block

    def arguments(self) -> List[str]:
        self.expect("(")
        args = []
        while not self.accept(")"):
            args.append(self.name())
            if self.peek().text == "(":
                self.units()
            self.accept(",")
        return args

    def neuron_block(self):
        self.expect("{")
        m = self.mod
        while not self.accept("}"):
            t = self.next()
            w = t.text
            if w in ("SUFFIX", "POINT_PROCESS", "ARTIFICIAL_CELL"):
                m.name = self.name()
                m.kind = {"SUFFIX": "density", "POINT_PROCESS": "point", "ARTIFICIAL_CELL": "artificial"}[w]
            elif w in ("RANGE", "GLOBAL", "NONSPECIFIC_CURRENT", "ELECTRODE_CURRENT", "RANDOM", "POINTER",
                       "BBCOREPOINTER"):
                names = [self.name()]
                while self.accept(","):
                    names.append(self.name())
                target = {"RANGE": m.ranges, "GLOBAL": m.globals_, "NONSPECIFIC_CURRENT": m.nonspecific,
                          "ELECTRODE_CURRENT": m.electrode, "RANDOM": m.randoms}.get(w)
                if target is None:
                    self.error(f"{w} variables are not supported by this runtime", t)
                target.extend(names)
            elif w == "USEION":
                ion = Ion(self.name(), [], [])
                while self.peek().text in ("READ", "WRITE", "VALENCE"):
                    kw = self.next().text
                    if kw == "VALENCE":
                        ion.valence = self.number()
                        continue
                    lst = ion.reads if kw == "READ" else ion.writes
                    lst.append(self.name())
                    while self.accept(","):
                        lst.append(self.name())
                m.ions.append(ion)
            elif w == "THREADSAFE":
                continue
            else:
                self.error(f"unsupported NEURON statement {w!r}", t)

    def declarations(self, block: str) -> List[Decl]:
        self.expect("{")
        out = []
        while not self.accept("}"):
            t = self.peek()
            if t.text in ("UNITSOFF", "UNITSON"):
                self.next()
                continue
            d = Decl(self.name(), line=t.line)
            if self.accept("["):
                d.extent = int(self.number())
                self.expect("]")
            if self.accept("="):
                d.default = self.number()
            if self.peek().text == "(":
                d.units = self.units()
            if self.accept("<"):
                lo = self.number()
                self.expect(",")
                hi = self.number()
                self.expect(">")
                d.limits = (lo, hi)
            if block == "STATE" and self.peek().text == "FROM":   # STATE x FROM a TO b
                self.next(); self.number(); self.expect("TO"); self.number()
            out.append(d)
        return out

    # -- statements
    def statements(self, in_net_receive: bool = False) -> List[Stmt]:
        self.expect("{")
        body: List[Stmt] = []
        while not self.accept("}"):
            s = self.statement(in_net_receive)
            if s is not None:
                body.append(s)
        return body

    def statement(self, in_net_receive: bool = False):
        t = self.peek()
        w = t.text
        if t.kind == "eof":
            self.error("unexpected end of file in a block")
        if w in ("UNITSOFF", "UNITSON"):
            self.next()
            return None
        if w in _REJECTED:
            self.error(f"{w} is not supported by this runtime", t)
        if w == "LOCAL":
            self.next()
            names = []
            while True:
                n = self.name()
                extent = 0
                if self.accept("["):
                    extent = int(self.number())
                    self.expect("]")
                names.append((n, extent))
                if not self.accept(","):
                    break
            return Local(names, t.line)
        if w == "SOLVE":
            self.next()
            block = self.name()
            method = ""
            if self.accept("METHOD"):
                method = self.name()
            if self.peek().text == "STEADYSTATE":
                self.error("STEADYSTATE is not supported by this runtime")
            return Solve(block, method, t.line)
        if w == "TABLE":   # TABLE x, y DEPEND a FROM lo TO hi WITH n : a cache, not semantics
            self.next()
            while self.peek().text != "WITH":
                if self.peek().kind == "eof":
                    self.error("TABLE without WITH", t)
                self.next()
            self.next()
            self.number()
            return None
        if w == "if":
            return self.if_statement()
        if w == "while":
            self.next()
            self.expect("(")
            cond = self.expression()
            self.expect(")")
            return While(cond, self.statements(in_net_receive), t.line)
        if w == "INITIAL" and in_net_receive:
            self.next()
            return EventInitial(self.statements(), t.line)
        if w == "{":
            return If(Num(1.0, "1"), self.statements(in_net_receive), [], t.line)
        if t.kind != "name":
            self.error(f"unexpected {w!r}", t)
        # assignment or call
        name_tok = self.next()
        name = name_tok.text
        if self.peek().text == "(":
            call = self.call_rest(name)
            return CallStmt(call, t.line)
        derivative = name.endswith("'")
        if derivative:
            name = name[:-1]
        target: Union[Name, Index] = Name(name)
        if self.accept("["):
            target = Index(name, self.expression())
            self.expect("]")
        self.expect("=")
        return Assign(target, self.expression(), derivative, t.line)

    def if_statement(self) -> If:
        t = self.expect("if")
        self.expect("(")
        cond = self.expression()
        self.expect(")")
        then = self.statements()
        orelse: List[Stmt] = []
        if self.accept("else"):
            orelse = [self.if_statement()] if self.peek().text == "if" else self.statements()
        return If(cond, then, orelse, t.line)

    # -- expressions (lowest to highest precedence)
    def expression(self) -> Expr:
        return self.or_expr()

    def or_expr(self):
        e = self.and_expr()
        while self.accept("||"):
            e = Binary("||", e, self.and_expr())
        return e

    def and_expr(self):
        e = self.cmp_expr()
        while self.accept("&&"):
            e = Binary("&&", e, self.cmp_expr())
        return e

    def cmp_expr(self):
        e = self.add_expr()
        while self.peek().text in ("<", ">", "<=", ">=", "==", "!="):
            op = self.next().text
            e = Binary(op, e, self.add_expr())
        return e

    def add_expr(self):
        e = self.mul_expr()
        while self.peek().text in ("+", "-"):
            op = self.next().text
            e = Binary(op, e, self.mul_expr())
        return e

    def mul_expr(self):
        e = self.unary_expr()
        while self.peek().text in ("*", "/"):
            op = self.next().text
            e = Binary(op, e, self.unary_expr())
        return e

    def unary_expr(self):
        if self.peek().text in ("-", "+", "!"):
            op = self.next().text
            return Unary(op, self.unary_expr())
        return self.pow_expr()

    def pow_expr(self):
        base = self.primary()
        if self.accept("^"):
            return Binary("^", base, self.unary_expr())   # right-associative, binds the exponent's sign
        return base

    def primary(self) -> Expr:
        t = self.next()
        if t.kind == "number":
            value = Num(float(t.text), t.text)
            if self.peek().text == "(" and self.peek(1).kind == "name" and self.peek(2).text == ")":
                self.units()   # a unit annotation on a literal, e.g. 1 (ms)
            return value
        if t.text == "(":
            e = self.expression()
            self.expect(")")
            return e
        if t.kind == "name":
            if t.text in self.mod.defines:
                v = self.mod.defines[t.text]
                return Num(v, repr(v))
            if self.peek().text == "(":
                return self.call_rest(t.text)
            if self.accept("["):
                idx = self.expression()
                self.expect("]")
                return Index(t.text, idx)
            return Name(t.text)
        self.error(f"unexpected {t.text!r} in an expression", t)

    def call_rest(self, name: str) -> Call:
        self.expect("(")
        args: List[Expr] = []
        while not self.accept(")"):
            args.append(self.expression())
            if self.peek().text == "(":
                self.units()
            self.accept(",")
        return Call(name, args)


def parse_mod(source: str, filename: str = "<string>") -> ModFile:
    """Parse a MOD source (compile_mod's first stage, src/compiler/frontend.jl:85-110)."""
    return _Parser(tokenize(source, filename), filename).parse()
