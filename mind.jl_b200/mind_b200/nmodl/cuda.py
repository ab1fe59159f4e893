"""Mechanism IR -> CUDA C for sm_100a: one struct of inlined device functions per MOD.

The phases follow MIND.jl's generated ones (src/compiler/codegen.jl:362-485) and the
runtime that calls them (src/runtime/cuda/micro.jl:394-598):

  initial(r)          INITIAL, at t = 0 on the initial voltage;
  current(r)          BREAKPOINT without its SOLVE statements, on the probe voltage r.v;
                      returns 0 + (NONSPECIFIC currents, then the ion currents a USEION
                      writes, in declaration order) - (ELECTRODE currents); the window
                      kernel calls it at v + 0.001 and at v, and the second call's field
                      writes persist (micro.jl:427-500);
  advance(r)          the hoisted SOLVE statements at t + dt on the new voltage: a
                      DERIVATIVE block integrated by cnexp, or a PROCEDURE (after_cvode);
  receive(r, w, f)    NET_RECEIVE with its first argument w and the event flag f.

Every phase loads the row's fields into locals (a struct the compiler keeps in registers),
runs the statements in source order, and writes back the fields the phase assigns -- the
shape of the reference's generated functions.  Expressions keep the MOD's operation order
(left-associative + - * /, `^` as pow); exp, log and pow are the project-owned mind_exp,
mind_log and mind_pow that the CPU oracle also uses.  cnexp lowers `x' = (inf - x)/tau`
and `x' = -x/tau` to x + (1 - exp(dt (-1/tau))) (inf - x) (codegen.jl:605-628) and any
other equation affine in its state to x + dt phi(a dt) b with the reference's affine-rate
arithmetic and zero-rate limit (codegen.jl:503-641).
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Set, Tuple

from .parser import (Assign, Binary, Block, Call, CallStmt, EventInitial, Expr, If, Index, Local, ModError,
                     ModFile, Name, Num, Solve, Stmt, Unary, While, parse_mod)

INPUTS = ("v", "t", "dt", "celsius")          # values the runtime supplies, never stored
_MATH = {"exp": "mind_exp", "log": "mind_log", "pow": "mind_pow", "fabs": "fabs", "sqrt": "sqrt",
         "floor": "floor", "ceil": "ceil", "fmin": "fmin", "fmax": "fmax", "log10": "log10",
         "sin": "sin", "cos": "cos", "tanh": "tanh", "expm1": "expm1"}
_NOOP_CALLS = {"at_time"}                     # fixed-step runs ignore them


@dataclass
class Column:
    name: str          # MOD field, "name[k]" for array elements (0-based)
    base: str
    index: int         # -1 for scalars
    default: float
    category: str      # parameter | state | assigned


@dataclass
class MechanismIR:
    """What the emitter and the host builders need from a MOD file."""

    name: str
    kind: str                       # density | point
    columns: List[Column]
    extents: Dict[str, int]         # array fields
    currents: List[str]             # summed into the membrane current, in order
    electrode: List[str]            # subtracted
    receive_args: List[str]
    ion_reads: List[Tuple[str, str]]
    mod: ModFile
    digest: int

    @property
    def field_names(self) -> Tuple[str, ...]:
        return tuple(c.name for c in self.columns)

    @property
    def defaults(self) -> Tuple[float, ...]:
        return tuple(c.default for c in self.columns)

    def column(self, base: str, index: int = -1) -> int:
        for k, c in enumerate(self.columns):
            if c.base == base and c.index == index:
                return k
        raise KeyError(base)


def lower(mod: ModFile, source: str = "") -> MechanismIR:
    """Fields, currents and NET_RECEIVE arity of a parsed MOD file."""
    if mod.kind == "artificial":
        raise ModError(mod.filename, 1, f"{mod.name}: artificial cells are not emitted (the runtime's NetStim "
                                        "is its own device code)")
    if mod.randoms:
        raise ModError(mod.filename, 1, f"{mod.name}: RANDOM variables are not supported in emitted mechanisms")
    columns: List[Column] = []
    extents: Dict[str, int] = {}
    seen: Set[str] = set()
    for category, decls in (("parameter", mod.parameters), ("state", mod.states), ("assigned", mod.assigned)):
        for d in decls:
            if d.name in INPUTS or d.name in seen:
                continue
            seen.add(d.name)
            default = d.default if d.default is not None else 0.0
            if d.extent:
                extents[d.name] = d.extent
                for k in range(d.extent):
                    columns.append(Column(f"{d.name}[{k}]", d.name, k, default, category))
            else:
                columns.append(Column(d.name, d.name, -1, default, category))
    ion_reads = []
    currents = list(mod.nonspecific)
    for ion in mod.ions:
        for r in ion.reads:
            ion_reads.append((r, ion.name))
            if r not in seen:
                seen.add(r)
                columns.append(Column(r, r, -1, 0.0, "assigned"))
        for w in ion.writes:
            if w not in seen:
                seen.add(w)
                columns.append(Column(w, w, -1, 0.0, "assigned"))
        name = "i" + ion.name
        if name in ion.writes and name not in currents:
            currents.append(name)
    for c in currents + list(mod.electrode):
        if c not in seen:
            raise ModError(mod.filename, 1, f"current {c} is not declared")
    receive = mod.blocks.get("net_receive")
    digest = int(hashlib.sha256(source.encode()).hexdigest()[:16], 16) if source else 0
    return MechanismIR(mod.name, mod.kind, columns, extents, currents, list(mod.electrode),
                       receive.args if receive else [], ion_reads, mod, digest)


def _literal(value: float) -> str:
    text = repr(float(value))
    if text in ("inf", "-inf", "nan"):
        raise ValueError(f"non-finite literal {text}")
    if "." not in text and "e" not in text:
        text += ".0"
    return text


@dataclass
class _Scope:
    args: Dict[str, str] = field(default_factory=dict)
    locals_: Dict[str, int] = field(default_factory=dict)
    ret: Optional[str] = None        # FUNCTION name (its return variable)
    derivative: bool = False         # inside a DERIVATIVE block lowered by cnexp


class Emitter:
    """CUDA C for one mechanism (see the module docstring for the phases)."""

    def __init__(self, ir: MechanismIR, cname: str):
        self.ir, self.mod, self.cname = ir, ir.mod, cname
        self.lines: List[str] = []
        self.fields = {c.base for c in ir.columns}
        self.writes_cache: Dict[str, Set[str]] = {}

    # ---- names and expressions
    def err(self, line: int, message: str):
        raise ModError(self.mod.filename, line, message)

    def ref(self, name: str, scope: _Scope, line: int) -> str:
        if scope.ret is not None and name == scope.ret:
            return "ret_"
        if name in scope.args:
            return scope.args[name]
        if name in scope.locals_:
            return f"l_{name}"
        if name in self.fields or name in INPUTS:
            return f"s.{name}"
        if name == "flag" and "flag" in scope.args:
            return scope.args["flag"]
        self.err(line, f"unknown name {name!r}")

    def expr(self, e: Expr, scope: _Scope, line: int) -> Tuple[str, str]:
        """(C code, type) with type "d" (double) or "b" (bool)."""
        if isinstance(e, Num):
            return _literal(e.value), "d"
        if isinstance(e, Name):
            return self.ref(e.name, scope, line), "d"
        if isinstance(e, Index):
            return self.element(e.name, e.index, scope, line), "d"
        if isinstance(e, Unary):
            code, t = self.expr(e.arg, scope, line)
            if e.op == "!":
                return f"(!{self.truth(code, t)})", "b"
            if e.op == "+":
                return self.num(code, t), "d"
            return f"(-{self.num(code, t)})", "d"
        if isinstance(e, Binary):
            a, ta = self.expr(e.left, scope, line)
            b, tb = self.expr(e.right, scope, line)
            if e.op in ("&&", "||"):
                return f"({self.truth(a, ta)} {e.op} {self.truth(b, tb)})", "b"
            if e.op in ("<", ">", "<=", ">=", "==", "!="):
                return f"({self.num(a, ta)} {e.op} {self.num(b, tb)})", "b"
            if e.op == "^":
                return f"mind_pow({self.num(a, ta)}, {self.num(b, tb)})", "d"
            return f"({self.num(a, ta)} {e.op} {self.num(b, tb)})", "d"
        if isinstance(e, Call):
            return self.call(e, scope, line), "d"
        self.err(line, f"unsupported expression {e!r}")

    @staticmethod
    def num(code: str, t: str) -> str:
        return f"({code} ? 1.0 : 0.0)" if t == "b" else code

    @staticmethod
    def truth(code: str, t: str) -> str:
        return code if t == "b" else f"({code} != 0.0)"

    def element(self, name: str, index: Expr, scope: _Scope, line: int) -> str:
        idx, t = self.expr(index, scope, line)
        extent = scope.locals_.get(name) or self.ir.extents.get(name)
        if not extent:
            self.err(line, f"{name} is not an array")
        base = f"l_{name}" if name in scope.locals_ else f"s.{name}"
        # trunc toward zero like Int(trunc(i)); an index outside the array is clamped to it
        return f"{base}[mind_gen_index({self.num(idx, t)}, {extent})]"

    def call(self, c: Call, scope: _Scope, line: int) -> str:
        args = [self.num(*self.expr(a, scope, line)) for a in c.args]
        if c.name in _MATH:
            return f"{_MATH[c.name]}({', '.join(args)})"
        block = self.mod.blocks.get(c.name)
        if block is None or block.kind not in ("procedure", "function", "derivative"):
            if c.name in ("net_send", "net_event", "net_move"):
                self.err(line, f"{c.name} is only supported in artificial cells, which are not emitted")
            self.err(line, f"unknown function {c.name!r}")
        if len(args) != len(block.args):
            self.err(line, f"{c.name} takes {len(block.args)} arguments")
        return f"{block.kind[0]}_{c.name}({', '.join(['s'] + args)})"

    # ---- statements
    def stmts(self, body: List[Stmt], scope: _Scope, indent: int, out: List[str]):
        pad = "    " * indent
        for st in body:
            if isinstance(st, Local):
                for name, extent in st.names:
                    scope.locals_[name] = extent
                    out.append(f"{pad}double l_{name}{f'[{extent}]' if extent else ''} = {{}};" if extent
                               else f"{pad}double l_{name} = 0.0;")
            elif isinstance(st, Assign):
                if st.derivative:
                    if not scope.derivative:
                        self.err(st.line, "a derivative outside a DERIVATIVE block")
                    out.extend(pad + x for x in self.cnexp(st, scope))
                    continue
                if isinstance(st.target, Name) and st.target.name in INPUTS:
                    self.err(st.line, f"{st.target.name} is read-only in this runtime")
                target = (self.element(st.target.name, st.target.index, scope, st.line)
                          if isinstance(st.target, Index) else self.ref(st.target.name, scope, st.line))
                value, t = self.expr(st.value, scope, st.line)
                out.append(f"{pad}{target} = {self.num(value, t)};")
            elif isinstance(st, CallStmt):
                if st.call.name in _NOOP_CALLS:
                    continue
                out.append(f"{pad}{self.call(st.call, scope, st.line)};")
            elif isinstance(st, If):
                cond, t = self.expr(st.cond, scope, st.line)
                out.append(f"{pad}if ({self.truth(cond, t)}) {{")
                self.stmts(st.then, scope, indent + 1, out)
                if st.orelse:
                    out.append(f"{pad}}} else {{")
                    self.stmts(st.orelse, scope, indent + 1, out)
                out.append(f"{pad}}}")
            elif isinstance(st, While):
                cond, t = self.expr(st.cond, scope, st.line)
                # a loop that never ends would hang the GPU: the trip count is bounded
                out.append(f"{pad}for (int guard_ = 0; guard_ < (1 << 20) && {self.truth(cond, t)}; ++guard_) {{")
                self.stmts(st.body, scope, indent + 1, out)
                out.append(f"{pad}}}")
            elif isinstance(st, Solve):
                pass   # hoisted into advance()
            elif isinstance(st, EventInitial):
                pass   # NET_RECEIVE INITIAL: the runtime's events carry no per-edge state
            else:
                self.err(getattr(st, "line", 1), f"unsupported statement {st!r}")

    def cnexp(self, st: Assign, scope: _Scope) -> List[str]:
        name = st.target.name
        if isinstance(st.target, Index):
            self.err(st.line, "cnexp of array states is not supported")
        state = self.ref(name, scope, st.line)
        v = st.value
        if isinstance(v, Binary) and v.op == "/":
            num, tau = v.left, v.right
            tau_ok = isinstance(tau, Num) or (isinstance(tau, Name) and tau.name != name)
            eq = None
            if tau_ok and isinstance(num, Binary) and num.op == "-" and isinstance(num.right, Name) \
                    and num.right.name == name and (isinstance(num.left, Num) or
                                                     (isinstance(num.left, Name) and num.left.name != name)):
                eq = self.num(*self.expr(num.left, scope, st.line))
            elif tau_ok and isinstance(num, Unary) and num.op == "-" and isinstance(num.arg, Name) \
                    and num.arg.name == name:
                eq = "0.0"
            if eq is not None:
                t = self.num(*self.expr(tau, scope, st.line))
                return [f"{state} = {state} + (1.0 - mind_exp(s.dt * (-1.0 / {t}))) * ({eq} - {state});"]
        if self.degree(v, name) > 1:
            self.err(st.line, "cnexp requires an equation affine in its own state")
        rate = self.affine(v, name, scope, st.line)
        return [f"{{ const double x0_ = {state}; const MindAffine r_ = {rate};",
                f"  {state} = x0_ + s.dt * mind_exponential_factor(r_.c * s.dt) * r_.v; }}"]

    def degree(self, e: Expr, name: str) -> int:
        if isinstance(e, Num):
            return 0
        if isinstance(e, Name):
            return int(e.name == name)
        if isinstance(e, Index):
            return int(e.name == name)
        if isinstance(e, Unary):
            return self.degree(e.arg, name)
        if isinstance(e, Binary) and e.op in ("+", "-"):
            return max(self.degree(e.left, name), self.degree(e.right, name))
        if isinstance(e, Binary) and e.op == "*":
            return min(2, self.degree(e.left, name) + self.degree(e.right, name))
        if isinstance(e, Binary) and e.op == "/":
            return self.degree(e.left, name) if self.degree(e.right, name) == 0 else 2
        args = e.args if isinstance(e, Call) else [e.left, e.right]
        return 2 if any(self.degree(a, name) for a in args) else 0

    def affine(self, e: Expr, name: str, scope: _Scope, line: int) -> str:
        if isinstance(e, Name):
            return f"MindAffine{{{self.ref(e.name, scope, line)}, {'1.0' if e.name == name else '0.0'}}}"
        if isinstance(e, Unary) and e.op in ("-", "+"):
            inner = self.affine(e.arg, name, scope, line)
            return f"(-{inner})" if e.op == "-" else inner
        if isinstance(e, Binary) and e.op in ("+", "-", "*", "/"):
            return f"({self.affine(e.left, name, scope, line)} {e.op} {self.affine(e.right, name, scope, line)})"
        return f"MindAffine{{{self.num(*self.expr(e, scope, line))}, 0.0}}"

    # ---- write sets (fields a phase assigns, through the calls it makes)
    def writes(self, body: List[Stmt], stack: Tuple[str, ...] = ()) -> Set[str]:
        out: Set[str] = set()
        local: Set[str] = set()
        for st in body:
            if isinstance(st, Local):
                local |= {n for n, _ in st.names}
            elif isinstance(st, Assign):
                out.add(st.target.name)
                out |= self.expr_writes(st.value, stack)
            elif isinstance(st, CallStmt):
                out |= self.expr_writes(st.call, stack)
            elif isinstance(st, If):
                out |= self.expr_writes(st.cond, stack) | self.writes(st.then, stack) | self.writes(st.orelse, stack)
            elif isinstance(st, While):
                out |= self.expr_writes(st.cond, stack) | self.writes(st.body, stack)
            elif isinstance(st, Solve):
                out |= self.block_writes(st.block, stack)
        return {n for n in out - local if n in self.fields}

    def expr_writes(self, e: Expr, stack) -> Set[str]:
        if isinstance(e, Call):
            out = set()
            for a in e.args:
                out |= self.expr_writes(a, stack)
            if e.name in self.mod.blocks:
                out |= self.block_writes(e.name, stack)
            return out
        if isinstance(e, Binary):
            return self.expr_writes(e.left, stack) | self.expr_writes(e.right, stack)
        if isinstance(e, Unary):
            return self.expr_writes(e.arg, stack)
        if isinstance(e, Index):
            return self.expr_writes(e.index, stack)
        return set()

    def block_writes(self, name: str, stack) -> Set[str]:
        if name in stack:
            self.err(self.mod.blocks[name].line, f"{name} calls itself")
        if name not in self.writes_cache:
            block = self.mod.blocks[name]
            w = self.writes(block.body, stack + (name,)) - set(block.args)
            self.writes_cache[name] = w
        return self.writes_cache[name]

    # ---- functions
    def callable_(self, block: Block) -> List[str]:
        scope = _Scope(args={a: f"a_{a}" for a in block.args})
        is_fn = block.kind == "function"
        if is_fn:
            scope.ret = block.name
        if block.kind == "derivative":
            scope.derivative = True
        params = ", ".join(["S &s"] + [f"double a_{a}" for a in block.args])
        rtype = "double" if is_fn else "void"
        out = [f"    __device__ static __forceinline__ {rtype} {block.kind[0]}_{block.name}({params}) {{"]
        if is_fn:
            out.append("        double ret_ = 0.0;")
        body: List[str] = []
        self.stmts(block.body, scope, 2, body)
        out += body
        if is_fn:
            out.append("        return ret_;")
        out.append("    }")
        return out

    def phase(self, name: str, statements: List[Stmt], scope: _Scope, tail: List[str], rtype: str = "void",
              params: str = "const MindGenRow &r") -> List[str]:
        out = [f"    __device__ static __forceinline__ {rtype} {name}({params}) {{", "        S s;", "        load(s, r);"]
        body: List[str] = []
        self.stmts(statements, scope, 2, body)
        out += body
        written = self.writes(statements)
        for c in self.ir.columns:
            if c.base in written:
                member = f"s.{c.base}" if c.index < 0 else f"s.{c.base}[{c.index}]"
                out.append(f"        r.at({self.ir.column(c.base, c.index)}) = {member};")
        out += tail
        out.append("    }")
        return out

    def emit(self) -> str:
        ir, mod = self.ir, self.mod
        lines = [f"/* {ir.name} ({ir.kind} mechanism), generated from {mod.filename.split('/')[-1]} by",
                 " * mind_b200.nmodl.  Columns: " + ", ".join(f"{k} {c.name}" for k, c in enumerate(ir.columns)) + ". */",
                 f"struct {self.cname} {{",
                 f"    static constexpr int kColumns = {len(ir.columns)};",
                 "    struct S {"]
        for c in ir.columns:
            if c.index < 0:
                lines.append(f"        double {c.base};")
            elif c.index == 0:
                lines.append(f"        double {c.base}[{ir.extents[c.base]}];")
        lines.append("        double v, t, dt, celsius;")
        lines.append("    };")
        lines.append("    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {")
        for k, c in enumerate(ir.columns):
            member = f"s.{c.base}" if c.index < 0 else f"s.{c.base}[{c.index}]"
            lines.append(f"        {member} = r.at({k});")
        lines.append("        s.v = r.v;")
        lines.append("        s.t = r.t;")
        lines.append("        s.dt = r.dt;")
        lines.append("        s.celsius = r.celsius;")
        lines.append("    }")
        # procedures and functions first (callers follow them)
        for block in mod.blocks.values():
            if block.kind in ("procedure", "function"):
                lines += self.callable_(block)
        # derivative blocks lowered by cnexp
        for block in mod.blocks.values():
            if block.kind == "derivative":
                lines += self.callable_(block)
        initial = mod.blocks.get("initial")
        lines += self.phase("initial", initial.body if initial else [], _Scope(), [])
        bp = mod.blocks.get("breakpoint")
        bp_body = bp.body if bp else []
        value = ["        double value = 0.0;"]
        value += [f"        value += s.{c};" for c in ir.currents]
        value += [f"        value -= s.{c};" for c in ir.electrode]
        value += ["        return value;"]
        lines += self.phase("current", [st for st in bp_body if not isinstance(st, Solve)], _Scope(), value,
                            rtype="double")
        solves = [st for st in bp_body if isinstance(st, Solve)]
        adv: List[Stmt] = []
        for st in solves:
            block = mod.blocks.get(st.block)
            if block is None:
                self.err(st.line, f"SOLVE of an unknown block {st.block}")
            if block.kind == "derivative" and st.method not in ("cnexp", ""):
                self.err(st.line, f"METHOD {st.method} is not supported (cnexp is)")
            if block.kind == "procedure" and st.method not in ("after_cvode", ""):
                self.err(st.line, f"METHOD {st.method} for a PROCEDURE is not supported")
            adv.append(CallStmt(Call(st.block, []), st.line))
        if not ir.currents and not ir.electrode:
            adv += [st for st in bp_body if not isinstance(st, Solve)]
        lines += self.phase("advance", adv, _Scope(), [])
        rec = mod.blocks.get("net_receive")
        if rec is not None:
            if len(rec.args) < 1:
                self.err(rec.line, "NET_RECEIVE needs its weight argument")
            scope = _Scope(args={rec.args[0]: "w_", "flag": "flag_"})
            for extra in rec.args[1:]:
                scope.locals_[extra] = 0   # further weights are not carried by this runtime's NetCons
            body = [f"        double l_{a} = 0.0;" for a in rec.args[1:]]
            code = self.phase("receive", rec.body, scope, [], params="const MindGenRow &r, double w_, double flag_")
            lines += code[:3] + body + code[3:]
        lines.append("};")
        return "\n".join(lines)


def emit_mechanism(ir: MechanismIR, cname: str) -> str:
    return Emitter(ir, cname).emit()


def compile_source(source: str, filename: str = "<string>") -> MechanismIR:
    """Parse and lower a MOD source (compile_mod, src/compiler/frontend.jl:85-110)."""
    return lower(parse_mod(source, filename), source)
