"""A translator for the Fortran 90 subset used by the reference's STEP_7 step
routines, producing Python that follows Fortran's arithmetic rules.

No Fortran compiler exists in this image, so the reference program cannot be
built.  To pin the CPU oracle to the reference itself, this module reads the
reference's own .f90 source text and executes it:

* types: declared kinds (REAL(dp) = float64, default REAL = float32,
  INTEGER = int); undeclared names follow implicit typing (i-n INTEGER,
  otherwise default REAL) in program units without `implicit none`;
* mixed-mode arithmetic promotes to the wider operand kind; float32 operations
  round to float32 (numpy float32 scalars); INTEGER division truncates;
* `x**2.0d0` (a real power with value 2) is x*x, which is how gfortran
  expands it; other real powers call pow;
* literals: `1.0d0` is REAL(8), `1.` / `273.0` are default REAL (float32);
* evaluation follows the parse tree: chains of + and * associate left to
  right, a leading sign applies to the whole first term.

Only what STEP_7's step and initialisation routines use is supported: module
declarations, allocate, DO loops, IF blocks, assignments (scalar, element and
whole-array), CALL, and the intrinsics tanh, sqrt, acos, abs, int, float,
real, dble, mod.  I/O statements are skipped except the list-directed reads of
input.dat in setup, which take their values from a parameter dictionary.
`do concurrent (i=a:b)` with one index (STEP_DOCONCURRENT's BC_g) runs as a
sequential DO loop, which is one of the orders the construct allows; cpp
conditionals are resolved against the macros a Program is given.
"""
from __future__ import annotations

import math
import re
from pathlib import Path

import numpy as np

F32 = np.float32
RANK = {"i": 0, "r4": 1, "r8": 2}


# --------------------------------------------------------------- preprocessing

def _strip_comment(line: str) -> str:
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def preprocess(text: str, defined=()) -> list[str]:
    """cpp conditionals (the macros in `defined`), comments, continuations."""
    lines, stack = [], []
    for raw in text.splitlines():
        s = raw.strip()
        if s.startswith("#"):
            tok = s.split()
            if tok[0] == "#ifdef":
                stack.append(tok[1] in defined)
            elif tok[0] == "#ifndef":
                stack.append(tok[1] not in defined)
            elif tok[0] == "#else":
                stack[-1] = not stack[-1]
            elif tok[0] == "#endif":
                stack.pop()
            continue
        if not all(stack):
            continue
        lines.append(_strip_comment(raw).rstrip())
    stmts, cur = [], ""
    for ln in lines:
        t = ln.strip()
        if cur:
            if t.startswith("&"):
                t = t[1:]
            cur += " " + t
        else:
            cur = t
        if cur.endswith("&"):
            cur = cur[:-1]
            continue
        if cur.strip():
            stmts.append(cur.strip())
        cur = ""
    return stmts


# ------------------------------------------------------------------- lexing

TOKEN = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([edED][+-]?\d+)?(_\w+)?)
  | (?P<dotop>\.(eq|ne|lt|le|gt|ge|and|or|not|true|false)\.)
  | (?P<name>[A-Za-z_]\w*)
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<op>\*\*|==|/=|<=|>=|::|[-+*/(),=:<>%])
  | (?P<ws>\s+)
""", re.X | re.I)


def lex(s: str):
    out, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot lex {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        out.append((kind, m.group(kind).lower() if kind != "str" else m.group(kind)))
    return out


# ------------------------------------------------------------------ parsing

class P:
    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError(f"expected {val!r}, got {tok}")
        self.i += 1
        return tok

    def at(self, *vals):
        return self.peek()[1] in vals

    # expr := or_expr
    def expr(self):
        return self.or_()

    def or_(self):
        a = self.and_()
        while self.at(".or."):
            self.take()
            a = ("or", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.at(".and."):
            self.take()
            a = ("and", a, self.not_())
        return a

    def not_(self):
        if self.at(".not."):
            self.take()
            return ("not", self.not_())
        return self.rel()

    REL = {".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">=",
           "==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}

    def rel(self):
        a = self.add()
        if self.peek()[1] in self.REL:
            op = self.REL[self.take()[1]]
            a = ("rel", op, a, self.add())
        return a

    def add(self):
        # level-2: [sign] add_operand { (+|-) add_operand }
        if self.at("+", "-"):
            sign = self.take()[1]
            a = self.mul()
            if sign == "-":
                a = ("neg", a)
        else:
            a = self.mul()
        while self.at("+", "-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.pow_()
        while self.at("*", "/"):
            op = self.take()[1]
            a = ("bin", op, a, self.pow_())
        return a

    def pow_(self):
        a = self.primary()
        if self.at("**"):
            self.take()
            # the exponent is a mult-operand: may carry its own sign
            if self.at("+", "-"):
                s = self.take()[1]
                b = self.pow_()
                b = ("neg", b) if s == "-" else b
            else:
                b = self.pow_()
            a = ("pow", a, b)
        return a

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return ("num", val)
        if kind == "dotop" and val in (".true.", ".false."):
            self.take()
            return ("logical", val == ".true.")
        if kind == "str":
            self.take()
            return ("str", val)
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return ("paren", e)
        if kind == "name":
            self.take()
            if self.at("("):
                self.take()
                args = []
                if not self.at(")"):
                    while True:
                        args.append(self.slice_or_expr())
                        if self.at(","):
                            self.take()
                            continue
                        break
                self.take(")")
                return ("call", val, args)
            return ("var", val)
        raise SyntaxError(f"unexpected token {kind} {val}")

    def slice_or_expr(self):
        if self.at(":"):
            self.take()
            lo = None
        else:
            lo = self.expr()
            if not self.at(":"):
                return lo
            self.take()
        hi = None if self.at(",", ")") else self.expr()
        return ("slice", lo, hi)


# ----------------------------------------------------------- symbol tables

class Sym:
    def __init__(self, name, typ, dims=None, alloc=False):
        self.name, self.typ, self.dims, self.alloc = name, typ, dims, alloc


def implicit_type(name: str) -> str:
    return "i" if name[0] in "ijklmn" else "r4"


def decl_type(spec: str, kinds: dict) -> str:
    spec = spec.replace(" ", "")
    if spec.startswith("integer"):
        return "i"
    if spec.startswith("real"):
        m = re.search(r"kind=(\w+)", spec) or re.search(r"real\((\w+)\)", spec)
        if not m:
            return "r4"
        k = m.group(1)
        k = kinds.get(k, k)
        return "r8" if str(k) == "8" else "r4"
    if spec.startswith("character"):
        return "c"
    if spec.startswith("logical"):
        return "l"
    raise SyntaxError(spec)


# ------------------------------------------------------------------ codegen

INTRINSIC_TYPE = {"tanh": None, "sqrt": None, "acos": None, "abs": None, "int": "i", "float": "r4",
                  "real": "r4", "dble": "r8", "mod": None, "min": None, "max": None, "exp": None}


class Unit:
    """One subroutine translated to a Python function."""

    def __init__(self, name, stmts, module, implicit_none):
        self.name, self.stmts, self.module = name, stmts, module
        self.implicit_none = implicit_none
        self.locals: dict[str, Sym] = {}
        self.assigned_globals = set()

    def sym(self, name):
        if name in self.locals:
            return self.locals[name]
        if name in self.module:
            return self.module[name]
        if self.implicit_none:
            raise NameError(f"{name} undeclared in {self.name}")
        s = Sym(name, implicit_type(name))
        self.locals[name] = s
        return s

    # expression -> (python code, type)
    def ex(self, e):
        k = e[0]
        if k == "num":
            v = e[1]
            m = re.fullmatch(r"([\d.]+)(?:([ed])([+-]?\d+))?(?:_(\w+))?", v)
            mant, ech, exp, kind = m.groups()
            if "." not in mant and ech is None:
                return (str(int(mant)), "i")
            txt = mant + (f"e{exp}" if exp else "")
            if ech == "d" or kind in ("dp", "8"):
                return (repr(float(txt)), "r8")
            return (f"F32({repr(float(txt))})", "r4")
        if k == "logical":
            return (repr(e[1]), "l")
        if k == "paren":
            c, t = self.ex(e[1])
            return (f"({c})", t)
        if k == "var":
            s = self.sym(e[1])
            return (e[1], s.typ)
        if k == "neg":
            c, t = self.ex(e[1])
            return (f"(-{c})", t)
        if k == "not":
            c, _ = self.ex(e[1])
            return (f"(not {c})", "l")
        if k in ("and", "or"):
            a, _ = self.ex(e[1])
            b, _ = self.ex(e[2])
            return (f"({a} {k} {b})", "l")
        if k == "rel":
            (a, ta), (b, tb) = self.ex(e[2]), self.ex(e[3])
            t = max(ta, tb, key=lambda x: RANK.get(x, 0))
            return (f"({self.conv(a, ta, t)} {e[1]} {self.conv(b, tb, t)})", "l")
        if k == "bin":
            op = e[1]
            (a, ta), (b, tb) = self.ex(e[2]), self.ex(e[3])
            t = max(ta, tb, key=lambda x: RANK[x])
            a, b = self.conv(a, ta, t), self.conv(b, tb, t)
            if t == "i" and op == "/":
                return (f"idiv({a}, {b})", "i")
            return (f"({a} {op} {b})", t)
        if k == "pow":
            (a, ta) = self.ex(e[1])
            be = e[2]
            inner = be[1] if be[0] == "paren" else be
            if inner[0] == "num":
                bc, bt = self.ex(inner)
                bv = float(eval(bc, {"F32": F32}))
                if bv == 2.0:
                    t = ta if bt == "i" else max(ta, bt, key=lambda x: RANK[x])
                    return (f"sq({self.conv(a, ta, t)})", t)
                if bt == "i":
                    return (f"ipow({a}, {int(bv)})", ta)
            (b, tb) = self.ex(be)
            t = max(ta, tb, key=lambda x: RANK[x])
            if t == "i":
                return (f"ipow({a}, {b})", "i")
            return (f"math.pow({self.conv(a, ta, 'r8')}, {self.conv(b, tb, 'r8')})", "r8")
        if k == "call":
            name, args = e[1], e[2]
            if name in INTRINSIC_TYPE and not self.is_array(name):
                return self.intrinsic(name, args)
            s = self.sym(name)
            idx = self.index(s, args)
            return (f"{name}[{idx}]", s.typ)
        raise SyntaxError(f"cannot translate {e}")

    def is_array(self, name):
        s = self.locals.get(name) or self.module.get(name)
        return bool(s and s.dims is not None)

    def intrinsic(self, name, args):
        cs = [self.ex(a) for a in args]
        if name == "tanh":
            c, t = cs[0]
            return (f"math.tanh({c})", "r8") if t == "r8" else (f"F32(math.tanh(float({c})))", "r4")
        if name in ("sqrt", "acos", "exp"):
            c, t = cs[0]
            return (f"math.{name}({self.conv(c, t, 'r8')})", "r8") if t == "r8" else \
                (f"F32(math.{name}(float({c})))", "r4")
        if name == "abs":
            c, t = cs[0]
            return (f"abs({c})", t)
        if name == "int":
            c, t = cs[0]
            return (f"int({c})", "i")
        if name in ("float", "real"):
            c, t = cs[0]
            return (f"F32({c})", "r4")
        if name == "dble":
            c, t = cs[0]
            return (f"float({c})", "r8")
        if name == "mod":
            (a, ta), (b, tb) = cs
            return (f"fmod_({a}, {b})", max(ta, tb, key=lambda x: RANK[x]))
        raise NotImplementedError(name)

    @staticmethod
    def conv(code, frm, to):
        if frm == to or to in ("l", "c"):
            return code
        if to == "r8":
            return f"float({code})"
        if to == "r4":
            return f"F32({code})"
        if to == "i":
            return f"int({code})"
        return code

    def index(self, s, args):
        if s.dims is None:
            raise SyntaxError(f"{s.name} is not an array")
        parts = []
        stride = "1"
        for d, a in enumerate(args):
            c, t = self.ex(a)
            lo = f"{s.name}__lo{d}"
            parts.append(f"({c} - {lo})" + ("" if d == 0 else f" * {s.name}__n0" if d == 1 else ""))
        return " + ".join(parts)

    # statements -> python lines
    def gen(self):
        body, i = [], 0
        out = self.block(0, body)
        params = "".join(f"    global {g}\n" for g in sorted(self.assigned_globals))
        return f"def {self.name}():\n" + params + ("\n".join(out) if out else "    pass") + "\n"

    def block(self, depth, _unused):
        lines = []
        ind = "    " * (depth + 1)
        while self.pos < len(self.stmts):
            st = self.stmts[self.pos]
            low = st.lower()
            key = re.sub(r"\s+", " ", low)
            if re.match(r"^(end ?do|enddo|end ?if|endif|else|else ?if\b.*|end subroutine.*|end)$", key) or \
                    re.match(r"^else ?if\s*\(", key):
                return lines
            self.pos += 1
            lines.extend(self.statement(st, key, ind, depth))
        return lines

    def statement(self, st, key, ind, depth):
        if re.match(r"^(use |implicit |write|open|close|flush|print|return$)", key):
            return []
        if key.startswith("read"):
            m = re.match(r"read\s*\(\s*112\s*,\s*\*\s*\)\s*id\(\d+\)\s*,\s*(\w+)", key)
            if m:
                var = m.group(1)
                s = self.sym(var)
                self.note_assign(var)
                return [f"{ind}{var} = {self.conv('PARAMS[%r]' % var, 'r8' if s.typ != 'i' else 'i', s.typ)}"]
            return []
        if re.match(r"^(real|integer|character|logical|double)", key) and ("::" in key or key.startswith("character")):
            self.declare(st)
            return []
        if key.startswith("allocate"):
            return self.allocate(st, ind)
        mc = re.match(r"^do concurrent\s*\(\s*(\w+)\s*=\s*([^:]+):([^:]+)\)$", key)
        if mc:
            key = f"do {mc.group(1)} = {mc.group(2)}, {mc.group(3)}"
        m = re.match(r"^do\s+(\w+)\s*=\s*(.+)$", key)
        if m:
            var = m.group(1)
            self.note_assign(var)
            p = P(lex(m.group(2)))
            a = p.expr(); p.take(","); b = p.expr()
            step = None
            if p.at(","):
                p.take(); step = p.expr()
            ca, _ = self.ex(a); cb, _ = self.ex(b)
            rng = f"range({ca}, ({cb}) + 1)" if step is None else f"range({ca}, ({cb}) + 1, {self.ex(step)[0]})"
            out = [f"{ind}for {var} in {rng}:"]
            inner = self.block(depth + 1, None)
            end = self.stmts[self.pos].lower().replace(" ", "")
            assert end in ("enddo", "end do".replace(" ", "")), end
            self.pos += 1
            return out + (inner or [ind + "    pass"])
        m = re.match(r"^if\s*\((.*)\)\s*then$", key)
        if m:
            return self.if_block(st, ind, depth)
        m = re.match(r"^if\s*\(", key)
        if m:
            p = P(lex(st[2:].strip()))
            p.take("(")
            cond = p.expr()
            p.take(")")
            rest = st[2:].strip()
            # the statement after the condition
            depth_ = 0
            for k, ch in enumerate(rest):
                if ch == "(":
                    depth_ += 1
                elif ch == ")":
                    depth_ -= 1
                    if depth_ == 0:
                        tail = rest[k + 1:].strip()
                        break
            c, _ = self.ex(cond)
            inner = self.statement(tail, re.sub(r"\s+", " ", tail.lower()), ind + "    ", depth + 1)
            return [f"{ind}if {c}:"] + (inner or [ind + "    pass"])
        m = re.match(r"^call\s+(\w+)", key)
        if m:
            return [f"{ind}{m.group(1)}()"]
        if key in ("stop",):
            return [f"{ind}raise RuntimeError('stop')"]
        return self.assignment(st, ind)

    def if_block(self, st, ind, depth):
        out = []
        first = True
        while True:
            key = re.sub(r"\s+", " ", st.lower())
            if first:
                cond_txt = re.match(r"^if\s*\((.*)\)\s*then$", key).group(1)
            else:
                m = re.match(r"^else ?if\s*\((.*)\)\s*then$", key)
                cond_txt = m.group(1) if m else None
            if cond_txt is not None:
                c, _ = self.ex(P(lex(cond_txt)).expr())
                out.append(f"{ind}{'if' if first else 'elif'} {c}:")
            else:
                out.append(f"{ind}else:")
            first = False
            inner = self.block(depth + 1, None)
            out.extend(inner or [ind + "    pass"])
            st = self.stmts[self.pos]
            self.pos += 1
            k2 = re.sub(r"\s+", "", st.lower())
            if k2 in ("endif",):
                return out

    def note_assign(self, var):
        if var not in self.locals and var in self.module:
            self.assigned_globals.add(var)

    def assignment(self, st, ind):
        toks = lex(st)
        p = P(toks)
        kind, name = p.take()
        if kind != "name":
            raise SyntaxError(st)
        s = self.sym(name)
        self.note_assign(name)
        if p.at("("):
            p.take("(")
            args = []
            while True:
                args.append(p.slice_or_expr())
                if p.at(","):
                    p.take(); continue
                break
            p.take(")")
            p.take("=")
            rhs = p.expr()
            if any(a[0] == "slice" for a in args):
                return self.whole_assign(name, s, rhs, ind)
            c, t = self.ex(rhs)
            return [f"{ind}{name}[{self.index(s, args)}] = {self.conv(c, t, s.typ)}"]
        p.take("=")
        rhs = p.expr()
        if s.dims is not None:
            return self.whole_assign(name, s, rhs, ind)
        c, t = self.ex(rhs)
        return [f"{ind}{name} = {self.conv(c, t, s.typ)}"]

    def whole_assign(self, name, s, rhs, ind):
        r = rhs
        while r[0] == "call" and r[2] and all(a[0] == "slice" for a in r[2]):
            r = ("var", r[1])
        if r[0] == "var" and self.is_array(r[1]):
            return [f"{ind}{name}[:] = {r[1]}"]
        c, t = self.ex(rhs)
        return [f"{ind}{name}[:] = [{self.conv(c, t, s.typ)}] * len({name})"]

    def declare(self, st):
        head, _, names = st.partition("::") if "::" in st else (st.split()[0], None, " ".join(st.split()[1:]))
        typ = decl_type(head.lower(), KINDS)
        alloc = "allocatable" in head.lower()
        param = "parameter" in head.lower()
        for part in split_top(names):
            part = part.strip()
            if not part:
                continue
            m = re.match(r"(\w+)\s*(\((.*)\))?\s*(=\s*(.*))?$", part)
            nm, dims = m.group(1).lower(), m.group(3)
            sym = Sym(nm, typ, dims=[d.strip() for d in split_top(dims)] if dims else None, alloc=alloc)
            self.locals[nm] = sym

    def allocate(self, st, ind):
        inner = st[st.index("(") + 1: st.rindex(")")]
        out = []
        for item in split_top(inner):
            m = re.match(r"\s*(\w+)\s*\((.*)\)\s*$", item)
            nm, dims = m.group(1).lower(), split_top(m.group(2))
            s = self.sym(nm)
            los, ns = [], []
            for d in dims:
                lo, hi = (d.split(":") + [None])[:2] if ":" in d else ("1", d)
                cl, _ = self.ex(P(lex(lo)).expr())
                ch, _ = self.ex(P(lex(hi)).expr())
                los.append(cl)
                ns.append(f"(({ch}) - ({cl}) + 1)")
            zero = "F32(0.0)" if s.typ == "r4" else ("0" if s.typ == "i" else "0.0")
            size = " * ".join(ns)
            out.append(f"{ind}{nm} = [{zero}] * ({size})")
            self.assigned_globals.add(nm)
            for d, lo in enumerate(los):
                out.append(f"{ind}{nm}__lo{d} = {lo}")
                self.assigned_globals.add(f"{nm}__lo{d}")
            out.append(f"{ind}{nm}__n0 = {ns[0]}")
            self.assigned_globals.add(f"{nm}__n0")
        return out


KINDS: dict = {}


def split_top(s):
    if s is None:
        return []
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


# ---------------------------------------------------------------- programme

def parse_module(path: Path):
    """module shared: kinds, scalars and allocatable arrays."""
    stmts = preprocess(path.read_text())
    module: dict[str, Sym] = {}
    init = []
    for st in stmts:
        low = re.sub(r"\s+", " ", st.lower())
        if low.startswith(("module", "end module", "implicit", "use ")):
            continue
        if "::" not in low:
            continue
        head, _, names = st.partition("::")
        hl = head.lower().replace(" ", "")
        if "parameter" in hl:
            for part in split_top(names):
                m = re.match(r"\s*(\w+)\s*=\s*(.*)$", part)
                nm, val = m.group(1).lower(), m.group(2).strip().lower()
                if hl.startswith("integer"):
                    if val.startswith("selected_real_kind(15"):
                        KINDS[nm] = 8
                    elif val.startswith("kind(1.)"):
                        KINDS[nm] = 4
                    elif val in KINDS:
                        KINDS[nm] = KINDS[val]
                    else:
                        init.append((nm, "i", val))
                    module[nm] = Sym(nm, "i")
                else:
                    typ = decl_type(hl, KINDS)
                    module[nm] = Sym(nm, typ)
                    init.append((nm, typ, val))
            continue
        typ = decl_type(hl, KINDS)
        for part in split_top(names):
            m = re.match(r"\s*(\w+)\s*(\((.*)\))?", part)
            if not m:
                continue
            nm = m.group(1).lower()
            dims = m.group(3)
            module[nm] = Sym(nm, typ, dims=split_top(dims) if dims else None, alloc="allocatable" in hl)
    return module, init


def subroutine_units(path: Path, module, defined=()):
    stmts = preprocess(path.read_text(), defined)
    units = []
    i = 0
    while i < len(stmts):
        low = stmts[i].lower().strip()
        m = re.match(r"^subroutine\s+(\w+)", low)
        if not m:
            i += 1
            continue
        name = m.group(1)
        j = i + 1
        while not re.match(r"^end\s*subroutine", stmts[j].lower().strip()):
            j += 1
        body = stmts[i + 1: j + 1]
        implicit_none = any(s.lower().replace(" ", "") == "implicitnone" for s in body)
        u = Unit(name, body, module, implicit_none)
        u.pos = 0
        units.append(u)
        i = j + 1
    return units


PRELUDE = '''
import math
import numpy as np
F32 = np.float32

def sq(x):
    return x * x

def idiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q

def ipow(a, n):
    r = a
    for _ in range(int(n) - 1):
        r = r * a
    return r

def fmod_(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return a - idiv(a, b) * b
    return math.fmod(a, b)
'''


class Program:
    """The reference's STEP_7 subroutines, executable from Python."""

    def __init__(self, ref_dir: Path, files, defined=()):
        """files: names in ref_dir, or paths (e.g. a sibling variant's file
        that replaces one routine); defined: cpp macros."""
        self.module, init = parse_module(ref_dir / "shared.f90")
        src = [PRELUDE]
        for nm, typ, val in init:
            u = Unit("_init", [], self.module, True)
            c, t = u.ex(P(lex(val)).expr())
            src.append(f"{nm} = {Unit.conv(c, t, typ)}")
        for nm, s in self.module.items():
            if s.dims is not None and not s.alloc:
                # fixed-size module array, e.g. cx(0:8)
                los, ns = [], []
                for d in s.dims:
                    lo, hi = d.split(":") if ":" in d else ("1", d)
                    los.append(int(lo)); ns.append(int(hi) - int(lo) + 1)
                zero = "F32(0.0)" if s.typ == "r4" else ("0" if s.typ == "i" else ("0.0" if s.typ == "r8" else "None"))
                src.append(f"{nm} = [{zero}] * {int(np.prod(ns))}")
                for d, lo in enumerate(los):
                    src.append(f"{nm}__lo{d} = {lo}")
                src.append(f"{nm}__n0 = {ns[0]}")
                continue
            if s.dims is None and not any(nm == x[0] for x in init):
                src.append(f"{nm} = {'0' if s.typ == 'i' else ('F32(0.0)' if s.typ == 'r4' else ('0.0' if s.typ == 'r8' else 'None'))}")
        self.units = {}
        for f in files:
            for u in subroutine_units(ref_dir / f, self.module, defined):
                code = u.gen()
                self.units[u.name] = code
                src.append(code)
        self.source = "\n".join(src)
        self.ns: dict = {}
        exec(compile(self.source, "<STEP_7>", "exec"), self.ns)

    def set_params(self, params: dict):
        self.ns["PARAMS"] = {k.lower(): v for k, v in params.items()}

    def call(self, name):
        self.ns[name.lower()]()

    def array(self, name, Nx, Ny) -> np.ndarray:
        a = np.array(self.ns[name.lower()], dtype=np.float64)
        return a.reshape(Ny + 2, Nx + 2)

    def scalar(self, name):
        return self.ns[name.lower()]
