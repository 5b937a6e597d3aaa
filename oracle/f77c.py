"""Fortran-77 to C translator for the reference program -- TEST INFRASTRUCTURE ONLY.

No Fortran compiler exists on these machines, so the reference (t3dsdsc.f with its include
files mhd01.for, mhd02.for, mhd03.for) cannot be built as it is.  This translator turns the
reference's own source, read where it lies, into one C file that gcc builds into a shared
library under oracle/_ref/ (git-ignored; nothing of the reference is committed).  The tests use
that library to check the oracle restatement against the reference itself.

It handles the subset of Fortran 77 (with the few Fortran 90 forms) that the reference uses:
fixed-form source with tab forms, `!` comments, `;` separators and the 72-column limit;
implicit typing; PARAMETER, DIMENSION, COMMON, INTEGER, REAL*8, DOUBLE PRECISION, LOGICAL,
CHARACTER declarations; statement functions; labelled and block DO loops (shared terminal
labels, EXIT), block and logical IF, GOTO, CONTINUE, CALL, RETURN, STOP.  Semantics kept:
column-major arrays with their declared bounds, arguments by reference, COMMON blocks as one
contiguous object each, local arrays static, DO trip counts fixed on entry, REAL*4 literals and
arithmetic (an unsuffixed real constant is single precision: `0.15` is the float 0.15, and
`5.0/3.0` is computed in single precision), integer division truncating toward zero,
integer powers by repeated multiplication.  Input/output statements (OPEN, READ, WRITE,
PRINT, CLOSE, INQUIRE, FORMAT) are dropped; any statement outside the subset, and every
routine named in `stubs`, becomes a call that aborts the run if it is ever reached.  MPI
calls go to a one-process stub (mpi_stub.c).

Edits of the reference are not made in its source but passed to `translate`:
  params   {name: value} overriding PARAMETER constants (grid sizes, process grid);
  assign   {(routine, variable): c_expression} replacing the right-hand side of every
           assignment to that variable in that routine (run-time flags of mhd03.for);
  stubs    routines whose body is replaced by an abort (file output, grid generators not used).
"""
from __future__ import annotations

import math
import os
import re
import sys

INTRINSIC_TYPES = {"integer": "i", "real": "f", "real*4": "f", "real*8": "d", "double precision": "d",
                   "logical": "l", "character": "c"}

# the constants of mpif.h the reference uses, with the values of the one-process stub
MPIF = {
    "mpi_comm_world": 91, "mpi_status_size": 4, "mpi_proc_null": -2, "mpi_double_precision": 11,
    "mpi_real8": 11, "mpi_integer": 7, "mpi_real": 10, "mpi_min": 101, "mpi_max": 102, "mpi_sum": 103,
    "mpi_logical": 8, "mpi_character": 9, "mpi_any_source": -1, "mpi_any_tag": -1, "mpi_success": 0,
}


class F77Error(Exception):
    pass


# ----------------------------------------------------------------------------------------------
# source reading
# ----------------------------------------------------------------------------------------------

def _strip_bang(text: str) -> str:
    out, q = [], None
    for ch in text:
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


def read_fixed(path: str):
    """Fixed-form lines -> [(label or None, text, file:line)] with continuations joined and
    includes spliced."""
    base = os.path.dirname(path)
    stmts = []
    with open(path, encoding="latin-1") as f:
        raw = f.read().split("\n")
    cur = None
    for ln, line in enumerate(raw, 1):
        line = line.rstrip("\r")
        if not line.strip():
            continue
        if line[0] in "cC*!":
            continue
        if line[0] == "\t":                                   # tab form: statement from column 7
            rest = line[1:]
            if rest[:1] in "123456789" and rest[:1] != "":
                label, cont, body = "", True, rest[1:]
            else:
                label, cont, body = "", False, rest
        else:
            line = line.expandtabs(8)
            label, contc, body = line[:5], line[5:6], line[6:72]
            cont = contc not in ("", " ", "0")
        body = _strip_bang(body)
        if cont:
            if cur is None:
                raise F77Error(f"{path}:{ln}: continuation without a statement")
            cur[1] += body
            continue
        if cur is not None:
            stmts.append(tuple(cur))
        lab = label.strip()
        cur = [int(lab) if lab else None, body, f"{os.path.basename(path)}:{ln}"]
    if cur is not None:
        stmts.append(tuple(cur))
    out = []
    for lab, text, where in stmts:
        parts = _split_semicolons(text)
        for q, p in enumerate(parts):
            if not p.strip() and not (q == 0 and lab):
                continue
            m = re.match(r"\s*include\s*'([^']+)'\s*$", p, re.I)
            if m:
                name = m.group(1)
                if name.lower() == "mpif.h":
                    out.append((None, "!mpif", where))
                    continue
                out.extend(read_fixed(os.path.join(base, name)))
                continue
            out.append((lab if q == 0 else None, p, where))
    return out


def _split_semicolons(text):
    parts, cur, q = [], [], None
    for ch in text:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == ";":
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def lower_code(text: str) -> str:
    out, q = [], None
    for ch in text:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


# ----------------------------------------------------------------------------------------------
# expressions
# ----------------------------------------------------------------------------------------------

TOKEN = re.compile(r"""
    (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][+-]?\d+)?)
  | (?P<dotop>\.(?:and|or|not|eqv|neqv|eq|ne|lt|le|gt|ge|true|false)\.)
  | (?P<name>[a-z_][a-z0-9_$]*)
  | (?P<str>'(?:[^']|'')*')
  | (?P<op>\*\*|//|/=|==|<=|>=|[-+*/(),:=<>])
  | (?P<ws>\s+)
""", re.X | re.I)


def tokenize(s: str):
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise F77Error(f"cannot tokenize {s[pos:pos + 20]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        v = m.group(kind)
        if kind == "num":
            # a number followed by a dot-operator: "1.eq." lexes as "1." + "eq." -> fix
            nxt = s[pos:pos + 5].lower()
            if v.endswith(".") and re.match(r"(and|or|not|eqv|neqv|eq|ne|lt|le|gt|ge|true|false)\.", s[pos:].lower()):
                v = v[:-1]
                pos -= 1
            del nxt
        toks.append((kind, v.lower() if kind != "str" else v))
    return toks


class Node:
    __slots__ = ("k", "a", "t")

    def __init__(self, k, *a):
        self.k, self.a, self.t = k, a, None

    def __repr__(self):
        return f"{self.k}{self.a}"


class Parser:
    """Fortran expression precedence: ** (right) > * / > unary +- > binary +- > // >
    relational > .not. > .and. > .or. > .eqv. .neqv."""
    REL = {".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">=",
           "==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}

    def __init__(self, toks):
        self.t, self.p = toks, 0

    def peek(self, o=0):
        return self.t[self.p + o] if self.p + o < len(self.t) else (None, None)

    def take(self, v=None):
        tok = self.peek()
        if v is not None and tok[1] != v:
            raise F77Error(f"expected {v!r}, got {tok!r}")
        self.p += 1
        return tok

    def parse(self):
        e = self.eqv()
        if self.p != len(self.t):
            raise F77Error(f"trailing tokens {self.t[self.p:]}")
        return e

    def eqv(self):
        e = self.lor()
        while self.peek()[1] in (".eqv.", ".neqv."):
            op = self.take()[1]
            e = Node("bin", "==" if op == ".eqv." else "!=", e, self.lor())
        return e

    def lor(self):
        e = self.land()
        while self.peek()[1] == ".or.":
            self.take()
            e = Node("bin", "||", e, self.land())
        return e

    def land(self):
        e = self.lnot()
        while self.peek()[1] == ".and.":
            self.take()
            e = Node("bin", "&&", e, self.lnot())
        return e

    def lnot(self):
        if self.peek()[1] == ".not.":
            self.take()
            return Node("not", self.lnot())
        return self.rel()

    def rel(self):
        e = self.concat()
        if self.peek()[1] in self.REL:
            op = self.REL[self.take()[1]]
            e = Node("bin", op, e, self.concat())
        return e

    def concat(self):
        e = self.add()
        while self.peek()[1] == "//":
            self.take()
            e = Node("concat", e, self.add())
        return e

    def add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            e = self.mul()
            e = Node("neg", e) if op == "-" else e
        else:
            e = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            e = Node("bin", op, e, self.mul())
        return e

    def mul(self):
        e = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            e = Node("bin", op, e, self.power())
        return e

    def power(self):
        b = self.primary()
        if self.peek()[1] == "**":
            self.take()
            if self.peek()[1] in ("+", "-"):       # a**-b
                op = self.take()[1]
                ex = self.power()
                ex = Node("neg", ex) if op == "-" else ex
            else:
                ex = self.power()
            return Node("pow", b, ex)
        return b

    def primary(self):
        kind, v = self.take()
        if kind == "num":
            return Node("num", v)
        if kind == "str":
            return Node("str", v)
        if kind == "dotop" and v in (".true.", ".false."):
            return Node("lit", v == ".true.")
        if v == "(":
            e = self.eqv()
            self.take(")")
            return e
        if kind == "name":
            if self.peek()[1] == "(":
                self.take("(")
                args = []
                if self.peek()[1] != ")":
                    while True:
                        if self.peek()[1] == ":":          # substring / section: unsupported
                            raise F77Error("substring")
                        args.append(self.eqv())
                        if self.peek()[1] == ":":
                            raise F77Error("substring")
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return Node("call", v, args)
            return Node("name", v)
        raise F77Error(f"unexpected token {v!r}")


def parse_expr(s: str) -> Node:
    return Parser(tokenize(s)).parse()


# ----------------------------------------------------------------------------------------------
# program units
# ----------------------------------------------------------------------------------------------

class Sym:
    def __init__(self, name):
        self.name = name
        self.type = None          # 'i' 'f' 'd' 'l' 'c'
        self.dims = None          # [(lo_expr, hi_expr)] Fortran expressions (strings)
        self.common = None        # common block name
        self.dummy = False
        self.param = None         # PARAMETER value (python number)
        self.stmtfn = None        # (args, Node)
        self.external = False
        self.charlen = None


class Unit:
    def __init__(self, kind, name, args, where):
        self.kind, self.name, self.args, self.where = kind, name, args, where
        self.syms = {}
        self.implicit = {}
        self.body = []            # (label, text, where)
        self.decl_done = False
        self.rettype = None

    def sym(self, n):
        if n not in self.syms:
            self.syms[n] = Sym(n)
        return self.syms[n]

    def type_of(self, n):
        s = self.syms.get(n)
        if s and s.type:
            return s.type
        if n in self.implicit:
            return self.implicit[n]
        c = n[0]
        if c in self.implicit:
            return self.implicit[c]
        return "i" if "i" <= c <= "n" else "f"


DECL_RE = re.compile(r"^(integer|real\*8|real\*4|real|double\s*precision|logical|character(?:\*\d+)?)\b\s*(.*)$")


def split_top(s: str, sep=","):
    """Split at top-level separators (not inside parentheses or quotes)."""
    out, depth, cur, q = [], 0, [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [p.strip() for p in out if p.strip()]


def parse_entity(s):
    """'a(1:n, m)' -> ('a', [('1','n'), ('1','m')]) ; 'a' -> ('a', None)"""
    m = re.match(r"^([a-z_][a-z0-9_]*)\s*(\*\s*\d+)?\s*(?:\((.*)\))?$", s.strip())
    if not m:
        raise F77Error(f"bad entity {s!r}")
    name, dims = m.group(1), m.group(3)
    if dims is None:
        return name, None
    out = []
    for d in split_top(dims):
        if ":" in d:
            lo, hi = d.split(":", 1)
        else:
            lo, hi = "1", d
        out.append((lo.strip(), hi.strip()))
    return name, out


def split_units(stmts):
    units, cur = [], None
    for lab, text, where in stmts:
        t = lower_code(text).strip()
        if cur is None or cur.decl_done is None:
            pass
        m = re.match(r"^(?:(character\*\d+|integer|real\*8|double\s*precision|logical)\s+)?"
                     r"(program|subroutine|function)\s+([a-z_][a-z0-9_]*)\s*(?:\((.*)\))?\s*$", t)
        if m and cur is None:
            kind, name = m.group(2), m.group(3)
            args = [a.strip() for a in (m.group(4) or "").split(",") if a.strip()]
            cur = Unit(kind, name, args, where)
            if m.group(1):
                cur.rettype = m.group(1)
            continue
        if cur is None:
            raise F77Error(f"{where}: statement outside a program unit: {t!r}")
        if t == "end" or re.match(r"^end\s*(subroutine|program|function)\b", t):
            if lab is not None:
                cur.body.append((lab, "continue", where))
            units.append(cur)
            cur = None
            continue
        cur.body.append((lab, text, where))
    if cur is not None:
        raise F77Error("missing END")
    return units


# ----------------------------------------------------------------------------------------------
# translation
# ----------------------------------------------------------------------------------------------

CT = {"i": "int", "f": "float", "d": "double", "l": "int", "c": "char"}


class Translator:
    def __init__(self, units, params_over, assign_over, stubs, empty=None):
        self.units = {u.name: u for u in units}
        self.order = [u.name for u in units]
        self.params_over = {k.lower(): v for k, v in (params_over or {}).items()}
        self.assign_over = {(r.lower(), v.lower()): e for (r, v), e in (assign_over or {}).items()}
        self.stubs = {s.lower() for s in (stubs or [])}
        self.empty = {s.lower() for s in (empty or [])}
        self.commons = {}             # block -> [(name, type, dims)]
        self.used_assign = set()
        self.out = []

    # ---- declarations ----
    def eval_const(self, u, s):
        """Evaluate a PARAMETER / dimension expression to a number."""
        e = parse_expr(s)
        return self._ceval(u, e)

    def _ceval(self, u, e):
        if e.k == "num":
            v = e.a[0].replace("d", "e")
            return float(v) if any(c in v for c in ".e") else int(v)
        if e.k == "name":
            n = e.a[0]
            s = u.syms.get(n)
            if s is not None and s.param is not None:
                return s.param
            if n in MPIF:
                return MPIF[n]
            raise F77Error(f"{u.name}: {n} is not a constant")
        if e.k == "neg":
            return -self._ceval(u, e.a[0])
        if e.k == "bin":
            a, b = self._ceval(u, e.a[1]), self._ceval(u, e.a[2])
            op = e.a[0]
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                if isinstance(a, int) and isinstance(b, int):
                    return int(a / b)
                return a / b
        if e.k == "pow":
            return self._ceval(u, e.a[0]) ** self._ceval(u, e.a[1])
        if e.k == "call" and e.a[0] in ("int", "mod", "max", "min"):
            vals = [self._ceval(u, x) for x in e.a[1]]
            if e.a[0] == "int":
                return int(vals[0])
            if e.a[0] == "mod":
                return int(math.fmod(vals[0], vals[1]))
            return max(vals) if e.a[0] == "max" else min(vals)
        raise F77Error(f"{u.name}: not a constant expression")

    def declare(self, u):
        body = []
        exec_started = False
        for lab, text, where in u.body:
            t = lower_code(text).strip()
            if t == "!mpif":
                for k, v in MPIF.items():
                    u.sym(k).param = v
                    u.sym(k).type = "i"
                continue
            if not exec_started:
                if self._declaration(u, t, where):
                    continue
                m = re.match(r"^([a-z_][a-z0-9_]*)\s*\(([^()]*)\)\s*=(.*)$", t)
                if m and not (u.syms.get(m.group(1)) and u.syms[m.group(1)].dims) and \
                        m.group(1) not in u.args and not self._is_array_decl_later(u, m.group(1)):
                    args = [a.strip() for a in m.group(2).split(",")]
                    if all(re.match(r"^[a-z_][a-z0-9_]*$", a) for a in args):
                        u.sym(m.group(1)).stmtfn = (args, parse_expr(m.group(3)))
                        continue
                exec_started = True
            body.append((lab, text, where))
        u.body = body
        for a in u.args:
            u.sym(a).dummy = True

    def _is_array_decl_later(self, u, name):
        return False

    def _declaration(self, u, t, where):
        m = re.match(r"^implicit\s+(real\*8|double\s*precision|integer|logical|real)\s*\((.*)\)$", t)
        if m:
            ty = INTRINSIC_TYPES[re.sub(r"\s+", " ", m.group(1))]
            for rng in m.group(2).split(","):
                rng = rng.strip()
                if "-" in rng:
                    a, b = [x.strip() for x in rng.split("-")]
                    for c in range(ord(a), ord(b) + 1):
                        u.implicit[chr(c)] = ty
                else:
                    u.implicit[rng] = ty
            return True
        if t.startswith("implicit none"):
            return True
        m = re.match(r"^parameter\s*\((.*)\)$", t)
        if m:
            for item in split_top(m.group(1)):
                n, e = item.split("=", 1)
                n = n.strip()
                v = self.params_over[n] if n in self.params_over else self.eval_const(u, e)
                s = u.sym(n)
                if s.type == "i" or (s.type is None and u.type_of(n) == "i"):
                    v = int(v)
                s.param = v
            return True
        m = re.match(r"^dimension\s+(.*)$", t)
        if m:
            for item in split_top(m.group(1)):
                n, d = parse_entity(item)
                u.sym(n).dims = d
            return True
        m = re.match(r"^common\s*/\s*([a-z0-9_]+)\s*/\s*(.*)$", t)
        if m:
            blk = m.group(1)
            for item in split_top(m.group(2)):
                n, d = parse_entity(item)
                s = u.sym(n)
                s.common = blk
                if d is not None:
                    s.dims = d
                u.__dict__.setdefault("common_order", {}).setdefault(blk, []).append(n)
            return True
        m = DECL_RE.match(t)
        if m and not re.match(r"^(integer|real|logical|double)\w*\s*function\b", t):
            kw = re.sub(r"\s+", " ", m.group(1))
            clen = None
            if kw.startswith("character"):
                ty = "c"
                clen = int(kw.split("*")[1]) if "*" in kw else 1
            else:
                ty = INTRINSIC_TYPES[kw]
            rest = m.group(2).strip()
            if rest.startswith("::"):
                rest = rest[2:]
            for item in split_top(rest):
                n, d = parse_entity(item)
                s = u.sym(n)
                s.type = ty
                s.charlen = clen
                if d is not None:
                    s.dims = d
            return True
        m = re.match(r"^external\s+(.*)$", t)
        if m:
            for n in split_top(m.group(1)):
                u.sym(n).external = True
            return True
        if re.match(r"^(save|data)\b", t):
            raise F77Error(f"{where}: {t.split()[0].upper()} is not handled")
        return False

    def collect_commons(self):
        for name in self.order:
            u = self.units[name]
            for blk, names in getattr(u, "common_order", {}).items():
                members = []
                for n in names:
                    s = u.syms[n]
                    ty = s.type or u.type_of(n)
                    dims = [(self.eval_const(u, lo), self.eval_const(u, hi)) for lo, hi in (s.dims or [])]
                    members.append((n, ty, dims))
                if blk in self.commons:
                    if self.commons[blk] != members:
                        raise F77Error(f"COMMON /{blk}/ differs between units ({name})")
                else:
                    self.commons[blk] = members

    # ---- expression emission: returns (c_text, type) ----
    def num(self, v):
        if re.match(r"^\d+$", v):
            return v, "i"
        if "d" in v:
            x = v.replace("d", "e")
            if x.endswith("e") or "." not in x.split("e")[0] and False:
                pass
            return f"((double){x if '.' in x.split('e')[0] or 'e' in x else x + '.0'})", "d"
        x = v if ("." in v or "e" in v) else v + ".0"
        if x.startswith("."):
            x = "0" + x
        if x.endswith("."):
            x = x + "0"
        x = re.sub(r"\.e", ".0e", x)
        return f"{x}f", "f"

    @staticmethod
    def promote(a, b):
        order = {"i": 0, "l": 0, "f": 1, "d": 2}
        return a if order.get(a, 0) >= order.get(b, 0) else b

    def expr(self, u, e, ctx=None):
        k = e.k
        if k == "num":
            return self.num(e.a[0])
        if k == "lit":
            return ("1" if e.a[0] else "0"), "l"
        if k == "str":
            raise F77Error("character expression")
        if k == "concat":
            raise F77Error("character expression")
        if k == "neg":
            s, t = self.expr(u, e.a[0], ctx)
            return f"(-{s})", t
        if k == "not":
            s, _ = self.expr(u, e.a[0], ctx)
            return f"(!{s})", "l"
        if k == "bin":
            op = e.a[0]
            a, ta = self.expr(u, e.a[1], ctx)
            b, tb = self.expr(u, e.a[2], ctx)
            if op in ("&&", "||"):
                return f"({a} {op} {b})", "l"
            if op in ("==", "!=", "<", "<=", ">", ">="):
                t = self.promote(ta, tb)
                return f"({self.cast(a, ta, t)} {op} {self.cast(b, tb, t)})", "l"
            t = self.promote(ta, tb)
            return f"({self.cast(a, ta, t)} {op} {self.cast(b, tb, t)})", t
        if k == "pow":
            a, ta = self.expr(u, e.a[0], ctx)
            b, tb = self.expr(u, e.a[1], ctx)
            if tb == "i":
                ex = e.a[1]
                if ex.k == "num" and re.match(r"^\d+$", ex.a[0]) and int(ex.a[0]) <= 8:
                    n = int(ex.a[0])
                    if n == 0:
                        return ("1" if ta == "i" else f"(({CT[ta]})1)"), ta
                    return f"pw{ta}{n}({a})", ta
                return f"ipow_{ta}({a}, {b})", ta
            t = self.promote(ta, tb)
            fn = "powf" if t == "f" else "pow"
            return f"{fn}({self.cast(a, ta, t)}, {self.cast(b, tb, t)})", t
        if k == "name":
            return self.name_ref(u, e.a[0])
        if k == "call":
            return self.call_expr(u, e.a[0], e.a[1], ctx)
        raise F77Error(f"expression {k}")

    def cast(self, s, t_from, t_to):
        if t_from == t_to or t_to in ("i", "l") and t_from in ("i", "l"):
            return s
        return f"(({CT[t_to]}){s})"

    def cname(self, u, n):
        s = u.syms.get(n)
        if s is not None and s.common:
            return f"cb_{s.common}.{n}"
        if (s is None or not (s.dummy or s.dims)) and not (u.kind == "function" and n == u.name):
            self.scalars_used.add(n)
        return f"v_{n}"

    def name_ref(self, u, n):
        s = u.syms.get(n)
        if s is not None and s.param is not None:
            v = s.param
            t = s.type or u.type_of(n)
            if t in ("i", "l"):
                return str(int(v)), "i"
            if t == "f":
                return f"{float(v)!r}f", "f"
            return f"((double){float(v)!r})", "d"
        if n in MPIF and (s is None or s.type is None):
            return str(MPIF[n]), "i"
        t = u.type_of(n)
        if s is not None and s.dims:
            raise F77Error(f"whole array {n} in an expression")
        if s is not None and s.dummy:
            return f"(*{self.cname(u, n)})", t
        if u.kind == "function" and n == u.name:
            return "v__result", t
        return self.cname(u, n), t

    def index(self, u, n, args, ctx):
        """C lvalue of element args of array n (column-major, declared bounds)."""
        s = u.syms[n]
        if len(args) != len(s.dims):
            raise F77Error(f"{n}: {len(args)} subscripts for rank {len(s.dims)}")
        base = self.cname(u, n)
        terms, stride = [], "1"
        for (lo, hi), a in zip(s.dims, args):
            sa, ta = self.expr(u, a, ctx)
            if ta != "i":
                sa = f"((long)({sa}))"
            los = self.dim_expr(u, lo)
            terms.append(f"((long)({sa}) - ({los})) * ({stride})")
            if hi != "*":
                his = self.dim_expr(u, hi)
                stride = f"({stride}) * (long)(({his}) - ({los}) + 1)"
        if s.common or not s.dummy:
            return f"{base}[{' + '.join(terms)}]"
        return f"{base}[{' + '.join(terms)}]"

    def dim_expr(self, u, s):
        s2, _ = self.expr(u, parse_expr(s))
        return s2

    def call_expr(self, u, n, args, ctx):
        s = u.syms.get(n)
        if s is not None and s.dims:
            t = u.type_of(n)
            return self.index(u, n, args, ctx), t
        if s is not None and s.stmtfn is not None:
            fargs, body = s.stmtfn
            if len(fargs) != len(args):
                raise F77Error(f"statement function {n}: argument count")
            vals = [self.expr(u, a, ctx) for a in args]
            sub = {}
            for fa, (v, t) in zip(fargs, vals):
                want = u.type_of(fa)
                sub[fa] = (self.cast(v, t, want), want)
            return self.expr_sub(u, body, sub), u.type_of(n)
        return self.intrinsic(u, n, args, ctx)

    def expr_sub(self, u, e, sub):
        """Emit a statement-function body with its dummy names replaced by argument values."""
        if e.k == "name" and e.a[0] in sub:
            return f"({sub[e.a[0]][0]})"
        saved = {}
        for fa, (v, t) in sub.items():
            saved[fa] = u.syms.get(fa)
        # substitute by rewriting the tree into a temporary unit-local view
        return self._emit_with_sub(u, e, sub)[0]

    def _emit_with_sub(self, u, e, sub):
        if e.k == "name" and e.a[0] in sub:
            return f"({sub[e.a[0]][0]})", sub[e.a[0]][1]
        if e.k in ("bin",):
            op = e.a[0]
            a, ta = self._emit_with_sub(u, e.a[1], sub)
            b, tb = self._emit_with_sub(u, e.a[2], sub)
            if op in ("&&", "||"):
                return f"({a} {op} {b})", "l"
            t = self.promote(ta, tb)
            if op in ("==", "!=", "<", "<=", ">", ">="):
                return f"({self.cast(a, ta, t)} {op} {self.cast(b, tb, t)})", "l"
            return f"({self.cast(a, ta, t)} {op} {self.cast(b, tb, t)})", t
        if e.k == "neg":
            a, ta = self._emit_with_sub(u, e.a[0], sub)
            return f"(-{a})", ta
        if e.k in ("num", "lit"):
            return self.expr(u, e)
        if e.k == "name":
            return self.expr(u, e)
        if e.k == "call" and not any(True for _ in []):
            # arguments may reference dummies
            n, args = e.a
            s = u.syms.get(n)
            if s is not None and s.dims:
                raise F77Error("array reference inside a statement function")
            vals = [self._emit_with_sub(u, x, sub) for x in args]
            return self._intrinsic_vals(n, vals)
        if e.k == "pow":
            a, ta = self._emit_with_sub(u, e.a[0], sub)
            b, tb = self._emit_with_sub(u, e.a[1], sub)
            t = self.promote(ta, tb)
            if tb == "i":
                return f"ipow_{ta}({a}, {b})", ta
            return f"{'powf' if t == 'f' else 'pow'}({self.cast(a, ta, t)}, {self.cast(b, tb, t)})", t
        raise F77Error(f"statement function body {e.k}")

    def intrinsic(self, u, n, args, ctx):
        vals = [self.expr(u, a, ctx) for a in args]
        return self._intrinsic_vals(n, vals)

    def _intrinsic_vals(self, n, vals):
        ts = [t for _, t in vals]
        s = [v for v, _ in vals]

        def fl(name_f, name_d):
            t = "d" if ts[0] == "d" else ("f" if ts[0] == "f" else "d")
            return f"{name_f if t == 'f' else name_d}({self.cast(s[0], ts[0], t)})", t
        generic = {"sqrt": ("sqrtf", "sqrt"), "tanh": ("tanhf", "tanh"), "exp": ("expf", "exp"),
                   "cos": ("cosf", "cos"), "sin": ("sinf", "sin"), "tan": ("tanf", "tan"),
                   "atan": ("atanf", "atan"), "log": ("logf", "log"), "log10": ("log10f", "log10"),
                   "cosh": ("coshf", "cosh"), "sinh": ("sinhf", "sinh"), "acos": ("acosf", "acos"),
                   "asin": ("asinf", "asin")}
        if n in generic:
            return fl(*generic[n])
        dspec = {"dsqrt": "sqrt", "dtanh": "tanh", "dexp": "exp", "dcos": "cos", "dsin": "sin",
                 "datan": "atan", "dlog": "log", "dcosh": "cosh", "dsinh": "sinh", "dlog10": "log10"}
        if n in dspec:
            return f"{dspec[n]}({self.cast(s[0], ts[0], 'd')})", "d"
        if n in ("alog",):
            return f"logf({self.cast(s[0], ts[0], 'f')})", "f"
        if n in ("abs", "dabs", "iabs"):
            t = ts[0]
            if t == "i":
                return f"abs({s[0]})", "i"
            return (f"fabsf({s[0]})" if t == "f" else f"fabs({s[0]})"), t
        if n in ("min", "max", "amin1", "amax1", "dmin1", "dmax1", "min0", "max0"):
            t = ts[0]
            for q in ts[1:]:
                t = self.promote(t, q)
            if n in ("dmin1", "dmax1"):
                t = "d"
            f = "min" if "min" in n else "max"
            acc = self.cast(s[0], ts[0], t)
            for v, tv in zip(s[1:], ts[1:]):
                acc = f"{f}_{t}({acc}, {self.cast(v, tv, t)})"
            return acc, t
        if n == "mod":
            t = self.promote(ts[0], ts[1])
            if t == "i":
                return f"({s[0]} % {s[1]})", "i"
            return f"{'fmodf' if t == 'f' else 'fmod'}({self.cast(s[0], ts[0], t)}, {self.cast(s[1], ts[1], t)})", t
        if n in ("int", "idint", "ifix"):
            return f"((int)({s[0]}))", "i"
        if n == "nint":
            return f"((int)lround({s[0]}))", "i"
        if n in ("dble", "dfloat"):
            return self.cast(s[0], ts[0], "d"), "d"
        if n in ("float", "real", "sngl"):
            return self.cast(s[0], ts[0], "f"), "f"
        if n in ("sign", "dsign"):
            t = self.promote(ts[0], ts[1])
            return f"sign_{t}({self.cast(s[0], ts[0], t)}, {self.cast(s[1], ts[1], t)})", t
        if n == "atan2" or n == "datan2":
            t = self.promote(ts[0], ts[1])
            return f"{'atan2f' if t == 'f' else 'atan2'}({self.cast(s[0], ts[0], t)}, {self.cast(s[1], ts[1], t)})", t
        raise F77Error(f"function {n}")

    # ---- statements ----
    def lvalue(self, u, target):
        e = parse_expr(target)
        if e.k == "name":
            n = e.a[0]
            s = u.syms.get(n)
            if s is not None and s.dims:
                raise F77Error(f"whole-array assignment to {n}")
            if s is not None and s.param is not None:
                raise F77Error(f"assignment to PARAMETER {n}")
            t = u.type_of(n)
            if t == "c":
                raise F77Error("character assignment")
            return self.name_ref(u, n)[0], t, n
        if e.k == "call":
            n = e.a[0]
            s = u.syms.get(n)
            if s is None or not s.dims:
                raise F77Error(f"assignment to non-array {n}(...)")
            if u.type_of(n) == "c":
                raise F77Error("character assignment")
            return self.index(u, n, e.a[1], None), u.type_of(n), n
        raise F77Error("bad assignment target")

    def call_arg(self, u, a, pre):
        """C argument for an actual argument (by reference)."""
        e = parse_expr(a)
        if e.k == "name":
            n = e.a[0]
            s = u.syms.get(n)
            if s is not None and s.dims:
                return f"&{self.cname(u, n)}[0]"
            if s is None or s.param is None:
                if n in MPIF and (s is None or s.type is None):
                    pass
                elif s is not None and s.dummy:
                    return self.cname(u, n)
                elif s is not None and s.external:
                    return f"(void*)f_{n}"
                else:
                    return f"&{self.name_ref(u, n)[0]}"
        if e.k == "call":
            n = e.a[0]
            s = u.syms.get(n)
            if s is not None and s.dims:
                return f"&{self.index(u, n, e.a[1], None)}"
        v, t = self.expr(u, e)
        tmp = f"t_{len(pre)}"
        pre.append(f"{CT[t] if t != 'l' else 'int'} {tmp} = {v};")
        return f"&{tmp}"

    def translate_unit(self, u):
        o = []
        params = []
        for a in u.args:
            s = u.syms[a]
            t = s.type or u.type_of(a)
            params.append(f"{CT[t] if t != 'c' else 'char'}* v_{a}")
        rett = "void"
        if u.kind == "function":
            rt = u.rettype or ""
            rett = "double" if "real" in rt or "double" in rt or not rt else ("int" if "integer" in rt else "double")
            if "character" in rt:
                rett = "void"
        fname = "f_main" if u.kind == "program" else f"f_{u.name}"
        sig = f"{rett} {fname}({', '.join(params) if params else 'void'})"
        if u.name in self.stubs or (u.kind == "function" and "character" in (u.rettype or "")):
            o.append(f"{sig} {{ ref_unreachable(\"routine {u.name} ({u.where}) is not translated\"); "
                     + ("return 0; }" if rett != "void" else "}"))
            return o, sig
        if u.name in self.empty:
            o.append(f"{sig} {{ /* {u.name} ({u.where}) disabled */ " + ("return 0; }" if rett != "void" else "}"))
            return o, sig
        o.append(f"{sig} {{")
        # locals
        for n, s in u.syms.items():
            if s.common or s.dummy or s.param is not None or s.stmtfn is not None or s.external:
                continue
            if n in MPIF and s.type is None:
                continue
            t = s.type or u.type_of(n)
            if t == "c":
                continue
            if s.dims:
                try:
                    size = 1
                    for lo, hi in s.dims:
                        size *= self.eval_const(u, hi) - self.eval_const(u, lo) + 1
                    o.append(f"  static REF_TLS {CT[t]} v_{n}[{size}];")
                except F77Error:
                    # bounds from run-time values (an automatic array): allocated at entry
                    ext = " * ".join(f"(long)(({self.dim_expr(u, hi)}) - ({self.dim_expr(u, lo)}) + 1)"
                                     for lo, hi in s.dims)
                    o.append(f"  {CT[t]}* v_{n} = ({CT[t]}*)calloc((size_t)({ext}), sizeof({CT[t]}));")
            elif not (u.kind == "function" and n == u.name):
                if self._is_function_name(n):
                    continue
                o.append(f"  {CT[t]} v_{n} = 0;")
        if u.kind == "function":
            o.append(f"  {rett} v__result = 0;")
        declared = {n for n in u.syms}
        self.scalars_used = set()
        body = []
        self.emit_body(u, body)
        for n in sorted(self.scalars_used - declared):     # implicitly typed local scalars
            t = u.type_of(n)
            o.append(f"  {CT[t] if t != 'l' else 'int'} v_{n} = 0;")
        o.extend(body)
        if u.kind == "function":
            o.append("  return v__result;")
        o.append("}")
        return o, sig

    def _is_function_name(self, n):
        return n in self.units and self.units[n].kind == "function"

    def emit_body(self, u, o):
        # DO structure: labelled DOs end at the statement with their label (possibly shared)
        stack = []        # open loops: (kind, label or None)
        labels_goto = set()
        for lab, text, where in u.body:
            for m in re.finditer(r"go\s*to\s*(\d+)", lower_code(text)):
                labels_goto.add(int(m.group(1)))
        ind = lambda: "  " * (len(stack) + 1)   # noqa: E731
        for lab, text, where in u.body:
            t = lower_code(text).strip()
            if lab is not None and lab in labels_goto:
                o.append(f"{ind()}L{lab}:;")
            try:
                self.statement(u, t, o, stack, ind, where)
            except F77Error as ex:
                msg = str(ex)[:80].replace('"', "'")
                o.append(f"{ind()}ref_unreachable(\"{where}: {msg}\");")
            if lab is not None:
                # close every labelled DO ending here (innermost first)
                while stack and stack[-1][0] == "do" and stack[-1][1] == lab:
                    stack.pop()
                    o.append(f"{ind()}}}}}")
        if stack:
            raise F77Error(f"{u.name}: unclosed blocks {stack}")

    def statement(self, u, t, o, stack, ind, where):
        if t in ("", "continue"):
            return
        m = re.match(r"^do\s*(\d+)\s*,?\s*([a-z_][a-z0-9_]*)\s*=(.*)$", t)
        m2 = re.match(r"^do\s+([a-z_][a-z0-9_]*)\s*=(.*)$", t)
        if m or m2:
            if m:
                lab, var, rng = int(m.group(1)), m.group(2), m.group(3)
            else:
                lab, var, rng = None, m2.group(1), m2.group(2)
            parts = split_top(rng)
            lo = self.expr(u, parse_expr(parts[0]))
            hi = self.expr(u, parse_expr(parts[1]))
            st = self.expr(u, parse_expr(parts[2])) if len(parts) > 2 else ("1", "i")
            vref, vt = self.name_ref(u, var)
            if vt != "i":
                raise F77Error("non-integer DO variable")
            n = len(stack)
            o.append(f"{ind()}{{ long n_{n} = ((long)({hi[0]}) - (long)({lo[0]}) + (long)({st[0]})) / (long)({st[0]}); "
                     f"int s_{n} = {st[0]}; {vref} = {lo[0]};")
            o.append(f"{ind()}for (; n_{n} > 0; --n_{n}, {vref} += s_{n}) {{")
            stack.append(("do", lab))
            return
        if t == "do":
            o.append(f"{ind()}{{ for (;;) {{")
            stack.append(("do", None))
            return
        if t in ("enddo", "end do"):
            if not stack or stack[-1] != ("do", None):
                raise F77Error("ENDDO without DO")
            stack.pop()
            o.append(f"{ind()}}}}}")
            return
        if t == "exit":
            o.append(f"{ind()}break;")
            return
        if t == "cycle":
            o.append(f"{ind()}continue;")
            return
        m = re.match(r"^if\s*\((.*)\)\s*then$", t)
        if m and _balanced_prefix(t[2:].strip()):
            c, _ = self.expr(u, parse_expr(m.group(1)))
            o.append(f"{ind()}if ({c}) {{")
            stack.append(("if", None))
            return
        m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", t)
        if m:
            if not stack or stack[-1][0] != "if":
                raise F77Error("ELSE IF without IF")
            c, _ = self.expr(u, parse_expr(m.group(1)))
            o.append(f"{'  ' * len(stack)}}} else if ({c}) {{")
            return
        if t == "else":
            o.append(f"{'  ' * len(stack)}}} else {{")
            return
        if t in ("endif", "end if"):
            if not stack or stack[-1][0] != "if":
                raise F77Error("ENDIF without IF")
            stack.pop()
            o.append(f"{ind()}}}")
            return
        if t.startswith("if"):
            cond, rest = _logical_if(t)
            if cond is not None:
                c, _ = self.expr(u, parse_expr(cond))
                inner = []
                self.statement(u, rest, inner, stack + [("lif", None)], lambda: "", where)
                o.append(f"{ind()}if ({c}) {{ {' '.join(inner)} }}")
                return
        m = re.match(r"^go\s*to\s*(\d+)$", t)
        if m:
            o.append(f"{ind()}goto L{m.group(1)};")
            return
        if t == "return":
            o.append(f"{ind()}return" + (" v__result;" if u.kind == "function" else ";"))
            return
        if t == "stop" or t.startswith("stop "):
            o.append(f"{ind()}ref_stop(\"{u.name}\");")
            return
        if re.match(r"^(write|print|open|close|inquire|format|rewind|backspace)\b", t):
            return
        if re.match(r"^read\b", t):
            o.append(f"{ind()}ref_unreachable(\"{where}: READ\");")
            return
        m = re.match(r"^call\s+([a-z_][a-z0-9_]*)\s*(?:\((.*)\))?$", t)
        if m:
            name, args = m.group(1), split_top(m.group(2) or "")
            pre = []
            cargs = [self.call_arg(u, a, pre) for a in args]
            if name.startswith("mpi_"):
                o.append(f"{ind()}{{ {' '.join(pre)} f_{name}({len(cargs)}, {', '.join(['(void*)' + c for c in cargs])}); }}")
            else:
                if name not in self.units:
                    raise F77Error(f"call of unknown routine {name}")
                o.append(f"{ind()}{{ {' '.join(pre)} f_{name}({', '.join(cargs)}); }}")
            return
        # assignment
        lhs, rhs = _split_assignment(t)
        if lhs is None:
            raise F77Error(f"statement not handled: {t[:60]}")
        lv, lt, lname = self.lvalue(u, lhs)
        key = (u.name, lname)
        if key in self.assign_over:
            self.used_assign.add(key)
            o.append(f"{ind()}{lv} = ({CT[lt]})({self.assign_over[key]});")
            return
        v, vt = self.expr(u, parse_expr(rhs))
        o.append(f"{ind()}{lv} = {self.cast(v, vt, lt)};")

    def run(self):
        for n in self.order:
            self.declare(self.units[n])
        self.collect_commons()
        out = [PRELUDE]
        for blk, members in self.commons.items():
            out.append("struct __attribute__((packed)) cb_t_%s {" % blk)
            for n, t, dims in members:
                size = 1
                for lo, hi in dims:
                    size *= hi - lo + 1
                out.append(f"  {CT[t]} {n}" + (f"[{size}]" if dims else "") + ";")
            out.append(f"}};\nREF_TLS struct cb_t_{blk} cb_{blk};")
        bodies, sigs = [], []
        for n in self.order:
            b, sig = self.translate_unit(self.units[n])
            bodies.append(b)
            sigs.append(sig)
        out.extend(s + ";" for s in sigs)
        for b in bodies:
            out.extend(b)
        out.append(self.symbol_table())
        missing = set(self.assign_over) - self.used_assign
        if missing:
            raise F77Error(f"assignment overrides that matched nothing: {sorted(missing)}")
        return "\n".join(out) + "\n"

    def symbol_table(self):
        rows = []
        for blk, members in self.commons.items():
            for n, t, dims in members:
                size = 1
                shape = []
                for lo, hi in dims:
                    size *= hi - lo + 1
                    shape.append(hi - lo + 1)
                rows.append((n, blk, t, size, shape))
        # (the table holds addresses: not for a build whose COMMON blocks are thread-local)
        o = ["#ifndef REF_NO_SYMBOLS",
             "typedef struct { const char* name; void* addr; char type; long size; int rank; long shape[7]; } ref_sym;",
             "static ref_sym ref_syms[] = {"]
        for n, blk, t, size, shape in rows:
            sh = ", ".join(str(x) for x in shape + [0] * (7 - len(shape)))
            o.append(f"  {{\"{n}\", (void*)&cb_{blk}.{n}, '{t}', {size}, {len(shape)}, {{{sh}}}}},")
        o.append("  {0, 0, 0, 0, 0, {0}}};")
        o.append("""int ref_symbol(const char* name, void** addr, char* type, long* size, int* rank, long* shape) {
  for (ref_sym* s = ref_syms; s->name; ++s) if (!strcmp(s->name, name)) {
    *addr = s->addr; *type = s->type; *size = s->size; *rank = s->rank;
    for (int q = 0; q < 7; ++q) shape[q] = s->shape[q];
    return 1;
  }
  return 0;
}
#endif""")
        return "\n".join(o)


def _balanced_prefix(s):
    """True when s = '(...)' followed by text, the parenthesis closing before the end."""
    return s.startswith("(")


def _logical_if(t):
    """'if (cond) stmt' -> (cond, stmt); None when t is not a logical IF."""
    m = re.match(r"^if\s*\(", t)
    if not m:
        return None, None
    depth, q = 0, None
    for i in range(m.end() - 1, len(t)):
        ch = t[i]
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                rest = t[i + 1:].strip()
                if rest == "then":
                    return None, None
                return t[m.end():i], rest
    raise F77Error("unbalanced IF")


def _split_assignment(t):
    depth, q = 0, None
    for i, ch in enumerate(t):
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0 and t[i + 1:i + 2] != "=" and t[i - 1:i] not in "<>/=":
            return t[:i].strip(), t[i + 1:].strip()
    return None, None


PRELUDE = r"""/* Generated by oracle/f77c.py from the reference program's Fortran source.  Test
 * infrastructure: not part of the product, not committed. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
/* REF_TLS empty: one program per process.  -DREF_TLS=__thread: every COMMON block and static
 * local array per thread, so that threads run as the ranks of an MPI decomposition. */
#ifndef REF_TLS
#define REF_TLS
#endif
void ref_unreachable(const char* what);
void ref_stop(const char* where);
#define DEF_POW(T, S) \
  static inline T pw##S##1(T a) { return a; } \
  static inline T pw##S##2(T a) { return a * a; } \
  static inline T pw##S##3(T a) { return a * a * a; } \
  static inline T pw##S##4(T a) { T b = a * a; return b * b; } \
  static inline T pw##S##5(T a) { T b = a * a; return b * b * a; } \
  static inline T pw##S##6(T a) { T b = a * a; return b * b * b; } \
  static inline T pw##S##7(T a) { T b = a * a; return b * b * b * a; } \
  static inline T pw##S##8(T a) { T b = a * a; b = b * b; return b * b; } \
  static inline T ipow_##S(T a, int n) { T r = 1; int neg = n < 0; if (neg) n = -n; \
    while (n) { if (n & 1) r *= a; a *= a; n >>= 1; } return neg ? (T)1 / r : r; } \
  static inline T min_##S(T a, T b) { return a < b ? a : b; } \
  static inline T max_##S(T a, T b) { return a > b ? a : b; } \
  static inline T sign_##S(T a, T b) { T m = a < 0 ? -a : a; return b >= 0 ? m : -m; }
DEF_POW(int, i)
DEF_POW(float, f)
DEF_POW(double, d)
void f_mpi_init(int n, ...);
void f_mpi_comm_size(int n, ...);
void f_mpi_comm_rank(int n, ...);
void f_mpi_barrier(int n, ...);
void f_mpi_finalize(int n, ...);
void f_mpi_abort(int n, ...);
void f_mpi_allreduce(int n, ...);
void f_mpi_reduce(int n, ...);
void f_mpi_gather(int n, ...);
void f_mpi_send(int n, ...);
void f_mpi_recv(int n, ...);
void f_mpi_sendrecv(int n, ...);
void f_mpi_type_commit(int n, ...);
void f_mpi_type_free(int n, ...);
void f_mpi_type_contiguous(int n, ...);
void f_mpi_type_vector(int n, ...);
"""


def translate(src_path: str, params=None, assign=None, stubs=None, empty=None) -> str:
    units = split_units(read_fixed(src_path))
    return Translator(units, params, assign, stubs, empty).run()


if __name__ == "__main__":
    sys.stdout.write(translate(sys.argv[1]))
