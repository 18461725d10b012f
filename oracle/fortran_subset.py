"""Fortran-77 subset -> C translator for the reference's time-step routines.

Test infrastructure.  It reads the reference's own fixed-form source
(3dmhdsub.f, 3dmhdparam.f) and emits C that evaluates every statement with
gfortran's semantics on x86-64: E-exponent and plain real literals are
REAL(4), D-exponent literals REAL*8, implicit typing REAL*8(A-H,O-Z) and
INTEGER(I-N), mixed operands widened before the operation, left-to-right
evaluation with no reassociation, X**2 as X*X, integer division truncating.
The emitted C is compiled with -ffp-contract=off so that no FMA appears.

Only the constructs the translated routines use are supported: labelled
and block DO loops (shared terminal labels included), block and logical
IF, assignments to scalars, array elements and array sections, CALL
(other translated routines, MPI_* mapped onto the mini-MPI of
oracle/ref_harness.c), RETURN, STOP, GOTO, and declarations (DIMENSION,
COMMON, PARAMETER, DATA, SAVE, LOGICAL, INTEGER, REAL*8, CHARACTER,
IMPLICIT, EXTERNAL, INCLUDE).  WRITE statements become no-ops.  Anything
else raises TranslateError, so nothing is silently mistranslated.

The output goes only to oracle/_ref/ (see oracle/make_ref.py); nothing
generated from the reference is committed.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field


class TranslateError(Exception):
    pass


# ----------------------------------------------------------------------------
# Fixed-form source reading
# ----------------------------------------------------------------------------

@dataclass
class Stmt:
    label: int | None
    text: str
    line: int


def _expand_tabs(line: str) -> str:
    out = []
    for ch in line:
        if ch == "\t":
            n = 8 - (len(out) % 8)
            out.extend(" " * n)
        else:
            out.append(ch)
    return "".join(out)


def _strip_inline_comment(text: str) -> str:
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


def read_fixed_form(path: str) -> list[Stmt]:
    """Return logical statements (continuations joined, comments dropped)."""
    stmts: list[Stmt] = []
    raw = open(path, encoding="latin-1").read().split("\n")
    for no, line in enumerate(raw, 1):
        if not line.strip():
            continue
        if line[0] in "cC*!":
            continue
        head = line[:6]
        if "\t" in head:
            p = line.index("\t")
            lab = line[:p].strip()
            rest = line[p + 1:]
            if not lab and rest[:1] in "123456789":
                cont, text = True, rest[1:]
            else:
                cont, text = False, rest
        else:
            e = _expand_tabs(line)
            lab = e[:5].strip()
            cont = len(e) > 5 and e[5] not in " 0"
            text = e[6:72]
        text = _strip_inline_comment(text)
        if cont:
            if not stmts:
                raise TranslateError(f"continuation without statement at line {no}")
            stmts[-1].text += text
            continue
        if not text.strip() and not lab:
            continue
        stmts.append(Stmt(int(lab) if lab else None, text, no))
    for s in stmts:
        s.text = s.text.strip()
    return stmts


def split_units(stmts: list[Stmt]) -> dict[str, list[Stmt]]:
    units: dict[str, list[Stmt]] = {}
    cur: list[Stmt] | None = None
    name = None
    for s in stmts:
        u = s.text.upper()
        m = re.match(r"^(SUBROUTINE|PROGRAM|FUNCTION|REAL\*8\s+FUNCTION)\s+(\w+)", u)
        if cur is None and m:
            name = m.group(2)
            cur = [s]
            continue
        if cur is not None:
            if re.fullmatch(r"END(\s+(SUBROUTINE|FUNCTION|PROGRAM)(\s+\w+)?)?", u.replace("\t", " ").strip()):
                units[name] = cur
                cur = None
                continue
            cur.append(s)
    return units


# ----------------------------------------------------------------------------
# Expressions
# ----------------------------------------------------------------------------

TOKEN_RE = re.compile(r"""
    (?P<ws>\s+)
  | (?P<real>(\d+\.\d*|\.\d+|\d+)([EeDd][+-]?\d+)|\d+\.\d*|\.\d+(?![A-Za-z]))
  | (?P<int>\d+)
  | (?P<dotop>\.(EQ|NE|LT|LE|GT|GE|AND|OR|NOT|TRUE|FALSE|EQV|NEQV)\.)
  | (?P<str>'[^']*')
  | (?P<name>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>\*\*|//|==|/=|<=|>=|[-+*/(),:<>=])
""", re.VERBOSE | re.IGNORECASE)


def tokenize(s: str):
    pos, out = 0, []
    while pos < len(s):
        m = TOKEN_RE.match(s, pos)
        if not m:
            raise TranslateError(f"cannot tokenize {s[pos:pos+20]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group(kind)
        if kind in ("name", "dotop"):
            val = val.upper()
        out.append((kind, val))
    out.append(("end", ""))
    return out


@dataclass
class Node:
    kind: str                 # num, name, call, un, bin, str, range
    val: object = None
    args: list = field(default_factory=list)


class Parser:
    # precedence: .OR. < .AND. < .NOT. < relational < + - < * / < unary - < **
    def __init__(self, text: str):
        self.t = tokenize(text)
        self.i = 0

    def peek(self):
        return self.t[self.i]

    def take(self, val=None):
        tok = self.t[self.i]
        if val is not None and tok[1] != val:
            raise TranslateError(f"expected {val!r}, got {tok[1]!r}")
        self.i += 1
        return tok

    def parse(self):
        e = self.p_or()
        if self.peek()[0] != "end":
            raise TranslateError(f"trailing tokens {self.t[self.i:]}")
        return e

    def p_or(self):
        a = self.p_and()
        while self.peek()[1] in (".OR.",):
            self.take()
            a = Node("bin", ".OR.", [a, self.p_and()])
        return a

    def p_and(self):
        a = self.p_not()
        while self.peek()[1] == ".AND.":
            self.take()
            a = Node("bin", ".AND.", [a, self.p_not()])
        return a

    def p_not(self):
        if self.peek()[1] == ".NOT.":
            self.take()
            return Node("un", ".NOT.", [self.p_not()])
        return self.p_rel()

    REL = {".EQ.": "==", ".NE.": "!=", ".LT.": "<", ".LE.": "<=", ".GT.": ">", ".GE.": ">=",
           "==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}

    def p_rel(self):
        a = self.p_add()
        if self.peek()[1] in self.REL:
            op = self.REL[self.take()[1]]
            a = Node("bin", op, [a, self.p_add()])
        return a

    def p_add(self):
        # Fortran: optional leading sign applies to the first add-operand.
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = self.p_mul()
            if op == "-":
                a = Node("un", "-", [a])
        else:
            a = self.p_mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = Node("bin", op, [a, self.p_mul()])
        return a

    def p_mul(self):
        a = self.p_pow()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = Node("bin", op, [a, self.p_pow()])
        return a

    def p_pow(self):
        a = self.p_prim()
        if self.peek()[1] == "**":
            self.take()
            # right associative; exponent may carry a sign
            if self.peek()[1] in ("+", "-"):
                op = self.take()[1]
                b = self.p_pow()
                if op == "-":
                    b = Node("un", "-", [b])
            else:
                b = self.p_pow()
            a = Node("bin", "**", [a, b])
        return a

    def p_prim(self):
        kind, val = self.peek()
        if kind == "real":
            self.take()
            return Node("num", ("real", val))
        if kind == "int":
            self.take()
            return Node("num", ("int", val))
        if kind == "dotop" and val in (".TRUE.", ".FALSE."):
            self.take()
            return Node("num", ("logical", val))
        if kind == "str":
            self.take()
            return Node("str", val)
        if val == "(":
            self.take()
            e = self.p_or()
            self.take(")")
            return e
        if kind == "name":
            self.take()
            if self.peek()[1] == "(":
                self.take()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.p_arg())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return Node("call", val, args)
            return Node("name", val)
        raise TranslateError(f"unexpected token {val!r}")

    def p_arg(self):
        # a subscript may be a section lo:hi with either side omitted
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.p_or()
            return Node("range", None, [None, hi])
        e = self.p_or()
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.p_or()
            return Node("range", None, [e, hi])
        return e


def parse_expr(text: str) -> Node:
    return Parser(text).parse()


# ----------------------------------------------------------------------------
# Symbols and code generation
# ----------------------------------------------------------------------------

RANK = {"i": 0, "f": 1, "d": 2}
CTYPE = {"i": "int", "f": "float", "d": "double", "l": "int", "c": "const char*"}

INTRINSICS = {"SQRT", "EXP", "LOG", "TANH", "COSH", "SINH", "COS", "SIN", "TAN", "ATAN", "ASIN", "ABS",
              "MIN", "MAX", "FLOAT", "REAL", "DBLE", "INT", "NINT", "MOD", "MINVAL", "MAXVAL", "SUM", "SIGN"}


@dataclass
class Array:
    name: str
    dims: list          # list of Node (upper bounds; lower bound 1)
    type: str


class Scope:
    """Names visible in one program unit."""

    def __init__(self, tr: "Translator", unit: str):
        self.tr = tr
        self.unit = unit
        self.arrays: dict[str, Array] = {}
        self.types: dict[str, str] = {}
        self.commons: set[str] = set()
        self.dummies: list[str] = []
        self.saved: dict[str, str] = {}   # DATA initialisers
        self.locals_used: set[str] = set()
        self.params_local: dict[str, Node] = {}

    def type_of(self, name: str) -> str:
        if name in self.types:
            return self.types[name]
        if name in self.tr.param_types:
            return self.tr.param_types[name]
        if name in self.tr.global_types:
            return self.tr.global_types[name]
        return "i" if name[0] in "IJKLMN" else "d"

    def array(self, name: str) -> Array | None:
        if name in self.arrays:
            return self.arrays[name]
        return None


class Translator:
    def __init__(self, param_file: str, overrides: set[str]):
        self.param_order: list[tuple[str, Node]] = []
        self.param_types: dict[str, str] = {}
        self.global_types: dict[str, str] = {}
        self.global_arrays: dict[str, Array] = {}
        self.common_scalars: dict[str, str] = {}
        self.overrides = overrides
        self.units: dict[str, list[Stmt]] = {}
        self.out_funcs: list[str] = []
        self.uid = 0
        self.param_base = os.path.basename(param_file).upper()
        self._read_params(param_file)
        # names from INCLUDE 'mpif.h', provided by the harness
        for n in ("MPI_COMM_WORLD", "MPI_STATUS_SIZE", "MPI_DOUBLE_PRECISION", "MPI_FLOAT",
                  "MPI_MIN", "MPI_MAX", "MPI_SUM"):
            self.global_types[n] = "i"

    # --- parameters -----------------------------------------------------
    def _read_params(self, path: str):
        self.param_decl_stmts = read_fixed_form(path)
        logicals: set[str] = set()
        for s in self.param_decl_stmts:
            u = s.text.upper()
            if u.startswith("LOGICAL"):
                for n in u[len("LOGICAL"):].split(","):
                    logicals.add(n.strip())
            elif u.startswith("PARAMETER"):
                body = s.text[s.text.index("(") + 1: s.text.rindex(")")]
                for item in _split_top(body, ","):
                    name, expr = item.split("=", 1)
                    name = name.strip().upper()
                    self.param_order.append((name, parse_expr(expr)))
                    if name in logicals:
                        self.param_types[name] = "l"
                    else:
                        self.param_types[name] = "i" if name[0] in "IJKLMN" else "d"
            elif u.startswith("DIMENSION"):
                # IPAR(32), PAR(64) are SETUP arguments; not used here
                pass

    # --- expression codegen --------------------------------------------
    def gen(self, n: Node, sc: Scope, sect=None) -> tuple[str, str]:
        """Return (C code, type).  sect maps array sections to loop indices."""
        k = n.kind
        if k == "num":
            typ, v = n.val
            if typ == "int":
                return v, "i"
            if typ == "logical":
                return ("1" if v == ".TRUE." else "0"), "l"
            vu = v.upper()
            if "D" in vu:
                return "(" + vu.replace("D", "E") + ")", "d"
            lit = vu if ("E" in vu or "." in vu) else vu + ".0"
            if lit.startswith("."):
                lit = "0" + lit
            if lit.endswith("."):
                lit = lit + "0"
            return "(" + lit + "f)", "f"
        if k == "str":
            return '"' + n.val[1:-1].replace('"', '\\"') + '"', "c"
        if k == "name":
            name = n.val
            arr = sc.array(name)
            if arr is not None:
                if sect is None:
                    raise TranslateError(f"whole array {name} outside an array assignment")
                return self._elem(arr, [Node("range", None, [None, None]) for _ in arr.dims], sc, sect)
            sc.locals_used.add(name)
            return name, sc.type_of(name)
        if k == "un":
            a, ta = self.gen(n.args[0], sc, sect)
            if n.val == "-":
                return f"(-{a})", ta
            return f"(!{a})", "l"
        if k == "bin":
            op = n.val
            a, ta = self.gen(n.args[0], sc, sect)
            b, tb = self.gen(n.args[1], sc, sect)
            if op in (".AND.", ".OR."):
                return f"({a} {'&&' if op == '.AND.' else '||'} {b})", "l"
            if op == "**":
                return self._pow(a, ta, b, tb, n.args[1])
            t = ta if RANK.get(ta, 0) >= RANK.get(tb, 0) else tb
            a = self._conv(a, ta, t)
            b = self._conv(b, tb, t)
            if op in ("==", "!=", "<", "<=", ">", ">="):
                return f"({a} {op} {b})", "l"
            return f"({a} {op} {b})", t
        if k == "call":
            name = n.val
            arr = sc.array(name)
            if arr is not None:
                return self._elem(arr, n.args, sc, sect)
            return self._intrinsic(name, n.args, sc, sect)
        raise TranslateError(f"cannot generate {n}")

    def _conv(self, code: str, frm: str, to: str) -> str:
        if frm == to or to in ("l", "c"):
            return code
        return f"(({CTYPE[to]}){code})"

    def _pow(self, a, ta, b, tb, bnode):
        if tb == "i":
            if bnode.kind == "num" and bnode.val[1] in ("2", "3", "4"):
                e = int(bnode.val[1])
                fn = {"i": "ipow_i", "f": "ipow_f", "d": "ipow_d"}[ta]
                return f"{fn}{e}({a})", ta
            fn = {"i": "ipow_in", "f": "ipow_fn", "d": "ipow_dn"}[ta]
            return f"{fn}({a}, {b})", ta
        t = ta if RANK[ta] >= RANK[tb] else tb
        if t == "f":
            return f"powf({self._conv(a, ta, 'f')}, {self._conv(b, tb, 'f')})", "f"
        return f"pow({self._conv(a, ta, 'd')}, {self._conv(b, tb, 'd')})", "d"

    def _elem(self, arr: Array, args, sc: Scope, sect):
        if len(args) != len(arr.dims):
            raise TranslateError(f"rank mismatch for {arr.name}")
        idx = []
        si = 0
        for d, a in zip(arr.dims, args):
            if a.kind == "range":
                if sect is None:
                    raise TranslateError(f"section of {arr.name} outside an array context")
                lo = a.args[0]
                lo_c = "1" if lo is None else self.gen(lo, sc)[0]
                idx.append(f"(({lo_c}) + {sect[si]})")
                si += 1
            else:
                c, t = self.gen(a, sc, sect)
                if t != "i":
                    raise TranslateError(f"non-integer subscript for {arr.name}")
                idx.append(c)
        dims_c = [self.gen(d, sc)[0] for d in arr.dims]
        off = f"(({idx[-1]}) - 1)"
        for j in range(len(idx) - 2, -1, -1):
            off = f"(({idx[j]}) - 1) + ({dims_c[j]}) * ({off})"
        return f"{arr.name}[{off}]", arr.type

    def section_extents(self, n: Node, sc: Scope) -> list[str] | None:
        """Extents of the section an array reference denotes, or None if scalar."""
        if n.kind == "name" and sc.array(n.val) is not None:
            arr = sc.array(n.val)
            return [self.gen(d, sc)[0] for d in arr.dims]
        if n.kind == "call" and sc.array(n.val) is not None:
            arr = sc.array(n.val)
            ext = []
            for d, a in zip(arr.dims, n.args):
                if a.kind == "range":
                    lo = "1" if a.args[0] is None else self.gen(a.args[0], sc)[0]
                    hi = self.gen(d, sc)[0] if a.args[1] is None else self.gen(a.args[1], sc)[0]
                    ext.append(f"(({hi}) - ({lo}) + 1)")
            return ext if ext else None
        return None

    def find_section_shape(self, n: Node, sc: Scope):
        ext = self.section_extents(n, sc)
        if ext is not None:
            return ext
        if n.kind == "call" and sc.array(n.val) is None and n.val in ("MINVAL", "MAXVAL", "SUM"):
            return None
        for a in n.args or []:
            if isinstance(a, Node) and a.kind != "range":
                r = self.find_section_shape(a, sc)
                if r is not None:
                    return r
        return None

    def _intrinsic(self, name, args, sc, sect):
        if name in ("MINVAL", "MAXVAL", "SUM"):
            if len(args) != 1:
                raise TranslateError(f"{name} with mask/dim")
            ext = self.section_extents(args[0], sc)
            if ext is None:
                raise TranslateError(f"{name} of a non-array")
            self.uid += 1
            fn = f"_red{self.uid}"
            loops = [f"_q{d}" for d in range(len(ext))]
            body_c, t = self.gen(args[0], sc, loops)
            # emit a helper lambda-like block as a GNU statement expression
            init = {"MINVAL": "HUGE_VAL", "MAXVAL": "-HUGE_VAL", "SUM": "0.0"}[name]
            if t != "d":
                raise TranslateError(f"{name} over non-double array")
            code = f"({{ double {fn} = {init}; "
            for d in range(len(ext) - 1, -1, -1):
                code += f"for (int {loops[d]} = 0; {loops[d]} < {ext[d]}; ++{loops[d]}) "
            if name == "MINVAL":
                code += f"{{ double _v = {body_c}; if (_v < {fn}) {fn} = _v; }} "
            elif name == "MAXVAL":
                code += f"{{ double _v = {body_c}; if (_v > {fn}) {fn} = _v; }} "
            else:
                code += f"{{ {fn} = {fn} + {body_c}; }} "
            code += f"{fn}; }})"
            return code, "d"
        gargs = [self.gen(a, sc, sect) for a in args]
        if name in ("FLOAT", "REAL"):
            c, t = gargs[0]
            return f"((float){c})", "f"
        if name == "DBLE":
            c, t = gargs[0]
            return f"((double){c})", "d"
        if name == "INT":
            c, t = gargs[0]
            return f"((int){c})", "i"
        if name == "NINT":
            c, t = gargs[0]
            return f"((int)lround({c}))", "i"
        if name in ("MIN", "MAX"):
            t = max((g[1] for g in gargs), key=lambda x: RANK[x])
            cs = [self._conv(c, tt, t) for c, tt in gargs]
            fn = ("fmin_" if name == "MIN" else "fmax_") + t
            code = cs[0]
            for c in cs[1:]:
                code = f"{fn}({code}, {c})"
            return code, t
        if name == "MOD":
            (a, ta), (b, tb) = gargs
            if ta == "i" and tb == "i":
                return f"({a} % {b})", "i"
            t = "d" if "d" in (ta, tb) else "f"
            return f"fmod({self._conv(a, ta, 'd')}, {self._conv(b, tb, 'd')})", "d"
        if name == "ABS":
            c, t = gargs[0]
            return ({"i": f"abs({c})", "f": f"fabsf({c})", "d": f"fabs({c})"}[t]), t
        if name == "SIGN":
            (a, ta), (b, tb) = gargs
            return f"copysign({a}, {b})", ta
        if name in ("SQRT", "EXP", "LOG", "TANH", "COSH", "SINH", "COS", "SIN", "TAN", "ATAN", "ASIN"):
            c, t = gargs[0]
            if t == "i":
                raise TranslateError(f"{name} of integer")
            f = name.lower()
            return (f"{f}f({c})" if t == "f" else f"{f}({c})"), t
        raise TranslateError(f"unknown function or array {name}")

    # --- declarations ---------------------------------------------------
    def scan_decls(self, unit: str, stmts: list[Stmt], sc: Scope):
        head = stmts[0].text.upper()
        m = re.match(r"SUBROUTINE\s+(\w+)\s*(\((.*)\))?", head)
        if m and m.group(3):
            sc.dummies = [a.strip() for a in m.group(3).split(",") if a.strip()]
        for s in stmts[1:]:
            u = s.text.upper()
            if u.startswith("DIMENSION"):
                for item in _split_top(s.text[len("DIMENSION"):], ","):
                    item = item.strip()
                    nm = item[:item.index("(")].strip().upper()
                    dims = [parse_expr(d) for d in _split_top(item[item.index("(") + 1: item.rindex(")")], ",")]
                    sc.arrays[nm] = Array(nm, dims, sc.type_of(nm))
            elif u.startswith("COMMON"):
                body = re.sub(r"^COMMON\s*/\s*\w*\s*/", "", u)
                for nm in body.split(","):
                    sc.commons.add(nm.strip())
            elif u.startswith("LOGICAL"):
                for nm in u[len("LOGICAL"):].split(","):
                    sc.types[nm.strip()] = "l"
            elif u.startswith("INTEGER"):
                for nm in u[len("INTEGER"):].split(","):
                    sc.types[nm.strip()] = "i"
            elif u.startswith("DATA"):
                for nm, val in re.findall(r"(\w+)\s*/\s*([^/]*)/", s.text[4:]):
                    sc.saved[nm.upper()] = val.strip()
            elif u.startswith("PARAMETER"):
                body = s.text[s.text.index("(") + 1: s.text.rindex(")")]
                for item in _split_top(body, ","):
                    nm, ex = item.split("=", 1)
                    sc.params_local[nm.strip().upper()] = parse_expr(ex)
        for nm in sc.arrays:
            sc.arrays[nm].type = sc.type_of(nm)

    # --- statements -----------------------------------------------------
    def translate_unit(self, unit: str, stmts: list[Stmt]) -> str:
        sc = Scope(self, unit)
        self.scan_decls(unit, stmts, sc)
        # register COMMON arrays and scalars as globals
        for nm in sc.commons:
            if nm.startswith("SP") and nm[2:].isdigit():
                continue   # zero-length IPAD spacers
            if nm in sc.arrays:
                if nm not in self.global_arrays:
                    self.global_arrays[nm] = sc.arrays[nm]
            else:
                self.common_scalars.setdefault(nm, sc.type_of(nm))
        body: list[str] = []
        stack: list[tuple] = []
        for s in stmts[1:]:
            u = s.text.upper()
            kw = re.match(r"[A-Z]+(\*\d+)?", u)
            kw = kw.group(0) if kw else ""
            if kw in ("DIMENSION", "COMMON", "LOGICAL", "INTEGER", "DATA", "SAVE", "PARAMETER",
                      "IMPLICIT", "CHARACTER", "EXTERNAL", "REAL*8") or u.startswith("INCLUDE"):
                if u.startswith("INCLUDE") and self.param_base not in u and "MPIF.H" not in u:
                    raise TranslateError(f"INCLUDE {u}")
                continue
            if s.label is not None:
                body.append(f"L_{s.label}:;")
            self._stmt(s, u, sc, body, stack)
            if s.label is not None:
                while stack and stack[-1][0] == "do" and stack[-1][1] == s.label:
                    stack.pop()
                    body.append("}}")
        if stack:
            raise TranslateError(f"unclosed blocks in {unit}: {stack}")
        return self._emit_function(unit, sc, body)

    def _stmt(self, s: Stmt, u: str, sc: Scope, body: list[str], stack: list):
        t = s.text
        # DO loops
        m = re.match(r"^DO\s*(\d+)\s*,?\s*(\w+)\s*=(.*)$", t, re.I)
        m2 = None if m else re.match(r"^DO\s+(\w+)\s*=(.*)$", t, re.I)
        if m or m2:
            if m:
                lab, var, rng = int(m.group(1)), m.group(2).upper(), m.group(3)
            else:
                lab, var, rng = None, m2.group(1).upper(), m2.group(2)
            parts = _split_top(rng, ",")
            lo = self.gen(parse_expr(parts[0]), sc)[0]
            hi = self.gen(parse_expr(parts[1]), sc)[0]
            st = self.gen(parse_expr(parts[2]), sc)[0] if len(parts) > 2 else "1"
            sc.locals_used.add(var)
            self.uid += 1
            u_ = self.uid
            body.append(f"{{ const int _hi{u_} = {hi}, _st{u_} = {st}; "
                        f"for ({var} = {lo}; _st{u_} > 0 ? {var} <= _hi{u_} : {var} >= _hi{u_}; {var} += _st{u_}) {{")
            stack.append(("do", lab))
            return
        if re.fullmatch(r"END\s*DO", u):
            if not stack or stack[-1] != ("do", None):
                raise TranslateError(f"END DO mismatch at {s.line}")
            stack.pop()
            body.append("}}")
            return
        if u == "CONTINUE":
            return
        m = re.match(r"^IF\s*\((.*)\)\s*THEN$", t, re.I)
        if m and _balanced_prefix(t):
            c = self.gen(parse_expr(m.group(1)), sc)[0]
            body.append(f"if ({c}) {{")
            stack.append(("if",))
            return
        m = re.match(r"^ELSE\s*IF\s*\((.*)\)\s*THEN$", t, re.I)
        if m:
            c = self.gen(parse_expr(m.group(1)), sc)[0]
            body.append(f"}} else if ({c}) {{")
            return
        if u == "ELSE":
            body.append("} else {")
            return
        if re.fullmatch(r"END\s*IF", u):
            if not stack or stack[-1] != ("if",):
                raise TranslateError(f"END IF mismatch at {s.line}")
            stack.pop()
            body.append("}")
            return
        if re.match(r"^IF\s*\(", t, re.I):
            cond, rest = _split_logical_if(t)
            c = self.gen(parse_expr(cond), sc)[0]
            inner: list[str] = []
            self._stmt(Stmt(None, rest, s.line), rest.upper(), sc, inner, stack)
            body.append(f"if ({c}) {{ " + " ".join(inner) + " }")
            return
        if u == "RETURN":
            body.append("return;")
            return
        if u.startswith("STOP"):
            body.append(f'ref_stop("{sc.unit}", {s.line});')
            return
        m = re.match(r"^GO\s*TO\s*(\d+)$", u)
        if m:
            body.append(f"goto L_{m.group(1)};")
            return
        if u.startswith("WRITE") or u.startswith("PRINT"):
            body.append(f"/* WRITE at line {s.line} */;")
            return
        if u.startswith("CALL"):
            body.append(self._call(t[4:].strip(), sc, s.line))
            return
        # assignment
        eq = _top_level_eq(t)
        if eq is None:
            raise TranslateError(f"unsupported statement at line {s.line}: {t}")
        lhs, rhs = parse_expr(t[:eq]), parse_expr(t[eq + 1:])
        body.append(self._assign(lhs, rhs, sc))

    def _assign(self, lhs: Node, rhs: Node, sc: Scope) -> str:
        ext = self.section_extents(lhs, sc)
        if ext is None:
            lc, lt = self.gen(lhs, sc)
            rc, rt = self.gen(rhs, sc)
            return f"{lc} = {self._conv(rc, rt, lt)};"
        loops = [f"_s{d}" for d in range(len(ext))]
        rext = self.find_section_shape(rhs, sc)
        if rext is not None and len(rext) != len(ext):
            raise TranslateError("non-conforming array assignment")
        lc, lt = self.gen(lhs, sc, loops)
        rc, rt = self.gen(rhs, sc, loops)
        code = "{ "
        for d in range(len(ext) - 1, -1, -1):
            code += f"for (int {loops[d]} = 0; {loops[d]} < {ext[d]}; ++{loops[d]}) "
        code += f"{lc} = {self._conv(rc, rt, lt)}; }}"
        return code

    def _call(self, text: str, sc: Scope, line: int) -> str:
        n = parse_expr(text) if "(" in text else Node("call", text.strip().upper(), [])
        name = n.val
        if name.startswith("MPI_"):
            return self._mpi(name, n.args, sc, line)
        if name not in self.units:
            raise TranslateError(f"CALL of untranslated {name}")
        args = []
        for a in n.args:
            if a.kind == "name" and sc.array(a.val) is not None:
                args.append(a.val)
            elif a.kind == "name":
                sc.locals_used.add(a.val)
                args.append("&" + a.val)
            else:
                raise TranslateError(f"unsupported actual argument in CALL {name}")
        return f"sub_{name}({', '.join(args)});"

    def _buf(self, a: Node, sc: Scope, pre: list[str], post: list[str], count_c: str, inbound: bool, outbound: bool):
        """Address of an MPI buffer argument; sections go through a temporary."""
        if a.kind == "name" and sc.array(a.val) is not None:
            return a.val
        if a.kind == "name":
            sc.locals_used.add(a.val)
            return "&" + a.val
        if a.kind == "call" and sc.array(a.val) is not None:
            ext = self.section_extents(a, sc)
            if ext is None:
                return "&" + self.gen(a, sc)[0]
            self.uid += 1
            tmp = f"_tmp{self.uid}"
            loops = [f"_s{d}" for d in range(len(ext))]
            ec, _ = self.gen(a, sc, loops)
            lin = loops[0]
            for d in range(1, len(ext)):
                stride = " * ".join(ext[:d])
                lin = f"{lin} + ({stride}) * {loops[d]}"
            nest = ""
            for d in range(len(ext) - 1, -1, -1):
                nest += f"for (int {loops[d]} = 0; {loops[d]} < {ext[d]}; ++{loops[d]}) "
            pre.append(f"double* {tmp} = (double*)malloc(sizeof(double) * ({count_c}));")
            if outbound:
                pre.append(f"{nest}{tmp}[{lin}] = {ec};")
            if inbound:
                post.append(f"{nest}{ec} = {tmp}[{lin}];")
            post.append(f"free({tmp});")
            return tmp
        raise TranslateError("unsupported MPI buffer")

    def _mpi(self, name: str, args: list, sc: Scope, line: int) -> str:
        g = lambda a: self.gen(a, sc)[0]
        pre, post = [], []
        if name in ("MPI_INIT", "MPI_FINALIZE", "MPI_BARRIER", "MPI_COMM_RANK", "MPI_COMM_SIZE"):
            if name == "MPI_FINALIZE":
                return "ref_finalize();"
            raise TranslateError(f"{name} inside translated routines")
        if name == "MPI_SEND":
            cnt = g(args[1])
            b = self._buf(args[0], sc, pre, post, cnt, False, True)
            call = f"ref_send({b}, {cnt}, {g(args[2])}, {g(args[3])}, {g(args[4])});"
        elif name == "MPI_RECV":
            cnt = g(args[1])
            b = self._buf(args[0], sc, pre, post, cnt, True, False)
            call = f"ref_recv({b}, {cnt}, {g(args[2])}, {g(args[3])}, {g(args[4])});"
        elif name == "MPI_SENDRECV":
            c1, c2 = g(args[1]), g(args[6])
            b1 = self._buf(args[0], sc, pre, post, c1, False, True)
            b2 = self._buf(args[5], sc, pre, post, c2, True, False)
            call = (f"ref_sendrecv({b1}, {c1}, {g(args[2])}, {g(args[3])}, {g(args[4])}, "
                    f"{b2}, {c2}, {g(args[7])}, {g(args[8])}, {g(args[9])});")
        elif name == "MPI_ALLREDUCE":
            cnt = g(args[2])
            b1 = self._buf(args[0], sc, pre, post, cnt, False, True)
            b2 = self._buf(args[1], sc, pre, post, cnt, True, False)
            call = f"ref_allreduce({b1}, {b2}, {cnt}, {g(args[3])}, {g(args[4])});"
        elif name == "MPI_BCAST":
            cnt = g(args[1])
            b = self._buf(args[0], sc, pre, post, cnt, True, True)
            call = f"ref_bcast({b}, {cnt}, {g(args[2])}, {g(args[3])});"
        else:
            raise TranslateError(f"unsupported {name} at line {line}")
        return "{ " + " ".join(pre + [call] + post) + " }"

    def _emit_function(self, unit: str, sc: Scope, body: list[str]) -> str:
        params = []
        for d in sc.dummies:
            if sc.array(d) is not None:
                params.append(f"double* {d}")
            else:
                params.append(f"{CTYPE[sc.type_of(d)]}* {d}_p")
        decls = []
        for d in sc.dummies:
            if sc.array(d) is None:
                decls.append(f"#define {d} (*{d}_p)")
        for nm, arr in sc.arrays.items():
            if nm in sc.commons or nm in sc.dummies:
                continue
            dims = " * ".join(f"({self.gen(x, sc)[0]})" for x in arr.dims)
            if nm in sc.saved:
                raise TranslateError("DATA for arrays")
            decls.append(f"{CTYPE[arr.type]} {nm}[{dims}];")
        for nm, ex in sc.params_local.items():
            c, t = self.gen(ex, sc)
            decls.append(f"const {CTYPE[sc.type_of(nm)]} {nm} = {c};")
        skip = set(sc.commons) | set(sc.dummies) | set(self.param_types) | set(sc.arrays) \
            | set(self.global_types) | set(sc.params_local)
        for nm in sorted(sc.locals_used - skip):
            t = CTYPE[sc.type_of(nm)]
            if nm in sc.saved:
                c, tt = self.gen(parse_expr(sc.saved[nm]), sc)
                decls.append(f"static {t} {nm} = {c};")
            else:
                decls.append(f"{t} {nm} = 0;")
        for nm in sc.saved:
            if nm not in sc.locals_used and nm not in skip:
                c, tt = self.gen(parse_expr(sc.saved[nm]), sc)
                decls.append(f"static {CTYPE[sc.type_of(nm)]} {nm} = {c};")
        undefs = [f"#undef {d}" for d in sc.dummies if sc.array(d) is None]
        return (f"void sub_{unit}({', '.join(params) or 'void'})\n{{\n    "
                + "\n    ".join(decls + body) + "\n}\n" + "\n".join(undefs) + "\n")

    # --- whole program ----------------------------------------------------
    def translate(self, sub_file: str, wanted: list[str]) -> str:
        stmts = read_fixed_form(sub_file)
        allunits = split_units(stmts)
        for w in wanted:
            if w not in allunits:
                raise TranslateError(f"unit {w} not found")
            self.units[w] = allunits[w]
        funcs = [self.translate_unit(w, self.units[w]) for w in wanted]
        out = ["/* Generated from the reference source by oracle/fortran_subset.py -- do not commit. */",
               '#include "ref_harness.h"', ""]
        # parameters
        for nm, t in self.param_types.items():
            out.append(f"{CTYPE[t]} {nm};")
        out.append("void ref_params_init(void)\n{")
        sc0 = Scope(self, "_params")
        for nm, ex in self.param_order:
            c, t = self.gen(ex, sc0)
            pt = self.param_types[nm]
            out.append(f"    if (!ref_param_override(\"{nm}\", (void*)&{nm}, '{pt}')) {nm} = {self._conv(c, t, pt)};")
        out.append("}")
        # common scalars and arrays
        for nm, t in sorted(self.common_scalars.items()):
            out.append(f"{CTYPE[t]} {nm};")
        for nm, arr in sorted(self.global_arrays.items()):
            out.append(f"{CTYPE[arr.type]}* {nm};")
        out.append("void ref_commons_alloc(void)\n{")
        for nm, arr in sorted(self.global_arrays.items()):
            dims = " * ".join(f"(size_t)({self.gen(x, sc0)[0]})" for x in arr.dims)
            out.append(f"    {nm} = ({CTYPE[arr.type]}*)calloc({dims} + 1, sizeof({CTYPE[arr.type]}));")
        out.append("}")
        out.append("size_t ref_common_size(const char* name)\n{")
        for nm, arr in sorted(self.global_arrays.items()):
            dims = " * ".join(f"(size_t)({self.gen(x, sc0)[0]})" for x in arr.dims)
            out.append(f"    if (!strcmp(name, \"{nm}\")) return {dims};")
        out.append("    return 0;\n}")
        out.append("void* ref_common_ptr(const char* name)\n{")
        for nm in sorted(self.global_arrays):
            out.append(f"    if (!strcmp(name, \"{nm}\")) return {nm};")
        for nm in sorted(self.common_scalars):
            out.append(f"    if (!strcmp(name, \"{nm}\")) return &{nm};")
        for nm in sorted(self.param_types):
            out.append(f"    if (!strcmp(name, \"{nm}\")) return &{nm};")
        out.append("    return 0;\n}")
        for w in wanted:
            sig = funcs[wanted.index(w)].split("\n")[0]
            out.insert(3, sig + ";")
        out.extend(funcs)
        return "\n".join(out) + "\n"


def _split_top(s: str, sep: str) -> list[str]:
    out, depth, cur, q = [], 0, [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return out


def _top_level_eq(t: str):
    depth = 0
    for i, ch in enumerate(t):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            if i + 1 < len(t) and t[i + 1] == "=":
                return None
            if i > 0 and t[i - 1] in "<>/=":
                return None
            return i
    return None


def _balanced_prefix(t: str) -> bool:
    i = t.index("(")
    depth = 0
    for j in range(i, len(t)):
        if t[j] == "(":
            depth += 1
        elif t[j] == ")":
            depth -= 1
            if depth == 0:
                return t[j + 1:].strip().upper() == "THEN"
    return False


def _split_logical_if(t: str) -> tuple[str, str]:
    i = t.index("(")
    depth = 0
    for j in range(i, len(t)):
        if t[j] == "(":
            depth += 1
        elif t[j] == ")":
            depth -= 1
            if depth == 0:
                return t[i + 1:j], t[j + 1:].strip()
    raise TranslateError(f"bad logical IF {t}")
