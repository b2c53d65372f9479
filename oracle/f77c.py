"""Translator from the Fortran subset of the reference's FMM path to C99.

Test infrastructure only: it lets the tests and the CPU baseline run the
reference's own Fortran (no Fortran compiler exists in this image) by
translating its source files, where they lie, into C under ``oracle/_ref/``
and compiling them with gcc (``oracle/Makefile`` target ``ref``).  Nothing it
writes is committed; the product never loads it.

The subset is what fmm2d's Laplace and Helmholtz paths use: fixed-form
Fortran 77 with ``implicit`` typing, labelled and block DO loops, logical and
arithmetic IF, GOTO, DATA / SAVE / PARAMETER, F90 ALLOCATABLE arrays, and
``C$OMP PARALLEL DO`` directives (translated to ``#pragma omp parallel for``).
Calling convention follows gfortran's: every subroutine ``foo`` becomes
``void foo_(...)`` taking every argument by pointer, so the translated library
exports the reference's own symbols (``cfmm2d_``, ``lfmm2d_s_cd_g_``, ...).

Semantics kept on purpose, because parity depends on them:
* single-precision literals (``0.1`` without a ``d`` exponent) stay float,
  as gfortran compiles them;
* complex arithmetic is C99 ``double _Complex`` compiled with
  ``-fcx-fortran-rules`` (gfortran's complex division rules);
* integer ``**`` and real ``**`` integer use repeated multiplication;
* a DO loop's trip count is fixed on entry.
"""
import os
import re
import sys

CT = {"i": "int", "f": "float", "d": "double", "c": "float _Complex",
      "z": "double _Complex", "l": "int", "s": "char"}
RANK = {"l": 0, "i": 1, "f": 2, "d": 3, "c": 4, "z": 5}


class TranslateError(Exception):
    pass


# ---------------------------------------------------------------------------
# source form: fixed-form lines -> logical statements
# ---------------------------------------------------------------------------
def strip_inline_comment(s):
    out, q = [], None
    for ch in s:
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


def logical_lines(text):
    """Yields (label, statement, kind) with kind 'stmt' or 'omp'."""
    stmts = []
    for raw in text.split("\n"):
        line = raw.rstrip("\r\n")
        if "\t" in line[:6]:
            # tab form: the statement starts after the tab
            head, _, rest = line.partition("\t")
            if rest[:1].isdigit() and rest[:1] != "0" and not head.strip():
                line = " " * 5 + rest[0] + rest[1:]
            else:
                line = head.ljust(6)[:6] + rest
        line = line.replace("\t", " ")
        if not line.strip():
            continue
        c0 = line[:1]
        low = line.lower()
        if c0 in "cC*!":
            if low.startswith(("c$omp", "!$omp", "*$omp")):
                body = line[5:]
                if body.startswith("$") or body.startswith("&"):
                    if stmts and stmts[-1][2] == "omp":
                        lab, s, k = stmts[-1]
                        stmts[-1] = (lab, s + " " + body[1:].strip(), k)
                    continue
                stmts.append((None, body.strip(), "omp"))
                continue
            if low.startswith(("c$ ", "!$ ", "*$ ")) or re.match(r"^[c!*]\$\s", low):
                line = "  " + line[2:]
            else:
                continue
        line = line[:72]
        if line.strip().startswith("!"):
            continue
        lab = line[:5].strip()
        cont = line[5:6]
        body = strip_inline_comment(line[6:])
        if cont not in (" ", "0", ""):
            if not stmts:
                raise TranslateError("continuation without statement")
            plab, s, k = stmts[-1]
            stmts[-1] = (plab, s + body.strip("\n"), k)
            continue
        if not body.strip() and not lab:
            continue
        stmts.append((lab or None, body, "stmt"))
    out = []
    for lab, s, k in stmts:
        if k == "stmt":
            s = s.strip()
            # several statements on one line separated by ';'
            parts = split_top(s, ";") if ";" in s else [s]
            for i, p in enumerate(parts):
                if p.strip():
                    out.append((lab if i == 0 else None, p.strip(), k))
        else:
            out.append((lab, s, k))
    return out


def split_top(s, sep=","):
    """Splits at `sep` outside parentheses and quotes."""
    out, depth, q, cur = [], 0, None, []
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
        elif ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
            continue
        cur.append(ch)
    out.append("".join(cur))
    return out


def find_top(s, ch):
    depth, q = 0, None
    for i, c in enumerate(s):
        if q:
            if c == q:
                q = None
            continue
        if c in "'\"":
            q = c
        elif c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        elif c == ch and depth == 0:
            return i
    return -1


def lower_code(s):
    """Lower-cases outside string literals."""
    out, q = [], None
    for ch in s:
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


# ---------------------------------------------------------------------------
# expressions
# ---------------------------------------------------------------------------
TOK = re.compile(r"""
 (?P<ws>\s+)
|(?P<num>(\d+\.\d*|\.\d+|\d+)([eEdD][+-]?\d+)?(_\w+)?)
|(?P<dop>\.(eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
|(?P<name>[a-zA-Z_]\w*)
|(?P<str>'([^']|'')*'|"[^"]*")
|(?P<op>\*\*|//|==|/=|<=|>=|[-+*/(),:=<>%])
""", re.X)


def tokenize(s):
    toks, i = [], 0
    while i < len(s):
        m = TOK.match(s, i)
        if not m:
            raise TranslateError(f"cannot tokenize at: {s[i:]!r}")
        i = m.end()
        k = m.lastgroup
        if k == "ws":
            continue
        v = m.group(k)
        if k == "num":
            # "1.eq.2": the lexer would read "1." as a number
            if v.endswith(".") and re.match(r"\.(eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv)\.",
                                            s[i - 1:].lower()):
                v = v[:-1]
                i -= 1
        toks.append((k, v.lower() if k != "str" else v))
    return toks


class Parser:
    BIN = {".or.": 1, ".and.": 2, ".eqv.": 0, ".neqv.": 0,
           ".eq.": 4, ".ne.": 4, ".lt.": 4, ".le.": 4, ".gt.": 4, ".ge.": 4,
           "==": 4, "/=": 4, "<": 4, "<=": 4, ">": 4, ">=": 4,
           "//": 5, "+": 6, "-": 6, "*": 7, "/": 7, "**": 9}

    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, v):
        k, x = self.next()
        if x != v:
            raise TranslateError(f"expected {v!r}, got {x!r}")

    def parse(self, minp=0):
        k, v = self.peek()
        if v in ("-", "+"):
            self.next()
            # unary minus binds looser than ** and * (Fortran: -a**2 = -(a**2))
            e = self.parse(7)
            left = ("un", v, e)
        elif v == ".not.":
            self.next()
            left = ("un", "!", self.parse(3))
        else:
            left = self.primary()
        while True:
            k, v = self.peek()
            if v not in self.BIN:
                break
            p = self.BIN[v]
            if p < minp:
                break
            self.next()
            if v == "**":
                right = self.parse(p)  # right associative
            else:
                right = self.parse(p + 1)
            left = ("bin", v, left, right)
        return left

    def primary(self):
        k, v = self.next()
        if k == "num":
            return ("num", v)
        if k == "str":
            return ("str", v)
        if k == "dop" and v in (".true.", ".false."):
            return ("num", "1" if v == ".true." else "0", "l")
        if v == "(":
            e = self.parse()
            if self.peek()[1] == ",":
                self.next()
                e2 = self.parse()
                self.expect(")")
                return ("cplx", e, e2)
            self.expect(")")
            return ("paren", e)
        if k == "name":
            if self.peek()[1] == "(":
                self.next()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.arg())
                        if self.peek()[1] == ",":
                            self.next()
                            continue
                        break
                self.expect(")")
                return ("call", v, args)
            return ("var", v)
        raise TranslateError(f"unexpected token {v!r}")

    def arg(self):
        # keyword argument (stat=ier) or a section bound "a:b"
        k, v = self.peek()
        if k == "name" and self.i + 1 < len(self.t) and self.t[self.i + 1][1] == "=":
            self.next()
            self.next()
            return ("kw", v, self.parse())
        if v == ":":
            self.next()
            hi = None if self.peek()[1] in (",", ")") else self.parse()
            return ("range", None, hi)
        e = self.parse()
        if self.peek()[1] == ":":
            self.next()
            hi = None if self.peek()[1] in (",", ")") else self.parse()
            return ("range", e, hi)
        return e


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.parse()
    if p.i != len(p.t):
        raise TranslateError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return e


# ---------------------------------------------------------------------------
# symbols and program units
# ---------------------------------------------------------------------------
class Sym:
    def __init__(self, name):
        self.name = name
        self.type = None
        self.dims = None       # list of (lo, hi) expression trees; hi may be '*' or ':'
        self.is_arg = False
        self.alloc = False
        self.save = False
        self.data = None       # list of C initialiser strings (flat, column-major)
        self.param = None      # expression tree of a PARAMETER
        self.external = False
        self.charlen = None

    @property
    def is_array(self):
        return self.dims is not None


TYPE_WORDS = [
    (r"double\s*precision", "d"), (r"double\s*complex", "z"), (r"real\s*\*\s*8", "d"),
    (r"real\s*\*\s*4", "f"), (r"complex\s*\*\s*16", "z"), (r"complex\s*\*\s*8", "c"),
    (r"integer\s*\*\s*4", "i"), (r"integer\s*\*\s*8", "i"), (r"integer", "i"),
    (r"real\s*\(\s*(kind\s*=\s*)?8\s*\)", "d"), (r"complex\s*\(\s*(kind\s*=\s*)?8\s*\)", "z"),
    (r"real", "f"), (r"complex", "c"), (r"logical", "l"),
    (r"character\s*\*\s*\(\s*\*\s*\)", "s"), (r"character\s*\(\s*len\s*=\s*[\w*]+\s*\)", "s"),
    (r"character\s*\*\s*\d+", "s"), (r"character", "s"),
]


def match_type(s):
    for pat, t in TYPE_WORDS:
        m = re.match(pat + r"(?=[\s,:(*]|$)", s) if pat in ("real", "complex", "integer",
                                                            "logical", "character") \
            else re.match(pat, s)
        if m:
            return t, s[m.end():]
    return None, s


class Unit:
    def __init__(self, kind, name, args, rettype=None):
        self.kind = kind
        self.name = name
        self.args = args
        self.rettype = rettype
        self.syms = {}
        self.implicit = {}
        for c in "abcdefghopqrstuvwxyz":
            self.implicit[c] = "f"
        for c in "ijklmn":
            self.implicit[c] = "i"
        self.body = []      # (label, stmt, kind)
        self.omp = []

    def sym(self, name):
        if name not in self.syms:
            self.syms[name] = Sym(name)
        return self.syms[name]

    def type_of(self, name):
        s = self.syms.get(name)
        if s and s.type:
            return s.type
        t = self.implicit.get(name[0])
        if t is None:
            raise TranslateError(f"{self.name}: no type for {name} (implicit none)")
        return t


INTRINSIC_FUNCS = {
    "abs", "dabs", "iabs", "cdabs", "zabs", "sqrt", "dsqrt", "cdsqrt", "zsqrt", "exp", "dexp",
    "cdexp", "zexp", "log", "dlog", "cdlog", "zlog", "log10", "dlog10", "sin", "dsin", "cos",
    "dcos", "tan", "dtan", "atan", "datan", "atan2", "datan2", "asin", "dasin", "acos", "dacos",
    "sinh", "cosh", "tanh", "dble", "dfloat", "float", "real", "dreal", "imag", "dimag", "aimag",
    "conjg", "dconjg", "dcmplx", "cmplx", "max", "min", "max0", "min0", "dmax1", "dmin1",
    "amax1", "amin1", "mod", "int", "idint", "ifix", "nint", "idnint", "floor", "ceiling",
    "sign", "dsign", "isign", "omp_get_wtime", "omp_get_thread_num", "omp_get_num_threads",
    "omp_get_max_threads", "second", "huge", "epsilon", "tiny", "allocated", "size", "sngl", "dint",
    "aint", "anint", "dnint", "cabs", "maxval", "minval", "sum",
}


def c_name(n):
    return "v_" + n


# ---------------------------------------------------------------------------
# translation of one unit
# ---------------------------------------------------------------------------
class UnitTranslator:
    def __init__(self, unit, known_funcs, omp=True):
        self.u = unit
        self.funcs = known_funcs     # name -> return type of Fortran functions
        self.out = []
        self.ind = 1
        self.tmp = 0
        self.do_stack = []           # open DO loops: (label or None)
        self.omp = omp
        self.pending_omp = None
        self.region_stack = []
        self.do_close = {}
        self.labels_used = set()
        self.used = set()

    # ---- types ----------------------------------------------------------
    def etype(self, e):
        k = e[0]
        if k == "num":
            if len(e) > 2:
                return e[2]
            v = e[1]
            if re.search(r"d", v):
                return "d"
            if "." in v or "e" in v:
                if "_8" in v:
                    return "d"
                return "f"
            return "i"
        if k == "str":
            return "s"
        if k == "paren":
            return self.etype(e[1])
        if k == "cplx":
            t = max(self.etype(e[1]), self.etype(e[2]), key=lambda x: RANK.get(x, 0))
            return "z" if t in ("d", "z") else "c"
        if k == "var":
            s = self.u.syms.get(e[1])
            if s and s.param is not None:
                return self.u.type_of(e[1])
            return self.u.type_of(e[1])
        if k == "un":
            if e[1] == "!":
                return "l"
            return self.etype(e[2])
        if k == "bin":
            op = e[1]
            if op in (".eq.", ".ne.", ".lt.", ".le.", ".gt.", ".ge.", ".and.", ".or.", "==",
                      "/=", "<", "<=", ">", ">=", ".eqv.", ".neqv."):
                return "l"
            a, b = self.etype(e[2]), self.etype(e[3])
            return self.promote(a, b)
        if k == "call":
            n = e[1]
            s = self.u.syms.get(n)
            if s and s.is_array:
                return self.u.type_of(n)
            return self.func_type(n, e[2])
        raise TranslateError(f"etype {e}")

    @staticmethod
    def promote(a, b):
        if "z" in (a, b):
            return "z"
        if "c" in (a, b):
            return "z" if "d" in (a, b) else "c"
        if "d" in (a, b):
            return "d"
        if "f" in (a, b):
            return "f"
        return "i"

    def func_type(self, n, args):
        ats = [self.etype(a) for a in args if a[0] not in ("kw", "range")]
        at = ats[0] if ats else "d"
        if n in ("abs", "dabs", "cdabs", "zabs", "cabs"):
            return {"z": "d", "c": "f"}.get(at, at)
        if n == "iabs":
            return "i"
        if n in ("sqrt", "exp", "log", "sin", "cos", "tan", "atan", "asin", "acos", "sinh",
                 "cosh", "tanh", "log10"):
            return at if at != "i" else "f"
        if n in ("dsqrt", "dexp", "dlog", "dlog10", "dsin", "dcos", "dtan", "datan", "datan2",
                 "dasin", "dacos", "dble", "dfloat", "dreal", "dimag", "dmax1", "dmin1", "dsign",
                 "dint", "dnint"):
            return "d"
        if n in ("cdsqrt", "zsqrt", "cdexp", "zexp", "cdlog", "zlog", "dconjg", "dcmplx"):
            return "z"
        if n == "atan2":
            return self.promote(ats[0], ats[1])
        if n in ("float", "sngl", "amax1", "amin1"):
            return "f"
        if n == "real":
            if len(args) > 1:
                return "d"
            return {"z": "d", "c": "f"}.get(at, "f")
        if n in ("imag", "aimag"):
            return {"z": "d", "c": "f"}.get(at, "d")
        if n == "conjg":
            return at
        if n == "cmplx":
            if len(args) == 3:
                return "z"
            return "c"
        if n in ("max", "min"):
            t = ats[0]
            for x in ats[1:]:
                t = self.promote(t, x)
            return t
        if n in ("max0", "min0", "int", "idint", "ifix", "nint", "idnint", "floor",
                 "ceiling", "isign", "omp_get_thread_num", "omp_get_num_threads",
                 "omp_get_max_threads", "size"):
            return "i"
        if n in ("mod", "sign"):
            return self.promote(ats[0], ats[1])
        if n in ("aint", "anint"):
            return at
        if n == "omp_get_wtime":
            return "d"
        if n == "second":
            return "f"
        if n in ("huge", "epsilon", "tiny"):
            return at
        if n == "allocated":
            return "l"
        if n in ("maxval", "minval", "sum"):
            return self.u.type_of(args[0][1])
        if n in self.funcs:
            return self.funcs[n]
        s = self.u.syms.get(n)
        if s and s.type:
            return s.type
        return self.u.type_of(n)

    # ---- expressions ----------------------------------------------------
    def param_expr(self, n):
        s = self.u.syms[n]
        t = self.u.type_of(n)
        return f"(({CT[t]})({self.cx(s.param)}))"

    def scalar_ref(self, n):
        s = self.u.syms.get(n)
        if s is not None and s.param is not None:
            return self.param_expr(n)
        if self.u.kind == "function" and n == self.u.name:
            return "v__result"
        self.used.add(n)
        if s is not None and s.is_arg and not s.is_array:
            return f"(*{c_name(n)})"
        return c_name(n)

    def dim_names(self, n, d):
        return f"{c_name(n)}_l{d}", f"{c_name(n)}_e{d}"

    def index(self, n, idx):
        s = self.u.syms[n]
        if len(idx) != len(s.dims) and not (len(idx) == 1 and len(s.dims) > 1):
            raise TranslateError(f"{self.u.name}: rank mismatch for {n}")
        terms = None
        for d in reversed(range(len(idx))):
            lo, e = self.dim_names(n, d)
            sub = f"((long)({self.cx(idx[d])}) - {lo})"
            terms = sub if terms is None else f"({sub} + {e} * {terms})"
        return f"{c_name(n)}[{terms}]"

    def cx(self, e):
        k = e[0]
        if k == "num":
            if len(e) > 2:
                return e[1]
            v = e[1]
            t = self.etype(e)
            v = re.sub(r"_\w+$", "", v)
            if t == "i":
                return v
            v = v.replace("d", "e")
            if v.startswith("."):
                v = "0" + v
            if re.match(r"^\d+e", v):
                v = v.replace("e", ".e", 1)
            if v.endswith("."):
                v += "0"
            return v + ("f" if t == "f" else "")
        if k == "str":
            body = e[1][1:-1].replace("''", "'").replace("\\", "\\\\").replace('"', '\\"')
            return '"' + body + '"'
        if k == "paren":
            return f"({self.cx(e[1])})"
        if k == "cplx":
            t = self.etype(e)
            ft = "double" if t == "z" else "float"
            return f"__builtin_complex(({ft})({self.cx(e[1])}), ({ft})({self.cx(e[2])}))"
        if k == "var":
            n = e[1]
            s = self.u.syms.get(n)
            if s and s.is_array:
                return c_name(n)
            return self.scalar_ref(n)
        if k == "un":
            if e[1] == "!":
                return f"(!{self.cx(e[2])})"
            return f"({e[1]}{self.cx(e[2])})"
        if k == "bin":
            return self.cbin(e)
        if k == "call":
            n = e[1]
            s = self.u.syms.get(n)
            if s and s.is_array:
                return self.index(n, e[2])
            return self.ccall_func(n, e[2])
        raise TranslateError(f"cx {e}")

    def cbin(self, e):
        op, a, b = e[1], e[2], e[3]
        ta, tb = self.etype(a), self.etype(b)
        A, B = self.cx(a), self.cx(b)
        cops = {".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">",
                ".ge.": ">=", ".and.": "&&", ".or.": "||", "==": "==", "/=": "!=", "<": "<",
                "<=": "<=", ">": ">", ">=": ">=", "+": "+", "-": "-", "*": "*", "/": "/"}
        if op == "**":
            if tb == "i":
                if ta == "i":
                    return f"f77_ipow({A}, {B})"
                if ta in ("z", "c"):
                    return f"f77_zpowi({A}, {B})"
                if ta == "f":
                    return f"f77_fpowi({A}, {B})"
                return f"f77_dpowi({A}, {B})"
            t = self.promote(ta, tb)
            if t in ("z", "c"):
                return f"cpow({A}, {B})"
            if t == "f":
                return f"powf({A}, {B})"
            return f"pow({A}, {B})"
        if op == ".eqv.":
            return f"((!!({A})) == (!!({B})))"
        if op == ".neqv.":
            return f"((!!({A})) != (!!({B})))"
        if op == "//":
            raise TranslateError("string concatenation")
        return f"({A} {cops[op]} {B})"

    def ccall_func(self, n, args):
        if n in ("maxval", "minval", "sum"):
            a0 = args[0]
            if a0[0] == "var":
                arr, lo, hi = a0[1], None, None
            elif a0[0] == "call" and len(a0[2]) == 1 and a0[2][0][0] == "range":
                arr, lo, hi = a0[1], a0[2][0][1], a0[2][0][2]
            else:
                raise TranslateError(f"{n} of {a0}")
            s = self.u.syms[arr]
            if len(s.dims) != 1:
                raise TranslateError(f"{n} of a rank-{len(s.dims)} array")
            t = self.u.type_of(arr)
            ln, en = self.dim_names(arr, 0)
            lo_c = self.cx(lo) if lo is not None else ln
            hi_c = self.cx(hi) if hi is not None else f"({ln} + {en} - 1)"
            init = {"maxval": "-2147483647 - 1" if t == "i" else "-HUGE_VAL",
                    "minval": "2147483647" if t == "i" else "HUGE_VAL", "sum": "0"}[n]
            upd = {"maxval": "if (f77_x > f77_r) f77_r = f77_x;",
                   "minval": "if (f77_x < f77_r) f77_r = f77_x;", "sum": "f77_r += f77_x;"}[n]
            return (f"({{ {CT[t]} f77_r = {init}; for (long f77_q = {lo_c}; f77_q <= {hi_c}; "
                    f"f77_q++) {{ {CT[t]} f77_x = {c_name(arr)}[f77_q - {ln}]; {upd} }} f77_r; }})")
        ats = [self.etype(a) for a in args if a[0] not in ("kw",)]
        cs = [self.cx(a) for a in args if a[0] not in ("kw",)]
        at = ats[0] if ats else None
        c0 = cs[0] if cs else None
        cplx = at in ("z", "c")

        def fam(d, f=None, z=None):
            if at in ("z", "c"):
                return f"{z}({c0})"
            if at == "f":
                return f"{f}({c0})"
            return f"{d}((double)({c0}))"
        if n in ("abs", "dabs", "iabs", "cdabs", "zabs", "cabs"):
            if at == "i":
                return f"abs({c0})"
            return fam("fabs", "fabsf", "cabs")
        if n in ("sqrt", "dsqrt", "cdsqrt", "zsqrt"):
            return fam("sqrt", "sqrtf", "csqrt")
        if n in ("exp", "dexp", "cdexp", "zexp"):
            return fam("exp", "expf", "cexp")
        if n in ("log", "dlog", "cdlog", "zlog"):
            return fam("log", "logf", "clog")
        if n in ("log10", "dlog10"):
            return fam("log10", "log10f", "clog10")
        for f in ("sin", "cos", "tan", "atan", "asin", "acos", "sinh", "cosh", "tanh"):
            if n in (f, "d" + f):
                return fam(f, f + "f", "c" + f)
        if n in ("atan2", "datan2"):
            return f"atan2({cs[0]}, {cs[1]})"
        if n in ("dble", "dfloat", "dreal"):
            return f"creal({c0})" if cplx else f"((double)({c0}))"
        if n in ("float", "sngl"):
            return f"((float)({c0}))"
        if n == "real":
            if cplx:
                return f"creal({c0})"
            if len(cs) > 1:
                return f"((double)({c0}))"
            return f"((float)({c0}))"
        if n in ("imag", "dimag", "aimag"):
            return f"cimag({c0})"
        if n in ("conjg", "dconjg"):
            return f"conj({c0})"
        if n in ("dcmplx", "cmplx"):
            ft = "double" if n == "dcmplx" or len(cs) == 3 else "float"
            if len(cs) == 1:
                if cplx:
                    return f"(({CT['z' if ft == 'double' else 'c']})({c0}))"
                return f"__builtin_complex(({ft})({c0}), ({ft})0)"
            return f"__builtin_complex(({ft})({cs[0]}), ({ft})({cs[1]}))"
        if n in ("max", "min", "max0", "min0", "dmax1", "dmin1", "amax1", "amin1"):
            t = self.func_type(n, args)
            fn = "max" if "max" in n else "min"
            r = f"(({CT[t]})({cs[0]}))"
            for c in cs[1:]:
                r = f"f77_{fn}_{t}({r}, ({CT[t]})({c}))"
            return r
        if n == "mod":
            t = self.promote(ats[0], ats[1])
            if t == "i":
                return f"(({cs[0]}) % ({cs[1]}))"
            return f"fmod({cs[0]}, {cs[1]})"
        if n in ("int", "idint", "ifix"):
            if cplx:
                return f"((int)creal({c0}))"
            return f"((int)({c0}))"
        if n in ("aint", "dint"):
            return f"trunc({c0})"
        if n in ("anint", "dnint"):
            return f"round({c0})"
        if n in ("nint", "idnint"):
            return f"((int)lround({c0}))"
        if n == "floor":
            return f"((int)floor({c0}))"
        if n == "ceiling":
            return f"((int)ceil({c0}))"
        if n in ("sign", "dsign", "isign"):
            t = self.promote(ats[0], ats[1])
            return f"f77_sign_{t}({cs[0]}, {cs[1]})"
        if n == "omp_get_wtime":
            return "f77_wtime()"
        if n == "second":
            return "((float)f77_wtime())"
        if n in ("omp_get_thread_num", "omp_get_num_threads", "omp_get_max_threads"):
            return f"f77_{n}()"
        if n == "huge":
            return {"i": "2147483647", "f": "3.4028234663852886e38f"}.get(at, "1.7976931348623157e308")
        if n == "epsilon":
            return "1.1920929e-7f" if at == "f" else "2.220446049250313e-16"
        if n == "tiny":
            return "1.17549435e-38f" if at == "f" else "2.2250738585072014e-308"
        if n == "allocated":
            return f"({c_name(args[0][1])} != 0)"
        if n in self.funcs or (n in self.u.syms and self.u.syms[n].type):
            return f"{n}_({', '.join(self.actual(a) for a in args)})"
        if n in INTRINSIC_FUNCS:
            raise TranslateError(f"intrinsic {n} not mapped")
        return f"{n}_({', '.join(self.actual(a) for a in args)})"

    def actual(self, a):
        """C expression passing actual argument `a` by reference."""
        k = a[0]
        if k == "var":
            n = a[1]
            s = self.u.syms.get(n)
            if s is None or s.param is None:
                if s is not None and s.is_array:
                    return c_name(n)
                if s is not None and s.is_arg:
                    return c_name(n)
                if s is not None and s.external:
                    return f"(void*){n}_"
                if self.u.kind == "function" and n == self.u.name:
                    return "&v__result"
                self.used.add(n)
                return f"&{c_name(n)}"
        if k == "call":
            n = a[1]
            s = self.u.syms.get(n)
            if s and s.is_array:
                return f"&{self.index(n, a[2])}"
        if k == "str":
            return self.cx(a)
        if k == "paren" and a[1][0] == "var":
            pass
        t = self.etype(a)
        return f"&({CT[t]}){{{self.cx(a)}}}"

    # ---- statements -----------------------------------------------------
    def emit(self, s):
        self.out.append("  " * self.ind + s)

    def close_do(self):
        self.ind -= 1
        self.emit("}")
        for c in self.do_close.pop(len(self.do_stack) - 1, []):
            self.emit(c)
        self.ind -= 1
        self.emit("}")
        self.do_stack.pop()

    def close_labelled_dos(self, lab):
        while self.do_stack and self.do_stack[-1][0] == lab:
            self.close_do()

    def stmt(self, lab, s, kind):
        if kind == "omp":
            self.omp_directive(s)
            return
        if lab:
            self.labels_used.add(lab)
            self.emit(f"L{lab}: ;")
        self.stmt_body(s, lab)
        if lab:
            self.close_labelled_dos(lab)

    def omp_directive(self, s):
        if not self.omp:
            return
        low = lower_code(s).strip()
        m = re.match(r"^parallel\s+do\b(.*)$", low)
        if m:
            self.pending_omp = ("parallel for", m.group(1))
            return
        m = re.match(r"^do\b(.*)$", low)
        if m:
            self.pending_omp = ("for", m.group(1))
            return
        m = re.match(r"^parallel\b(.*)$", low)
        if m:
            r = self.omp_clauses(m.group(1))
            self.emit("#pragma omp parallel " + self.clause_str(r, with_sched=False))
            self.emit("{")
            self.ind += 1
            for d in self.heap_private_decls(r["heap"]):
                self.emit(d)
            self.region_stack.append(r["heap"])
            return
        if re.match(r"^end\s+parallel\s+do", low) or re.match(r"^end\s+do", low):
            return
        if re.match(r"^end\s+parallel", low):
            for n in self.region_stack.pop():
                self.emit(f"free({c_name(n)});")
            self.ind -= 1
            self.emit("}")
            return
        if low.startswith("barrier"):
            self.emit("#pragma omp barrier")
            return
        if low.startswith("critical"):
            self.emit("#pragma omp critical")
            self.emit("{")
            self.ind += 1
            return
        if low.startswith("end critical"):
            self.ind -= 1
            self.emit("}")
            return
        raise TranslateError(f"omp directive {s!r}")

    def omp_clauses(self, cl):
        """Parsed clauses: private scalars / fixed arrays (C private), heap
        arrays that each thread must get its own copy of, schedule, reduction."""
        r = {"private": [], "heap": [], "schedule": None, "reduction": [], "firstprivate": []}
        for m in re.finditer(r"(\w+)\s*(\(([^)]*)\))?", cl):
            w, arg = m.group(1), m.group(3)
            if w == "shared":
                continue  # default(shared) covers it
            if w in ("private", "firstprivate", "lastprivate"):
                if w == "lastprivate":
                    raise TranslateError("lastprivate")
                for n in [x.strip() for x in arg.split(",") if x.strip()]:
                    s = self.u.syms.get(n)
                    if s is not None and s.is_arg and not s.is_array:
                        raise TranslateError(f"{self.u.name}: private dummy scalar {n}")
                    if s is not None and s.param is not None:
                        continue
                    self.used.add(n)
                    if s is not None and s.is_array and (s.alloc or self.try_const_size(s) is None):
                        if w == "firstprivate":
                            raise TranslateError("firstprivate heap array")
                        r["heap"].append(n)
                    else:
                        r[w].append(c_name(n))
            elif w == "default":
                pass
            elif w == "schedule":
                r["schedule"] = arg.strip()
            elif w == "reduction":
                op, _, names = arg.partition(":")
                r["reduction"].append(f"reduction({op.strip()}:" +
                                      ", ".join(c_name(n.strip()) for n in names.split(",")) + ")")
            elif w in ("nowait", "no", "wait"):
                pass
            else:
                raise TranslateError(f"omp clause {w}")
        return r

    def clause_str(self, r, with_sched=True, with_priv=True):
        out = ["default(shared)"] if with_priv else []
        if with_priv:
            if r["private"]:
                out.append(f"private({', '.join(r['private'])})")
            if r["firstprivate"]:
                out.append(f"firstprivate({', '.join(r['firstprivate'])})")
            out += r["reduction"]
        if with_sched and r["schedule"]:
            out.append(f"schedule({r['schedule']})")
        return " ".join(out)

    def heap_private_decls(self, names):
        """Per-thread copies of heap arrays, sized like the shared ones."""
        out = []
        for n in names:
            t = self.u.type_of(n)
            s = self.u.syms[n]
            size = " * ".join(self.dim_names(n, d)[1] for d in range(len(s.dims)))
            out.append(f"{CT[t]}* {c_name(n)} = ({CT[t]}*)f77_alloc(sizeof({CT[t]}) * "
                       f"(({size}) > 0 ? ({size}) : 1));")
        return out

    def stmt_body(self, s, lab=None):
        low = lower_code(s).strip()
        # IF (...) THEN / logical IF / arithmetic IF
        m = re.match(r"^(else\s*)?if\s*\(", low)
        if m and not self.is_assignment(low):
            p = low.index("(", m.start())
            depth = 0
            for j in range(p, len(low)):
                if low[j] == "(":
                    depth += 1
                elif low[j] == ")":
                    depth -= 1
                    if depth == 0:
                        break
            cond = low[p + 1:j]
            rest = low[j + 1:].strip()
            if m.group(1):
                if rest != "then":
                    raise TranslateError(f"else if without then: {s}")
                self.ind -= 1
                self.emit(f"}} else if ({self.cx(parse_expr(cond))}) {{")
                self.ind += 1
                return
            if rest == "then":
                self.emit(f"if ({self.cx(parse_expr(cond))}) {{")
                self.ind += 1
                return
            if re.match(r"^\d+\s*,\s*\d+\s*,\s*\d+$", rest):
                l1, l2, l3 = [x.strip() for x in rest.split(",")]
                self.tmp += 1
                e = parse_expr(cond)
                t = self.etype(e)
                self.emit(f"{{ {CT[t]} f77_t{self.tmp} = {self.cx(e)}; "
                          f"if (f77_t{self.tmp} < 0) goto L{l1}; "
                          f"else if (f77_t{self.tmp} == 0) goto L{l2}; else goto L{l3}; }}")
                return
            self.emit(f"if ({self.cx(parse_expr(cond))}) {{")
            self.ind += 1
            self.stmt_body(rest)
            self.ind -= 1
            self.emit("}")
            return
        if low == "else":
            self.ind -= 1
            self.emit("} else {")
            self.ind += 1
            return
        if re.match(r"^end\s*if$", low):
            self.ind -= 1
            self.emit("}")
            return
        m = re.match(r"^do\s*while\s*\((.*)\)$", low)
        if m:
            if self.pending_omp:
                raise TranslateError("omp do on a do while")
            self.do_close[len(self.do_stack)] = []
            self.emit(f"while ({self.cx(parse_expr(m.group(1)))}) {{")
            self.ind += 1
            self.emit("{")
            self.ind += 1
            self.do_stack.append((None, None))
            return
        m = re.match(r"^do(\s+(\d+)\s*,?\s*|\s+)([a-z]\w*)\s*=(.+)$", low)
        if m and len(split_top(m.group(4))) >= 2:
            dlab = m.group(2)
            var = m.group(3)
            parts = [parse_expr(x) for x in split_top(m.group(4))]
            pragma, pclose = self.take_omp()
            self.tmp += 1
            k = self.tmp
            v = self.scalar_ref(var)
            vt = CT[self.u.type_of(var)]
            a, b = self.cx(parts[0]), self.cx(parts[1])
            if len(parts) == 3:
                st = self.cx(parts[2])
                if pragma:
                    raise TranslateError("omp do with a step")
                self.emit(f"{{ const {vt} f77_b{k} = {b}, f77_s{k} = {st};")
                self.emit(f"for ({v} = {a}; f77_s{k} > 0 ? {v} <= f77_b{k} : {v} >= f77_b{k};"
                          f" {v} += f77_s{k}) {{")
            else:
                self.emit(f"{{ const {vt} f77_b{k} = {b};")
                for p in pragma or []:
                    self.emit(p)
                self.emit(f"for ({v} = {a}; {v} <= f77_b{k}; {v}++) {{")
            self.ind += 1
            self.do_close[len(self.do_stack)] = pclose
            self.do_stack.append((dlab, var))
            return
        if re.match(r"^end\s*do$", low):
            self.close_do()
            return
        if low == "continue":
            return
        m = re.match(r"^go\s*to\s*(\d+)$", low)
        if m:
            self.labels_used.add(m.group(1))
            self.emit(f"goto L{m.group(1)};")
            return
        if low == "return":
            self.emit("goto f77_return;")
            return
        if low == "stop" or low.startswith("stop "):
            self.emit("exit(0);")
            return
        if low == "exit":
            self.emit("break;")
            return
        if low == "cycle":
            self.emit("continue;")
            return
        m = re.match(r"^call\s+([a-z]\w*)\s*(\((.*)\))?$", low)
        if m:
            name = m.group(1)
            args = []
            if m.group(3) and m.group(3).strip():
                args = [self.parse_arg(x) for x in split_top(m.group(3))]
            self.emit(f"{name}_({', '.join(self.actual(a) for a in args)});")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", low)
        if m:
            for item in split_top(m.group(1)):
                item = item.strip()
                if re.match(r"^stat\s*=", item):
                    var = item.split("=", 1)[1].strip()
                    self.emit(f"{self.scalar_ref(var)} = 0;")
                    continue
                self.allocate(item)
            return
        m = re.match(r"^deallocate\s*\((.*)\)$", low)
        if m:
            for item in split_top(m.group(1)):
                n = item.strip()
                if n.startswith("stat"):
                    continue
                self.emit(f"free({c_name(n)}); {c_name(n)} = 0;")
            return
        if re.match(r"^(write|print|format|read|open|close)\b", low):
            return
        if self.is_assignment(low):
            i = find_top(low, "=")
            lhs, rhs = low[:i].strip(), low[i + 1:].strip()
            L = parse_expr(lhs)
            R = parse_expr(rhs)
            if L[0] == "var":
                s = self.u.syms.get(L[1])
                if s is not None and s.is_array:
                    self.whole_array_assign(L[1], R)
                    return
            lt = self.etype(L)
            self.emit(f"{self.cx(L)} = ({CT[lt]})({self.cx(R)});")
            return
        raise TranslateError(f"{self.u.name}: cannot translate statement {s!r}")

    def parse_arg(self, x):
        x = x.strip()
        return Parser(tokenize(x)).arg()

    def whole_array_assign(self, n, R):
        if R[0] == "var" and self.u.syms.get(R[1]) and self.u.syms[R[1]].is_array:
            raise TranslateError("array copy")
        t = self.u.type_of(n)
        self.emit(f"for (long f77_k = 0; f77_k < {self.size_expr(n)}; f77_k++) "
                  f"{c_name(n)}[f77_k] = ({CT[t]})({self.cx(R)});")

    def size_expr(self, n):
        s = self.u.syms[n]
        parts = []
        for d, (lo, hi) in enumerate(s.dims):
            if hi in ("*", ":") and not s.alloc:
                raise TranslateError(f"size of assumed-size array {n}")
            parts.append(self.dim_names(n, d)[1])
        return " * ".join(parts)

    def take_omp(self):
        """Lines that open the pending OpenMP loop (emitted after the loop
        bounds, directly before the for) and the lines that close it."""
        if self.pending_omp is None:
            return None, []
        kind, cl = self.pending_omp
        self.pending_omp = None
        r = self.omp_clauses(cl)
        if not r["heap"]:
            return [f"#pragma omp {kind} {self.clause_str(r, with_priv=(kind != 'for'))}"], []
        if kind != "parallel for":
            raise TranslateError("heap private array on an orphaned omp do")
        opn = [f"#pragma omp parallel {self.clause_str(r, with_sched=False)}", "{"]
        opn += self.heap_private_decls(r["heap"])
        opn.append(f"#pragma omp for {self.clause_str(r, with_priv=False)}")
        close = [f"free({c_name(n)});" for n in r["heap"]] + ["}"]
        return opn, close

    def is_assignment(self, low):
        i = find_top(low, "=")
        if i < 0:
            return False
        if low[i + 1:i + 2] == "=" or low[i - 1:i] in ("/", "<", ">"):
            return False
        lhs = low[:i].strip()
        return re.match(r"^[a-z]\w*\s*(\(.*\))?$", lhs) is not None and not re.match(
            r"^(if|do)\s*\(", lhs)

    def allocate(self, item):
        m = re.match(r"^([a-z]\w*)\s*\((.*)\)$", item)
        if not m:
            raise TranslateError(f"allocate {item}")
        n = m.group(1)
        s = self.u.syms[n]
        dims = split_top(m.group(2))
        if len(dims) != len(s.dims):
            raise TranslateError(f"allocate rank {item}")
        sz = []
        for d, dd in enumerate(dims):
            if ":" in dd:
                lo, hi = dd.split(":", 1)
            else:
                lo, hi = "1", dd
            ln, en = self.dim_names(n, d)
            self.emit(f"{ln} = (long)({self.cx(parse_expr(lo))}); "
                      f"{en} = (long)({self.cx(parse_expr(hi))}) - {ln} + 1; "
                      f"if ({en} < 0) {en} = 0;")
            sz.append(en)
        t = self.u.type_of(n)
        self.emit(f"free({c_name(n)}); "
                  f"{c_name(n)} = ({CT[t]}*)f77_alloc(sizeof({CT[t]}) * {' * '.join(sz)});")

    # ---- unit ------------------------------------------------------------
    def translate(self):
        u = self.u
        params = []
        for a in u.args:
            s = u.sym(a)
            s.is_arg = True
            if s.external:
                params.append(f"void* {c_name(a)}")
                continue
            t = u.type_of(a)
            params.append(f"const char* {c_name(a)}" if t == "s" else f"{CT[t]}* {c_name(a)}")
        if u.kind == "function" and u.rettype is None:
            u.rettype = u.type_of(u.name)
        rt = CT[u.rettype] if u.kind == "function" else "void"
        self.proto = f"{rt} {u.name}_({', '.join(params) if params else 'void'})"
        # the body first: it records which undeclared names are used as variables
        self.out = []
        self.ind = 1
        self.used = set()
        for lab, st, kind in u.body:
            self.stmt(lab, st, kind)
        if self.do_stack:
            raise TranslateError("unclosed DO loop")
        body = self.out
        decl, entry, frees = [], [], []
        if u.kind == "function":
            decl.append(f"{rt} v__result = 0;")
        names = list(u.syms) + sorted(n for n in self.used if n not in u.syms)
        for n in names:
            s = u.syms.get(n) or Sym(n)
            if s.param is not None or s.external or (s.is_arg and not s.is_array):
                continue
            if u.kind == "function" and n == u.name:
                continue
            if not s.is_array and n not in self.used:
                continue  # declared but only used as a function name, or unused
            t = u.type_of(n)
            if t == "s":
                if not s.is_arg:
                    decl.append(f"const char* {c_name(n)} = 0;")
                continue
            if not s.is_array:
                if s.data is not None or s.save:
                    init = f" = {s.data[0]}" if s.data else ""
                    decl.append(f"static {CT[t]} {c_name(n)}{init};")
                else:
                    decl.append(f"{CT[t]} {c_name(n)};")
                continue
            if s.alloc:
                for d in range(len(s.dims)):
                    ln, en = self.dim_names(n, d)
                    decl.append(f"long {ln} = 1, {en} = 0;")
                decl.append(f"{CT[t]}* {c_name(n)} = 0;")
                frees.append(f"  free({c_name(n)});")
                continue
            for d, (lo, hi) in enumerate(s.dims):
                ln, en = self.dim_names(n, d)
                if hi == "*":
                    entry.append(f"const long {ln} = {self.cx(lo)}; const long {en} = 1;")
                else:
                    entry.append(f"const long {ln} = {self.cx(lo)}; "
                                 f"const long {en} = (long)({self.cx(hi)}) - {ln} + 1;")
            if s.is_arg:
                continue
            csize = self.try_const_size(s)
            if s.data is not None or s.save:
                init = " = {" + ", ".join(s.data) + "}" if s.data is not None else ""
                entry.append(f"static {CT[t]} {c_name(n)}[{csize}]{init};")
            elif csize is not None:
                entry.append(f"{CT[t]} {c_name(n)}[{max(csize, 1)}];")
            else:
                # automatic array: on the heap, as gfortran does without -fstack-arrays
                size = " * ".join(self.dim_names(n, d)[1] for d in range(len(s.dims)))
                entry.append(f"{CT[t]}* {c_name(n)} = ({CT[t]}*)f77_alloc(sizeof({CT[t]}) * "
                             f"(({size}) > 0 ? ({size}) : 1));")
                frees.append(f"  free({c_name(n)});")
        lines = [self.proto + " {"] + ["  " + d for d in decl] + ["  " + e for e in entry] + body
        lines.append("f77_return: ;")
        lines += frees
        if u.kind == "function":
            lines.append("  return v__result;")
        lines.append("}")
        return "\n".join(lines)

    def try_const_size(self, s):
        try:
            return self.const_size(s)
        except (TranslateError, ValueError, TypeError):
            return None

    def const_size(self, s):
        n = 1
        for lo, hi in s.dims:
            n *= int(eval_const(self.u, hi)) - int(eval_const(self.u, lo)) + 1
        return n


def eval_const(u, e):
    k = e[0]
    if k == "num":
        return float(e[1].replace("d", "e")) if any(c in e[1] for c in ".de") else int(e[1])
    if k == "var":
        s = u.syms.get(e[1])
        if s is None or s.param is None:
            raise TranslateError(f"not a constant: {e[1]}")
        return eval_const(u, s.param)
    if k == "paren":
        return eval_const(u, e[1])
    if k == "un":
        v = eval_const(u, e[2])
        return -v if e[1] == "-" else v
    if k == "bin":
        a, b = eval_const(u, e[2]), eval_const(u, e[3])
        if e[1] == "+":
            return a + b
        if e[1] == "-":
            return a - b
        if e[1] == "*":
            return a * b
        if e[1] == "/":
            return a // b if isinstance(a, int) and isinstance(b, int) else a / b
        if e[1] == "**":
            return a ** b
    raise TranslateError(f"not a constant expression {e}")


# ---------------------------------------------------------------------------
# declarations
# ---------------------------------------------------------------------------
def parse_dims(u, s):
    dims = []
    for d in split_top(s):
        d = d.strip()
        if d in ("*", ":"):
            dims.append((("num", "1"), d))
            continue
        if find_top(d, ":") >= 0:
            lo, hi = d.split(":", 1)
            hi = hi.strip()
            dims.append((parse_expr(lo), "*" if hi == "*" else (":" if not hi else parse_expr(hi))))
        else:
            dims.append((("num", "1"), parse_expr(d)))
    return dims


def parse_entities(u, text, t, attrs=()):
    for ent in split_top(text):
        ent = ent.strip()
        if not ent:
            continue
        init = None
        i = find_top(ent, "=")
        if i >= 0:
            ent, init = ent[:i].strip(), ent[i + 1:].strip()
        m = re.match(r"^([a-z]\w*)\s*(\*\s*\d+)?\s*(\((.*)\))?$", ent)
        if not m:
            raise TranslateError(f"{u.name}: declaration {ent!r}")
        n = m.group(1)
        s = u.sym(n)
        if t:
            s.type = t
            if m.group(2) and t == "d" and False:
                pass
        if m.group(4) is not None:
            s.dims = parse_dims(u, m.group(4))
        if "allocatable" in attrs:
            s.alloc = True
        if "parameter" in attrs and init is not None:
            s.param = parse_expr(init)
        if "save" in attrs:
            s.save = True
        if "external" in attrs:
            s.external = True


def data_values(u, text, dest_type):
    vals = []
    for v in split_top(text):
        v = v.strip()
        rep = 1
        m = re.match(r"^(\d+)\s*\*\s*(.*)$", v)
        if m and not re.match(r"^\d+\s*\*\s*\*", v):
            rep, v = int(m.group(1)), m.group(2)
        vals += [v] * rep
    return vals


def handle_data(u, tr, s):
    # data a, b /1, 2/, c(1), c(2) /3, 4/
    body = s[4:].strip()
    groups = re.findall(r"([^/]+)/([^/]*)/\s*,?", body)
    for names, values in groups:
        targets = []
        for n in split_top(names):
            n = n.strip()
            if not n:
                continue
            m = re.match(r"^([a-z]\w*)\s*(\((.*)\))?$", n)
            if not m:
                raise TranslateError(f"data target {n}")
            targets.append((m.group(1), m.group(3)))
        vals = data_values(u, values, None)
        k = 0
        for name, sub in targets:
            sym = u.sym(name)
            t = u.type_of(name)
            if sym.is_array and sub is None:
                size = tr.const_size(sym)
                init = []
                for _ in range(size):
                    init.append(c_init(tr, vals[k], t))
                    k += 1
                sym.data = init
            elif sym.is_array:
                idx = [int(eval_const(u, parse_expr(x))) for x in split_top(sub)]
                size = tr.const_size(sym)
                if sym.data is None:
                    sym.data = ["0"] * size
                lin, mul = 0, 1
                for d, (lo, hi) in enumerate(sym.dims):
                    lin += (idx[d] - int(eval_const(u, lo))) * mul
                    mul *= int(eval_const(u, hi)) - int(eval_const(u, lo)) + 1
                sym.data[lin] = c_init(tr, vals[k], t)
                k += 1
            else:
                sym.data = [c_init(tr, vals[k], t)]
                k += 1


def c_init(tr, v, t):
    e = parse_expr(v)
    return f"({CT[t]})({tr.cx(e)})"


def build_units(path):
    text = open(path, encoding="latin-1").read()
    units = []
    cur = None
    for lab, s, kind in logical_lines(text):
        if kind == "omp":
            if cur is not None:
                cur.body.append((lab, s, kind))
            continue
        low = lower_code(s).strip()
        m = re.match(r"^((?:[a-z]+\s*(?:\*\s*\d+)?\s+)*)?(subroutine|function)\s+([a-z]\w*)\s*(\((.*)\))?$",
                     low)
        if cur is None and m:
            prefix = (m.group(1) or "").strip()
            args = [a.strip() for a in (m.group(5) or "").split(",") if a.strip()]
            rt = None
            if m.group(2) == "function":
                rt, rest = match_type(prefix) if prefix else (None, "")
            cur = Unit(m.group(2), m.group(3), args, rt)
            if rt is not None:
                cur.sym(cur.name).type = rt
            units.append(cur)
            continue
        if cur is None:
            continue
        if re.match(r"^end(\s*(subroutine|function)(\s+\w+)?)?$", low):
            cur = None
            continue
        cur.body.append((lab, s, kind))
    return units


def process_decls(u, tr):
    body = []
    data_stmts = []
    for lab, s, kind in u.body:
        if kind == "omp":
            body.append((lab, s, kind))
            continue
        low = lower_code(s).strip()
        if low.startswith("implicit"):
            rest = low[8:].strip()
            if rest == "none":
                u.implicit = {}
                continue
            t, r = match_type(rest)
            if t is None:
                raise TranslateError(f"implicit {s}")
            for rng in re.findall(r"([a-z])\s*-\s*([a-z])", r):
                for c in range(ord(rng[0]), ord(rng[1]) + 1):
                    u.implicit[chr(c)] = t
            continue
        if "::" in low:
            head, ents = low.split("::", 1)
            parts = [p.strip() for p in split_top(head)]
            t, _ = match_type(parts[0])
            attrs = set()
            dimattr = None
            for p in parts[1:]:
                md = re.match(r"^dimension\s*\((.*)\)$", p)
                if md:
                    dimattr = md.group(1)
                    continue
                attrs.add(p)
            if dimattr is not None:
                ents = ",".join(e.strip() + (f"({dimattr})" if "(" not in e else "")
                                for e in split_top(ents))
            parse_entities(u, ents, t, attrs)
            continue
        t, rest = match_type(low)
        if t is not None and not tr.is_assignment(low) and (rest[:1] in (" ", ",", "") or
                                                             low.startswith(("real", "double",
                                                                             "complex",
                                                                             "integer",
                                                                             "character",
                                                                             "logical"))):
            if re.match(r"^\s*function\b", rest):
                raise TranslateError("typed function inside unit")
            parse_entities(u, rest.lstrip(", "), t)
            continue
        m = re.match(r"^dimension\s+(.*)$", low)
        if m:
            parse_entities(u, m.group(1), None)
            continue
        m = re.match(r"^parameter\s*\((.*)\)$", low)
        if m:
            for ent in split_top(m.group(1)):
                n, v = ent.split("=", 1)
                u.sym(n.strip()).param = parse_expr(v.strip())
            continue
        if re.match(r"^save\b", low):
            names = low[4:].strip()
            if not names:
                for sy in u.syms.values():
                    sy.save = True
            else:
                for n in split_top(names):
                    u.sym(n.strip()).save = True
            continue
        if re.match(r"^external\b", low):
            for n in split_top(low[8:]):
                u.sym(n.strip()).external = True
            continue
        if re.match(r"^intrinsic\b", low):
            continue
        if re.match(r"^data\b", low):
            data_stmts.append(low)
            continue
        body.append((lab, s, kind))
    for d in data_stmts:
        handle_data(u, tr, d)
    u.body = body


def referenced_names(u):
    names = set()
    for lab, s, kind in u.body:
        if kind == "omp":
            continue
        for k, v in tokenize(lower_code(s)) if True else []:
            if k == "name":
                names.add(v)
    return names


def translate_file(path, funcs, omp=True, skip_bad=True):
    units = build_units(path)
    out, protos, skipped = [], [], []
    for u in units:
        tr = UnitTranslator(u, funcs, omp)
        try:
            process_decls(u, tr)
            code = tr.translate()
        except TranslateError as e:
            if not skip_bad:
                raise TranslateError(f"{os.path.basename(path)}:{u.name}: {e}")
            skipped.append((u.name, str(e)))
            continue
        out.append(code)
        protos.append(tr.proto)
    return units, protos, out, skipped


RUNTIME = r"""
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <time.h>
static inline void* f77_alloc(size_t n) { void* p = malloc(n ? n : 1); if (!p) { fprintf(stderr, "f77_alloc failed\n"); abort(); } return p; }
static inline int f77_ipow(int a, int b) { int r = 1; if (b < 0) return a == 1 ? 1 : (a == -1 ? (b & 1 ? -1 : 1) : 0); while (b) { if (b & 1) r *= a; a *= a; b >>= 1; } return r; }
static inline double f77_dpowi(double a, int b) { double r = 1; int n = b < 0 ? -b : b; double x = a; while (n) { if (n & 1) r *= x; x *= x; n >>= 1; } return b < 0 ? 1 / r : r; }
static inline float f77_fpowi(float a, int b) { float r = 1; int n = b < 0 ? -b : b; float x = a; while (n) { if (n & 1) r *= x; x *= x; n >>= 1; } return b < 0 ? 1 / r : r; }
static inline double _Complex f77_zpowi(double _Complex a, int b) { double _Complex r = 1; int n = b < 0 ? -b : b; double _Complex x = a; while (n) { if (n & 1) r *= x; x *= x; n >>= 1; } return b < 0 ? 1 / r : r; }
static inline int f77_max_i(int a, int b) { return a > b ? a : b; }
static inline int f77_min_i(int a, int b) { return a < b ? a : b; }
static inline double f77_max_d(double a, double b) { return a > b ? a : b; }
static inline double f77_min_d(double a, double b) { return a < b ? a : b; }
static inline float f77_max_f(float a, float b) { return a > b ? a : b; }
static inline float f77_min_f(float a, float b) { return a < b ? a : b; }
static inline int f77_sign_i(int a, int b) { int x = a < 0 ? -a : a; return b >= 0 ? x : -x; }
static inline double f77_sign_d(double a, double b) { return copysign(fabs(a), b); }
static inline float f77_sign_f(float a, float b) { return copysignf(fabsf(a), b); }
static inline double f77_wtime(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  struct timespec t; clock_gettime(CLOCK_MONOTONIC, &t); return t.tv_sec + 1e-9 * t.tv_nsec;
#endif
}
#ifdef _OPENMP
static inline int f77_omp_get_thread_num(void) { return omp_get_thread_num(); }
static inline int f77_omp_get_num_threads(void) { return omp_get_num_threads(); }
static inline int f77_omp_get_max_threads(void) { return omp_get_max_threads(); }
#else
static inline int f77_omp_get_thread_num(void) { return 0; }
static inline int f77_omp_get_num_threads(void) { return 1; }
static inline int f77_omp_get_max_threads(void) { return 1; }
#endif
"""


STUBS = """
#include "f77rt.h"
/* printing helpers of src/common/prini.f: silent here */
void prini_() {}
void prin2_() {}
void prinf_() {}
void prinf_long_() {}
void prin2_long_() {}
void prinl_() {}
void cpu_time_(double* t) { *t = f77_wtime(); }
"""


def main(argv):
    """f77c.py OUT_DIR SRC.f ... : writes OUT_DIR/<name>.c for every source."""
    out_dir = argv[1]
    srcs = argv[2:]
    omp = os.environ.get("F77C_OMP", "1") == "1"
    os.makedirs(out_dir, exist_ok=True)
    # function return types (first pass)
    funcs = {}
    for p in srcs:
        for u in build_units(p):
            if u.kind == "function":
                rt = u.rettype
                if rt is None:
                    tr = UnitTranslator(u, {}, omp)
                    process_decls(u, tr)
                    rt = u.type_of(u.name)
                funcs[u.name] = rt
    results, names = [], {}
    for p in srcs:
        units, protos, code, skipped = translate_file(p, funcs, omp)
        for n, why in skipped:
            sys.stderr.write(f"f77c: skipped {os.path.basename(p)}:{n}: {why}\n")
        for u in units:
            names[u.name] = CT[funcs[u.name]] if u.kind == "function" else "void"
        results.append((p, code))
    with open(os.path.join(out_dir, "f77rt.h"), "w") as f:
        f.write("#pragma once\n" + RUNTIME + "\n")
        # unprototyped declarations: Fortran passes any array to any dummy
        for n in sorted(names):
            f.write(f"{names[n]} {n}_();\n")
        f.write("void prini_(); void prin2_(); void prinf_(); void prinf_long_();\n")
        f.write("void prin2_long_(); void prinl_(); void cpu_time_();\n")
    with open(os.path.join(out_dir, "f77stubs.c"), "w") as f:
        f.write(STUBS)
    for p, code in results:
        name = os.path.splitext(os.path.basename(p))[0]
        with open(os.path.join(out_dir, name + ".c"), "w") as f:
            f.write(f"/* translated from {os.path.basename(p)} by oracle/f77c.py */\n")
            f.write('#include "f77rt.h"\n\n')
            f.write("\n\n".join(code) + "\n")


if __name__ == "__main__":
    main(sys.argv)
