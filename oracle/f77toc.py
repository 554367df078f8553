#!/usr/bin/env python3
"""f77toc.py -- mechanical Fortran-77 -> C99 translation of LSMLIB toolbox routines.

TEST INFRASTRUCTURE ONLY (the oracle's "reference" build).  No Fortran compiler
exists on this machine, so the reference's own toolbox sources are compiled by
translating them statement by statement into C and building that C with gcc.
The translation keeps what decides the floating-point result bit for bit:

* every REAL is a C double (the reference's FP64 build uses -fdefault-real-8,
  configure.ac:242-246), every unsuffixed real literal is a double literal;
* expressions are parsed with Fortran precedence and left-to-right association
  and emitted fully parenthesised, so gcc (run with -ffp-contract=off, no
  -ffast-math) evaluates exactly the Fortran expression tree;
* x**2 is emitted as (x)*(x) (gfortran expands integer powers into multiplies);
* MAX/MIN over reals become a > b ? a : b chains (gfortran's MAX_EXPR, equal
  for non-NaN data), ABS on reals becomes fabs, SQRT sqrt;
* the configure substitutions of the FP64 build are applied
  (@tiny_nonzero_number@ = 1.d-99, @lsmlib_zero_tol@ = 1.d-11,
  configure.ac:264-272);
* arguments are passed by reference (F77 ABI); expression arguments of CALL
  become C99 compound-literal temporaries;
* DO loop bounds are evaluated once before the loop, as Fortran requires.

Only the statement forms used by the translated routines are supported
(declarations incl. LOGICAL, PARAMETER, DO/ENDDO, block IF/ELSEIF/ELSE/ENDIF,
CALL, RETURN, assignment; .EQV./.NEQV. and SIGN(a,b) as gfortran evaluates
them: |a| with the sign bit of b); anything else raises an error instead of
being guessed.

Usage: f77toc.py OUT.c SRC.f[.in]... -- reads the sources where they lie and
writes one C file whose functions are named ref_<lower-case fortran name>_.
"""
import re
import sys

SUBST = {"@tiny_nonzero_number@": "1.d-99", "@lsmlib_zero_tol@": "1.d-11"}

# ----------------------------------------------------------------------------
# fixed-form source -> logical statements
# ----------------------------------------------------------------------------

def expand_fixed(line):
    """Apply gfortran's fixed-form tab rule: a tab in the label field moves the
    statement to column 7; later tabs are blanks."""
    if line.startswith("\t"):
        rest = line[1:]
        if rest[:1].isdigit() and rest[:1] != "0":
            return "     " + rest[0] + rest[1:].replace("\t", " ")
        return "      " + rest.replace("\t", " ")
    head = line[:6]
    if "\t" in head:
        k = head.index("\t")
        return (line[:k] + " " * (6 - k) + line[k + 1:]).replace("\t", " ")
    return line.replace("\t", " ")


def logical_lines(text, path):
    out = []  # (lineno, text)
    for no, raw in enumerate(text.split("\n"), 1):
        for k, v in SUBST.items():
            raw = raw.replace(k, v)
        if not raw.strip():
            continue
        if raw[0] in "cC*!":
            continue
        line = expand_fixed(raw.rstrip("\n"))
        body = line[6:72]
        if len(line) > 72 and line[72:].strip():
            raise SystemExit("%s:%d: text beyond column 72" % (path, no))
        if "!" in body:
            body = body[: body.index("!")]
        cont = len(line) > 5 and line[5] not in " 0"
        if cont:
            if not out:
                raise SystemExit("%s:%d: continuation without statement" % (path, no))
            out[-1] = (out[-1][0], out[-1][1] + " " + body)
        else:
            out.append((no, body))
    # ';' separates statements (a trailing ';' leaves an empty statement)
    res = []
    for n, s in out:
        for part in s.split(";"):
            if part.strip():
                res.append((n, part.strip().lower()))
    return res


# ----------------------------------------------------------------------------
# expressions
# ----------------------------------------------------------------------------
TOK = re.compile(r"""
  (?P<num>(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?)
 |(?P<dotop>\.(lt|le|gt|ge|eq|ne|and|or|not|true|false|eqv|neqv)\.)
 |(?P<id>[a-z_][a-z0-9_]*)
 |(?P<pow>\*\*)
 |(?P<op>[-+*/(),=:])
 |(?P<ws>\s+)
""", re.X)


def tokenize(s):
    pos, toks = 0, []
    while pos < len(s):
        m = TOK.match(s, pos)
        if not m:
            raise SyntaxError("cannot tokenize: %r at %d" % (s, pos))
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group(kind)
        if kind == "num":
            # a number immediately followed by a dot-operator was over-eaten:
            # "1.eq." is impossible here, but "2.and." would be; guard anyway
            pass
        toks.append((kind, val))
    return toks


class P:
    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError("expected %r got %r" % (val, tok))
        self.i += 1
        return tok

    # Fortran precedence: .eqv./.neqv. < .or. < .and. < .not. < relational
    # < +,- < *,/ < **
    def expr(self):
        a = self.orx()
        while self.peek()[1] in (".eqv.", ".neqv."):
            op = self.take()[1]
            a = ("eqv" if op == ".eqv." else "neqv", a, self.orx())
        return a

    def orx(self):
        a = self.andx()
        while self.peek()[1] == ".or.":
            self.take(); a = ("or", a, self.andx())
        return a

    def andx(self):
        a = self.notx()
        while self.peek()[1] == ".and.":
            self.take(); a = ("and", a, self.notx())
        return a

    def notx(self):
        if self.peek()[1] == ".not.":
            self.take(); return ("not", self.notx())
        return self.rel()

    RELS = {".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">=",
            ".eq.": "==", ".ne.": "!="}

    def rel(self):
        a = self.add()
        if self.peek()[1] in self.RELS:
            op = self.RELS[self.take()[1]]
            a = ("rel", op, a, self.add())
        return a

    def add(self):
        # leading unary sign applies to the first term: -a*b = -(a*b)
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
            a = self.mul()
            if sign == "-":
                a = ("neg", a)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.pw()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = ("bin", op, a, self.pw())
        return a

    def pw(self):
        a = self.prim()
        if self.peek()[0] == "pow":
            self.take()
            # right associative; the exponent may carry a sign
            if self.peek()[1] in ("+", "-"):
                sign = self.take()[1]
                b = self.pw()
                b = ("neg", b) if sign == "-" else b
            else:
                b = self.pw()
            a = ("pow", a, b)
        return a

    def prim(self):
        kind, val = self.peek()
        if kind == "num":
            self.take(); return ("num", val)
        if kind == "id":
            self.take()
            if self.peek()[1] == "(":
                self.take()
                args = []
                if self.peek()[1] != ")":
                    args.append(self.expr())
                    while self.peek()[1] == ",":
                        self.take(); args.append(self.expr())
                self.take(")")
                return ("ref", val, args)
            return ("id", val)
        if val == "(":
            self.take(); a = self.expr(); self.take(")")
            return ("paren", a)
        if val in (".true.", ".false."):
            self.take(); return ("bool", val == ".true.")
        raise SyntaxError("unexpected token %r" % (val,))


def parse_expr(s):
    p = P(tokenize(s))
    e = p.expr()
    if p.i != len(p.t):
        raise SyntaxError("trailing tokens in %r" % s)
    return e


def c_num(v):
    if re.fullmatch(r"\d+", v):
        return v, "int"
    m = re.fullmatch(r"(\d*)\.?(\d*)([ed])?([+-]?\d+)?", v)
    mant = v
    exp = ""
    k = re.search(r"[ed]", v)
    if k:
        mant, exp = v[: k.start()], v[k.start() + 1:]
    if "." not in mant:
        mant = mant + ".0"
    if mant.endswith("."):
        mant += "0"
    if mant.startswith("."):
        mant = "0" + mant
    return mant + ("e" + exp if exp else ""), "real"


INTRINSIC = {"abs", "max", "min", "sqrt", "mod", "dble", "real", "int",
             "float", "sign", "exp", "log", "sin", "cos", "nint"}


class Sub:
    def __init__(self, name, args):
        self.name, self.args = name, args
        self.types = {}      # name -> 'int' | 'real'
        self.dims = {}       # name -> list of (lo_expr, hi_expr)
        self.params = {}     # name -> expr string
        self.param_order = []
        self.body = []       # (lineno, stmt)

    # ---- typing ----
    def etype(self, e):
        k = e[0]
        if k == "num":
            return c_num(e[1])[1]
        if k == "id":
            return self.types.get(e[1], "real" if e[1][0] not in "ijklmn" else "int")
        if k == "paren":
            return self.etype(e[1])
        if k == "neg":
            return self.etype(e[1])
        if k in ("bin",):
            a, b = self.etype(e[2]), self.etype(e[3])
            return "real" if "real" in (a, b) else "int"
        if k == "pow":
            return self.etype(e[1])
        if k in ("rel", "and", "or", "not", "eqv", "neqv", "bool"):
            return "logical"
        if k == "ref":
            f = e[1]
            if f in self.dims:
                return self.types[f]
            if f in ("sqrt", "dble", "real", "float", "exp", "log", "sin", "cos"):
                return "real"
            if f in ("int", "nint", "mod"):
                return "int"
            ts = [self.etype(a) for a in e[2]]
            return "real" if "real" in ts else "int"
        raise ValueError(e)

    def is_dummy(self, n):
        return n in self.args

    # ---- emission ----
    def cx(self, e):
        k = e[0]
        if k == "num":
            return c_num(e[1])[0]
        if k == "id":
            n = e[1]
            if n in self.dims:
                return n
            if self.is_dummy(n):
                return "(*%s)" % n
            return n
        if k == "paren":
            return "(%s)" % self.cx(e[1])
        if k == "neg":
            return "(-%s)" % self.cx(e[1])
        if k == "bin":
            a, b = self.cx(e[2]), self.cx(e[3])
            if e[1] == "/" and self.etype(e) == "int":
                return "(%s / %s)" % (a, b)
            return "(%s %s %s)" % (a, e[1], b)
        if k == "pow":
            base, ex = e[1], e[2]
            if ex == ("num", "2"):
                b = self.cx(base)
                return "(%s * %s)" % (b, b)
            raise SyntaxError("unsupported power %r" % (ex,))
        if k == "rel":
            return "(%s %s %s)" % (self.cx(e[2]), e[1], self.cx(e[3]))
        if k == "and":
            return "(%s && %s)" % (self.cx(e[1]), self.cx(e[2]))
        if k == "or":
            return "(%s || %s)" % (self.cx(e[1]), self.cx(e[2]))
        if k == "not":
            return "(!%s)" % self.cx(e[1])
        if k == "bool":
            return "1" if e[1] else "0"
        if k in ("eqv", "neqv"):
            return "((!!%s) %s (!!%s))" % (self.cx(e[1]), "==" if k == "eqv" else "!=",
                                           self.cx(e[2]))
        if k == "ref":
            f, args = e[1], e[2]
            if f in self.dims:
                return "%s[%s]" % (f, self.index(f, args))
            if f == "abs":
                t = self.etype(args[0])
                return ("fabs(%s)" if t == "real" else "abs(%s)") % self.cx(args[0])
            if f in ("max", "min"):
                t = "real" if "real" in [self.etype(a) for a in args] else "int"
                fn = ("f77_%s_r" if t == "real" else "f77_%s_i") % f
                acc = self.cx(args[0])
                for a in args[1:]:
                    acc = "%s(%s, %s)" % (fn, acc, self.cx(a))
                return acc
            if f == "sqrt":
                return "sqrt(%s)" % self.cx(args[0])
            if f == "sign" and "real" in [self.etype(a) for a in args]:
                # |a| with the sign of b (gfortran: the sign bit of b)
                return "copysign(fabs(%s), %s)" % (self.cx(args[0]), self.cx(args[1]))
            if f == "mod":
                return "(%s %% %s)" % (self.cx(args[0]), self.cx(args[1]))
            if f in ("dble", "real", "float"):
                return "((double)%s)" % self.cx(args[0])
            if f == "int":
                return "((int)%s)" % self.cx(args[0])
            raise SyntaxError("unsupported function %s" % f)
        raise ValueError(e)

    def bound(self, s):
        return self.cx(parse_expr(s))

    def index(self, name, args):
        dims = self.dims[name]
        if len(args) != len(dims):
            raise SyntaxError("rank mismatch for %s" % name)
        # column-major: off = (i1-lo1) + n1*((i2-lo2) + n2*(i3-lo3))
        terms = None
        for (lo, hi), a in reversed(list(zip(dims, args))):
            d = "((long)%s - (long)%s)" % (self.cx(a), self.bound(lo))
            if terms is None:
                terms = d
            else:
                n = "((long)%s - (long)%s + 1)" % (self.bound(hi), self.bound(lo))
                terms = "%s + %s * (%s)" % (d, n, terms)
        return terms


def split_top(s, sep=","):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur); cur = ""
        else:
            cur += ch
    out.append(cur)
    return [x.strip() for x in out if x.strip() != ""]


def parse_units(lines, path):
    subs, cur = [], None
    for no, s in lines:
        m = re.match(r"subroutine\s+([a-z0-9_]+)\s*\((.*)\)\s*$", s)
        if m:
            cur = Sub(m.group(1), [a.strip() for a in m.group(2).split(",") if a.strip()])
            cur.path = path
            cur.lineno = no
            subs.append(cur)
            continue
        if cur is None:
            raise SystemExit("%s:%d: statement outside subroutine" % (path, no))
        if s == "end":
            cur.body.append((no, "end"))
            cur = None
            continue
        if s == "implicit none":
            continue
        m = re.match(r"(integer|real|double precision|logical)\s+(.*)$", s)
        if m and not re.match(r"(integer|real|logical)\s*=", s):
            t = {"integer": "int", "logical": "int"}.get(m.group(1), "real")
            for item in split_top(m.group(2)):
                mm = re.match(r"([a-z0-9_]+)\s*(\((.*)\))?$", item)
                if not mm:
                    raise SystemExit("%s:%d: bad declaration %r" % (path, no, item))
                n = mm.group(1)
                cur.types[n] = t
                if mm.group(2):
                    dims = []
                    for d in split_top(mm.group(3)):
                        if ":" in d:
                            lo, hi = split_top(d, ":")
                        else:
                            lo, hi = "1", d
                        dims.append((lo, hi))
                    cur.dims[n] = dims
            continue
        m = re.match(r"parameter\s*\((.*)\)$", s)
        if m:
            for item in split_top(m.group(1)):
                n, v = item.split("=", 1)
                cur.params[n.strip()] = v.strip()
                cur.param_order.append(n.strip())
            continue
        cur.body.append((no, s))
    return subs


def emit_sub(sub, known, out):
    cname = "ref_%s_" % sub.name
    args = []
    for a in sub.args:
        t = sub.types.get(a)
        if t is None:
            raise SystemExit("%s: undeclared dummy %s" % (sub.name, a))
        args.append(("double *%s" if t == "real" else "int *%s") % a)
    out.append("/* %s, %s:%d */" % (sub.name, sub.path.split("/src/")[-1] if "/src/" in sub.path else sub.path, sub.lineno))
    out.append("void %s(%s) {" % (cname, ", ".join(args)))
    # parameters (as constants, in declaration order)
    for n in sub.param_order:
        t = sub.types.get(n, "real")
        ct = "double" if t == "real" else "int"
        out.append("  const %s %s = %s;" % (ct, n, sub.cx(parse_expr(sub.params[n]))))
    # locals
    for n, t in sub.types.items():
        if n in sub.args or n in sub.params:
            continue
        ct = "double" if t == "real" else "int"
        if n in sub.dims:
            size = "1"
            for lo, hi in sub.dims[n]:
                size = "(%s) * (%s - %s + 1)" % (size, sub.bound(hi), sub.bound(lo))
            out.append("  %s %s[%s];" % (ct, n, size))
        else:
            out.append("  %s %s;" % (ct, n))
    depth = 1
    loopno = 0
    for no, s in sub.body:
        ind = "  " * depth
        if s == "end":
            break
        if s == "return":
            out.append(ind + "return;")
            continue
        if s in ("enddo", "end do"):
            depth -= 1
            out.append("  " * depth + "}}")
            continue
        if s in ("endif", "end if"):
            depth -= 1
            out.append("  " * depth + "}")
            continue
        if s == "else":
            out.append("  " * (depth - 1) + "} else {")
            continue
        m = re.match(r"else\s*if\s*\((.*)\)\s*then$", s)
        if m:
            out.append("  " * (depth - 1) + "} else if (%s) {" % sub.cx(parse_expr(m.group(1))))
            continue
        m = re.match(r"if\s*\((.*)\)\s*then$", s)
        if m:
            out.append(ind + "if (%s) {" % sub.cx(parse_expr(m.group(1))))
            depth += 1
            continue
        m = re.match(r"do\s+([a-z0-9_]+)\s*=\s*(.*)$", s)
        if m:
            v = m.group(1)
            parts = split_top(m.group(2))
            if len(parts) != 2:
                raise SystemExit("%s:%d: unsupported DO form" % (sub.path, no))
            lo, hi = [sub.cx(parse_expr(x)) for x in parts]
            loopno += 1
            out.append(ind + "{ const long hi_%d = %s; for (%s = %s; %s <= hi_%d; %s++) {"
                       % (loopno, hi, v, lo, v, loopno, v))
            depth += 1
            continue
        m = re.match(r"call\s+([a-z0-9_]+)\s*\((.*)\)$", s)
        if m:
            callee = m.group(1)
            if callee not in known:
                raise SystemExit("%s:%d: call to untranslated %s" % (sub.path, no, callee))
            cargs = []
            for a in split_top(m.group(2)):
                e = parse_expr(a)
                if e[0] == "id" and (e[1] in sub.dims or sub.is_dummy(e[1])):
                    cargs.append(e[1])
                elif e[0] == "id" and e[1] not in sub.params:
                    cargs.append("&" + e[1])
                else:
                    t = sub.etype(e)
                    ct = "double" if t == "real" else "int"
                    cargs.append("&(%s){%s}" % (ct, sub.cx(e)))
            out.append(ind + "ref_%s_(%s);" % (callee, ", ".join(cargs)))
            continue
        m = re.match(r"([a-z0-9_]+\s*(\(.*?\))?)\s*=\s*(.*)$", s)
        if m:
            lhs = parse_expr(m.group(1))
            rhs = parse_expr(m.group(3))
            out.append(ind + "%s = %s;" % (sub.cx(lhs), sub.cx(rhs)))
            continue
        raise SystemExit("%s:%d: unsupported statement %r" % (sub.path, no, s))
    out.append("}")
    out.append("")


HEADER = """/* Generated by oracle/f77toc.py from the reference's Fortran sources.
 * Build output only (oracle/_ref/), never committed. */
#include <math.h>
#include <stdlib.h>
static inline double f77_max_r(double a, double b) { return a > b ? a : b; }
static inline double f77_min_r(double a, double b) { return a < b ? a : b; }
static inline int f77_max_i(int a, int b) { return a > b ? a : b; }
static inline int f77_min_i(int a, int b) { return a < b ? a : b; }
"""


def main(argv):
    out_path, srcs = argv[1], argv[2:]
    want = None
    if srcs and srcs[0].startswith("--only="):
        want = set(srcs[0][7:].split(","))
        srcs = srcs[1:]
    subs = []
    for p in srcs:
        subs += parse_units(logical_lines(open(p).read(), p), p)
    if want is not None:
        # keep wanted routines and everything they call, transitively
        byname = {s.name: s for s in subs}
        keep, todo = set(), list(want)
        while todo:
            n = todo.pop()
            if n in keep:
                continue
            if n not in byname:
                raise SystemExit("routine %s not found" % n)
            keep.add(n)
            for _, st in byname[n].body:
                m = re.match(r"call\s+([a-z0-9_]+)", st)
                if m:
                    todo.append(m.group(1))
        subs = [s for s in subs if s.name in keep]
    known = {s.name for s in subs}
    out = [HEADER]
    for s in subs:
        args = []
        for a in s.args:
            args.append(("double *" if s.types.get(a) == "real" else "int *") + a)
        out.append("void ref_%s_(%s);" % (s.name, ", ".join(args)))
    out.append("")
    for s in subs:
        emit_sub(s, known, out)
    open(out_path, "w").write("\n".join(out) + "\n")
    print("translated %d routines -> %s" % (len(subs), out_path))


if __name__ == "__main__":
    main(sys.argv)
