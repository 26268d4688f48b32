"""Literal execution of the reference's Fortran FLUXES LMAG branch on numpy arrays.

Test infrastructure (the checker for the MHD restatement in r3d_oracle.c): the reference C++
aborts on --lmag (src/fluxes.cpp:539-541) and no Fortran compiler or MPI exists here, so the
Fortran source itself (golden/fortran/3dmhdsub.f, the `IF (LMAG) THEN ... ENDIF` block of
SUBROUTINE FLUXES, lines 2146-2651) is read and its statements are executed as written:

* fixed-form lines: comments (c, C, *, ! in column 1) dropped, continuation lines (non-blank,
  non-zero column 6, or a leading tab followed by a digit 1-9) joined, statement labels taken
  from columns 1-5;
* statements: `DO <label> <var>=<lo>,<hi>` nests closed by `<label> CONTINUE`, assignments to
  arrays or scalars, and `IF (MYPEZ.EQ.0) THEN / ELSE IF (MYPEZ.EQ.NPEZ-1) THEN / ENDIF`;
* expressions: a recursive-descent parser for + - * / and ** (left to right, unary minus),
  numbers, scalars, array references and the intrinsics EXP, LOG, TANH; integer index and bound
  expressions use integer division.  Literals without a D exponent (4.0E00, 2.0) are default
  REAL (single precision) as in Fortran: an operation on two of them, or an intrinsic of one,
  is evaluated in float32 and widened only when it meets a REAL*8 variable (IMPLICIT REAL*8), so
  -4.0E00*LOG(2.0E00) is the single-precision product; x**2 is x*x;
* conditions of IF (...) THEN / ELSE / ENDIF: MYPEZ.EQ.0 and MYPEZ.EQ.NPEZ-1 select the faces
  (see below); other comparisons (.EQ. .NE. .GT. .LT. .GE. .LE.) of scalars are evaluated.

Each DO nest is executed as one whole-array numpy statement over the loop box.  That is exact
because no statement of the block reads the array it writes at another index (checked at run
time); the operations are IEEE double, one rounding each, in the source order, which is what a
sequential Fortran evaluation without contraction computes.  The z-edge blocks are run for both
faces of the global domain, the multi-rank case (rank 0 holds the top, rank NPEZ-1 the bottom).
Arrays are the oracle's global (NZ, NY, NX) arrays; Fortran A(I,J,K) is A[K-1, J-1, I-1].
"""
from __future__ import annotations

import math
import re
from typing import Dict, List, Tuple

import numpy as np

ARRAYS_1D = {"DXXDX": 2, "D2XXDX2": 2, "DYYDY": 1, "D2YYDY2": 1, "DZZDZ": 0, "D2ZZDZ2": 0,
             "EXX": 2, "WYY": 1, "ZEE": 0, "ROM": 0, "WWZ": 0}


def read_block(path: str, first: int = 2146, last: int = 2651) -> List[Tuple[str, str]]:
    """(label, statement) pairs of source lines first..last (1-based, inclusive)."""
    raw = open(path).read().split("\n")[first - 1:last]
    stmts: List[List[str]] = []
    for line in raw:
        if not line.strip() or line[0] in "cC*!":
            continue
        if line.startswith("\t"):
            # tab format: a tab followed by a digit 1-9 continues the statement before, any
            # other tab-led line is a statement (no label)
            if len(line) > 1 and line[1] in "123456789":
                stmts[-1][1] += line[2:].strip()
                continue
            stmts.append(["", line.strip()])
            continue
        line = line.expandtabs(8)
        if len(line) > 5 and line[:5].strip() == "" and line[5] not in " 0\t":
            stmts[-1][1] += line[6:].strip()
            continue
        m = re.match(r"^\s*(\d+)?\s*(.*)$", line.replace("\t", " "))
        stmts.append([m.group(1) or "", m.group(2).strip()])
    return [(a, b) for a, b in stmts]


# --------------------------------------------------------------------- expressions -------
_TOK = re.compile(r"\s*(?:(\d+\.\d*(?:[EeDd][+-]?\d+)?|\d+(?:[EeDd][+-]?\d+)?)|([A-Z][A-Z0-9_]*)|(\*\*|\S))")


def _tokens(s: str):
    out, pos = [], 0
    while pos < len(s):
        m = _TOK.match(s, pos)
        if not m or m.end() == pos:
            break
        pos = m.end()
        if m.group(1):
            out.append(("num", m.group(1)))
        elif m.group(2):
            out.append(("id", m.group(2)))
        else:
            out.append(("op", m.group(3)))
    return out


class _Parser:
    """Expression tree: ('num', text) ('id', name) ('ref', name, [args]) ('neg', e) (op, a, b)."""

    def __init__(self, text):
        self.t = _tokens(text)
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expr(self):
        if self.peek() == ("op", "-"):
            self.take()
            node = ("neg", self.term())
        elif self.peek() == ("op", "+"):
            self.take()
            node = self.term()
        else:
            node = self.term()
        while self.peek()[0] == "op" and self.peek()[1] in "+-":
            op = self.take()[1]
            node = (op, node, self.term())
        return node

    def term(self):
        node = self.power()
        while self.peek()[0] == "op" and self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            node = (op, node, self.power())
        return node

    def power(self):
        node = self.factor()
        if self.peek() == ("op", "**"):
            self.take()
            node = ("**", node, self.factor())
        return node

    def factor(self):
        kind, val = self.take()
        if kind == "num":
            return ("num", val)
        if kind == "id":
            if self.peek() == ("op", "("):
                self.take()
                args = [self.expr()]
                while self.peek() == ("op", ","):
                    self.take()
                    args.append(self.expr())
                assert self.take() == ("op", ")")
                return ("ref", val, args)
            return ("id", val)
        if (kind, val) == ("op", "("):
            node = self.expr()
            assert self.take() == ("op", ")")
            return node
        if (kind, val) == ("op", "-"):
            return ("neg", self.factor())
        raise ValueError(f"unexpected token {val!r}")


def parse(text: str):
    p = _Parser(text)
    node = p.expr()
    if p.i != len(p.t):
        raise ValueError(f"trailing tokens in {text!r}")
    return node


# ------------------------------------------------------------------------- evaluation -----
def _libm(f):
    """An intrinsic evaluated by the C math library element by element (math.* call libm), as a
    compiled Fortran does; numpy's vectorised exp/log may differ from libm in the last bit."""
    vec = np.vectorize(f, otypes=[np.float64])

    def call(x):
        if isinstance(x, np.ndarray):
            return vec(x)
        return f(float(x))
    return call


INTRINSICS = {"EXP": _libm(math.exp), "LOG": _libm(math.log), "TANH": _libm(math.tanh)}


def _is_r4(v) -> bool:
    """A default-REAL (single precision) value: a literal, or a result computed from them."""
    return isinstance(v, np.float32)


class Block:
    """The LMAG statements, executable on a dict of arrays and scalars."""

    def __init__(self, path: str, first: int = 2146, last: int = 2651, guard: str = "LMAG"):
        self.stmts = read_block(path, first, last)
        if not self.stmts or not re.match(r"IF\s*\(\s*" + re.escape(guard) + r"\s*\)\s*THEN",
                                          self.stmts[0][1].replace(" ", "")):
            raise ValueError(f"the block must start with IF ({guard}) THEN")

    # integer expressions (bounds, constant indices)
    def _int(self, node, env, loopvar_offsets=None):
        kind = node[0]
        if kind == "num":
            return int(node[1])
        if kind == "id":
            return int(env[node[1]])
        if kind == "neg":
            return -self._int(node[1], env)
        a, b = self._int(node[1], env), self._int(node[2], env)
        if kind == "+":
            return a + b
        if kind == "-":
            return a - b
        if kind == "*":
            return a * b
        return int(a / b)  # Fortran integer division truncates toward zero

    @staticmethod
    def _loopvar_offset(node):
        """I+c / I-c / I -> ('I', c); None if node holds no loop variable."""
        if node[0] == "id" and node[1] in ("I", "J", "K"):
            return node[1], 0
        if node[0] in "+-" and node[1][0] == "id" and node[1][1] in ("I", "J", "K") and node[2][0] == "num":
            return node[1][1], int(node[2][1]) * (1 if node[0] == "+" else -1)
        return None

    def _index(self, args, env, box):
        """numpy index (k, j, i) for A(args) over box {'I': (lo, hi), ...} (1-based)."""
        out = []
        for axis_var, arg in zip(("I", "J", "K"), args):
            lv = self._loopvar_offset(arg)
            if lv is not None:
                var, off = lv
                if var != axis_var:
                    raise ValueError("transposed index")
                lo, hi = box[var]
                out.append(slice(lo + off - 1, hi + off))
            else:
                c = self._int(arg, env)
                out.append(slice(c - 1, c))
        return (out[2], out[1], out[0])

    def _value(self, node, env, box):
        kind = node[0]
        if kind == "num":
            text = node[1]
            if "D" in text or "d" in text:  # double-precision literal
                return float(text.replace("D", "E").replace("d", "e"))
            return np.float32(text)  # default REAL
        if kind == "id":
            return env[node[1]]
        if kind == "neg":
            v = self._value(node[1], env, box)
            return np.float32(-v) if _is_r4(v) else -v
        if kind == "ref" and node[1] in INTRINSICS:
            v = self._value(node[2][0], env, box)
            f = INTRINSICS[node[1]]
            # a single-precision argument gives the single-precision result (the double result
            # rounded once: the correctly rounded float of these intrinsics)
            return np.float32(f(v)) if _is_r4(v) else f(v)
        if kind == "**":
            base, ex = self._value(node[1], env, box), node[2]
            if ex[0] != "num" or ex[1] != "2":
                raise ValueError("only x**2 is supported")
            return base * base
        if kind == "ref":
            name, args = node[1], node[2]
            arr = env[name]
            if name in ARRAYS_1D:
                axis = ARRAYS_1D[name]
                lv = self._loopvar_offset(args[0])
                if lv is None:
                    return float(arr[self._int(args[0], env) - 1])
                var, off = lv
                lo, hi = box[var]
                v = arr[lo + off - 1:hi + off]
                shape = [1, 1, 1]
                shape[axis] = v.shape[0]
                return v.reshape(shape)
            return arr[self._index(args, env, box)]
        a = self._value(node[1], env, box)
        b = self._value(node[2], env, box)
        if _is_r4(a) and _is_r4(b):  # single precision throughout
            a, b = np.float32(a), np.float32(b)
        else:  # mixed: the REAL*4 operand is widened exactly
            a = float(a) if _is_r4(a) else a
            b = float(b) if _is_r4(b) else b
        if kind == "+":
            r = a + b
        elif kind == "-":
            r = a - b
        elif kind == "*":
            r = a * b
        else:
            r = a / b
        return np.float32(r) if (_is_r4(a) and _is_r4(b)) else r

    _CMP = {"EQ": np.equal, "NE": np.not_equal, "GT": np.greater, "LT": np.less, "GE": np.greater_equal,
            "LE": np.less_equal}

    def _cond(self, cond, env, top, bottom):
        c = cond.replace(" ", "")
        if c == "MYPEZ.EQ.0":
            return top
        if c == "MYPEZ.EQ.NPEZ-1":
            return bottom
        m = re.fullmatch(r"(.+?)\.(EQ|NE|GT|LT|GE|LE)\.(.+)", c)
        if not m:
            raise ValueError(f"unsupported condition {cond}")
        a = self._value(parse(m.group(1)), env, {})
        b = self._value(parse(m.group(3)), env, {})
        return bool(self._CMP[m.group(2)](float(a), float(b)))

    @staticmethod
    def _refs(node, name):
        if node[0] == "ref":
            hits = [node[2]] if node[1] == name else []
            for a in node[2]:
                hits += Block._refs(a, name)
            return hits
        if node[0] in ("num", "id"):
            return []
        if node[0] == "neg":
            return Block._refs(node[1], name)
        return Block._refs(node[1], name) + Block._refs(node[2], name)

    def _assign(self, stmt, env, box):
        lhs, rhs = stmt.split("=", 1)
        lt, rt = parse(lhs), parse(rhs)
        if lt[0] == "id":  # scalar (IMPLICIT REAL*8: a REAL*4 value is widened on assignment)
            v = self._value(rt, env, box)
            env[lt[1]] = float(v) if _is_r4(v) else v
            return
        name, args = lt[1], lt[2]
        for other in self._refs(rt, name):
            if other != args:
                raise ValueError(f"{name} read at another index than it is written: not vectorisable")
        env[name][self._index(args, env, box)] = self._value(rt, env, box)

    def run(self, env: Dict[str, object], top: bool = True, bottom: bool = True):
        """Execute the block in env (arrays are modified in place)."""
        stmts = self.stmts[1:]
        # the block's closing ENDIF is the last statement
        if stmts and re.fullmatch(r"END\s*IF", stmts[-1][1]):
            stmts = stmts[:-1]
        loops: List[Tuple[str, str, int, int]] = []
        body: List[str] = []
        cond_stack: List[bool] = []
        taken: List[bool] = []  # an earlier branch of the IF at this depth was taken
        for label, st in stmts:
            m = re.fullmatch(r"DO\s*(\d+)\s*([IJK])\s*=\s*(.+?)\s*,\s*(.+)", st)
            if m:
                loops.append((m.group(1), m.group(2), self._int(parse(m.group(3)), env),
                              self._int(parse(m.group(4)), env)))
                continue
            m = re.fullmatch(r"(ELSE\s*)?IF\s*\((.*)\)\s*THEN", st)
            if m:
                cond = m.group(2).replace(" ", "")
                active = self._cond(cond, env, top, bottom)
                if m.group(1):
                    if cond.startswith("MYPEZ"):
                        cond_stack[-1] = active  # separate ranks: the two faces are independent
                    else:
                        taken[-1] = taken[-1] or cond_stack[-1]
                        cond_stack[-1] = active and not taken[-1]
                else:
                    cond_stack.append(active)
                    taken.append(False)
                continue
            if st == "ELSE":
                taken[-1] = taken[-1] or cond_stack[-1]
                cond_stack[-1] = not taken[-1]
                continue
            if re.fullmatch(r"END\s*IF", st):
                cond_stack.pop()
                taken.pop()
                continue
            if st == "CONTINUE":
                if not loops or loops[-1][0] != label:
                    raise ValueError(f"CONTINUE {label} closes no DO")
                nest = [lp for lp in loops if lp[0] == label]
                loops = [lp for lp in loops if lp[0] != label]
                if all(cond_stack):
                    box = {var: (lo, hi) for _, var, lo, hi in nest}
                    for b in body:
                        self._assign(b, env, box)
                body = []
                continue
            if loops:
                body.append(st)
            elif all(cond_stack):
                self._assign(st, env, {})
        if loops or cond_stack:
            raise ValueError("unbalanced DO / IF")
        return env


def lmag_inputs(o_mhd, o_hydro):
    """The LMAG block's inputs for the state held by o_mhd: FU..FT, UU, VV, WW and RO (= 1/rho)
    from the hydro part of FLUXES, run by o_hydro (an oracle holding the same state with B = 0;
    the hydro part does not read B), B from o_mhd, metric lines and constants."""
    env = {}
    for n in ("fu", "fv", "fw", "ft", "uu", "vv", "ww", "ro"):
        env[n.upper()] = o_hydro.field(n).copy()
    for n in ("bx", "by", "bz"):
        env[n.upper()] = o_mhd.field(n).copy()
    for n in ("RU", "RV", "RW", "TT", "WW1", "WW2", "WW3"):
        env[n] = np.zeros_like(env["FU"])
    for n in ("dxxdx", "d2xxdx2", "dyydy", "d2yydy2", "dzzdz", "d2zzdz2"):
        env[n.upper()] = np.array(o_mhd.line(n))
    for n in ("hx", "h2x", "hy", "h2y", "hz", "h2z", "obeta", "orm", "ocv"):
        env[n.upper()] = o_mhd.param(n)
    env.update(ILAP=2, IX=2, IY=2, NX=o_mhd.NX, NY=o_mhd.NY, NZ=o_mhd.NZ, MYPEZ=0, NPEZ=2)
    return env
