"""A small WGSL interpreter for the subset used by the reference's
simulation shaders (src/shaders/{common,stats,vel,tmpl_comp,tmpl_scalar,
advect,fluid,combust,mg}.wgsl).

It lets the golden-vector generator (make_golden.py, run in a container that
has the reference checkout) execute the reference's own kernel source on
small grids, so that the C++ oracle and the CUDA kernels are pinned to the
reference's code rather than to a restatement of it.

Semantics: f32 values are numpy float32 scalars or arrays (every operation
rounds to single precision, no fused multiply-add), i32/u32 are numpy int32 /
uint32 (wrapping), abstract integer literals are Python ints, booleans are
Python bools.  Builtins follow the WGSL specification formulas:
mix(a,b,t) = a*(1-t) + b*t, smoothstep(e0,e1,x) = t*t*(3-2t) with
t = clamp((x-e0)/(e1-e0), 0, 1), clamp(x,lo,hi) = min(max(x,lo),hi),
length(v) = sqrt(sum of squares, left to right), select(f,t,c) = c ? t : f.
exp() is numpy's float32 exp (within a few ulp of any GPU's).

Workgroup reductions: every invocation runs with local_invocation_index 0
and the 64-lane tree reductions wsum/wmax (stats.wgsl:15-36) return the
invocation's own value, so each invocation adds (or maxes) its own
contribution into the statistics atomics.  Totals are the same sums in a
different order (the reference's float atomics have no fixed order either).
"""
from __future__ import annotations

import math
import re
import warnings
from typing import Any, Callable, Dict, List, Optional

import numpy as np

warnings.filterwarnings("ignore", category=RuntimeWarning)

F32 = np.float32
I32 = np.int32
U32 = np.uint32

# ---------------------------------------------------------------- tokenizer
_TOKEN = re.compile(r"""
    (?P<ws>\s+|//[^\n]*|/\*.*?\*/)
  | (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[uif]?|0[xX][0-9a-fA-F]+u?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>->|\+\+|--|<<=|>>=|<<|>>|<=|>=|==|!=|&&|\|\||\+=|-=|\*=|/=|%=|&=|\|=|\^=|[-+*/%<>=!&|^~(){}\[\];,.:@])
""", re.S | re.X)


def tokenize(src: str):
    toks = []
    pos = 0
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise SyntaxError(f"bad character at {src[pos:pos + 30]!r}")
        pos = m.end()
        if m.lastgroup == "ws":
            continue
        toks.append((m.lastgroup, m.group(m.lastgroup)))
    toks.append(("eof", ""))
    return toks


# ------------------------------------------------------------------- parser
class Parser:
    """Recursive-descent parser producing tuples (kind, ...)."""

    def __init__(self, src: str):
        self.t = tokenize(src)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def accept(self, v):
        if self.t[self.i][1] == v:
            self.i += 1
            return True
        return False

    def expect(self, v):
        tok = self.next()
        if tok[1] != v:
            raise SyntaxError(f"expected {v!r}, got {tok[1]!r} near token {self.i}")
        return tok

    def ident(self):
        tok = self.next()
        if tok[0] != "id":
            raise SyntaxError(f"expected identifier, got {tok[1]!r}")
        return tok[1]

    def attrs(self):
        out = []
        while self.peek()[1] == "@":
            self.next()
            name = self.ident()
            args = []
            if self.accept("("):
                while not self.accept(")"):
                    args.append(self.expr())
                    self.accept(",")
            out.append((name, args))
        return out

    def _split_shift(self):
        """Inside a template list '>>' closes two lists."""
        if self.peek()[1] == ">>":
            self.t[self.i] = ("op", ">")
            self.t.insert(self.i + 1, ("op", ">"))

    def type_(self):
        name = self.ident()
        params = []
        if self.peek()[1] == "<":
            self.next()
            while True:
                if self.peek()[0] == "num":
                    params.append(("num", self.next()[1]))
                else:
                    params.append(self.type_())
                self._split_shift()
                if self.accept(">"):
                    break
                self.expect(",")
        return ("type", name, params)

    def module(self):
        decls = []
        while self.peek()[0] != "eof":
            at = self.attrs()
            kw = self.peek()[1]
            if kw == "struct":
                self.next()
                name = self.ident()
                self.expect("{")
                members = []
                while not self.accept("}"):
                    self.attrs()
                    mn = self.ident()
                    self.expect(":")
                    members.append((mn, self.type_()))
                    self.accept(",")
                self.accept(";")
                decls.append(("struct", name, members))
            elif kw == "var":
                self.next()
                space = None
                if self.accept("<"):
                    space = self.ident()
                    if self.accept(","):
                        self.ident()
                    self.expect(">")
                name = self.ident()
                ty = None
                if self.accept(":"):
                    ty = self.type_()
                init = None
                if self.accept("="):
                    init = self.expr()
                self.expect(";")
                decls.append(("gvar", name, space, ty, init, at))
            elif kw in ("const", "override"):
                self.next()
                name = self.ident()
                ty = None
                if self.accept(":"):
                    ty = self.type_()
                init = None
                if self.accept("="):
                    init = self.expr()
                self.expect(";")
                decls.append((kw, name, ty, init))
            elif kw == "fn":
                self.next()
                name = self.ident()
                self.expect("(")
                params = []
                while not self.accept(")"):
                    pat = self.attrs()
                    pn = self.ident()
                    self.expect(":")
                    params.append((pn, self.type_(), pat))
                    self.accept(",")
                ret = None
                if self.accept("->"):
                    self.attrs()
                    ret = self.type_()
                body = self.block()
                decls.append(("fn", name, params, ret, body, at))
            else:
                raise SyntaxError(f"unexpected {kw!r} at module scope")
        return decls

    def block(self):
        self.expect("{")
        stmts = []
        while not self.accept("}"):
            stmts.append(self.stmt())
        return ("block", stmts)

    def stmt(self):
        kw = self.peek()[1]
        if kw == "{":
            return self.block()
        if kw in ("let", "var", "const"):
            self.next()
            name = self.ident()
            ty = None
            if self.accept(":"):
                ty = self.type_()
            init = None
            if self.accept("="):
                init = self.expr()
            self.expect(";")
            return ("decl", kw, name, ty, init)
        if kw == "if":
            self.next()
            cond = self.expr()
            then = self.block()
            els = None
            if self.accept("else"):
                if self.peek()[1] == "if":
                    els = ("block", [self.stmt()])
                else:
                    els = self.block()
            return ("if", cond, then, els)
        if kw == "for":
            self.next()
            self.expect("(")
            init = None if self.peek()[1] == ";" else self.simple_stmt()
            self.expect(";")
            cond = None if self.peek()[1] == ";" else self.expr()
            self.expect(";")
            upd = None if self.peek()[1] == ")" else self.simple_stmt(no_semi=True)
            self.expect(")")
            body = self.block()
            return ("for", init, cond, upd, body)
        if kw == "loop":
            self.next()
            return ("loop", self.block())
        if kw == "break":
            self.next()
            self.expect(";")
            return ("break",)
        if kw == "continue":
            self.next()
            self.expect(";")
            return ("continue",)
        if kw == "return":
            self.next()
            val = None if self.peek()[1] == ";" else self.expr()
            self.expect(";")
            return ("return", val)
        s = self.simple_stmt()
        self.expect(";")
        return s

    def simple_stmt(self, no_semi=False):
        kw = self.peek()[1]
        if kw in ("var", "let"):
            self.next()
            name = self.ident()
            ty = None
            if self.accept(":"):
                ty = self.type_()
            init = None
            if self.accept("="):
                init = self.expr()
            return ("decl", kw, name, ty, init)
        lhs = self.expr()
        op = self.peek()[1]
        if op in ("=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>="):
            self.next()
            rhs = self.expr()
            return ("assign", op, lhs, rhs)
        if op in ("++", "--"):
            self.next()
            return ("assign", "+=" if op == "++" else "-=", lhs, ("lit", 1))
        return ("exprstmt", lhs)

    # ----- expressions (precedence climbing)
    BIN = [["||"], ["&&"], ["|"], ["^"], ["&"], ["==", "!="], ["<", ">", "<=", ">="],
           ["<<", ">>"], ["+", "-"], ["*", "/", "%"]]

    def expr(self, level=0):
        if level == len(self.BIN):
            return self.unary()
        lhs = self.expr(level + 1)
        while self.peek()[1] in self.BIN[level]:
            # a '<' that opens a template list never reaches here
            op = self.next()[1]
            rhs = self.expr(level + 1)
            lhs = ("bin", op, lhs, rhs)
        return lhs

    def unary(self):
        op = self.peek()[1]
        if op in ("-", "!", "~"):
            self.next()
            return ("un", op, self.unary())
        if op == "&":
            self.next()
            return ("addr", self.unary())
        if op == "*":
            self.next()
            return ("deref", self.unary())
        return self.postfix(self.primary())

    def postfix(self, e):
        while True:
            if self.accept("."):
                e = ("member", e, self.ident())
            elif self.accept("["):
                idx = self.expr()
                self.expect("]")
                e = ("index", e, idx)
            else:
                return e

    def primary(self):
        kind, v = self.peek()
        if kind == "num":
            self.next()
            return ("lit", _literal(v))
        if v == "(":
            self.next()
            e = self.expr()
            self.expect(")")
            return e
        if kind == "id":
            self.next()
            if v in ("true", "false"):
                return ("lit", v == "true")
            targs = None
            if self.peek()[1] == "<" and v in ("array", "vec2", "vec3", "vec4", "bitcast"):
                self.next()
                targs = []
                while True:
                    if self.peek()[0] == "num":
                        targs.append(("num", self.next()[1]))
                    else:
                        targs.append(self.type_())
                    if self.accept(">"):
                        break
                    self.expect(",")
            if self.accept("("):
                args = []
                while not self.accept(")"):
                    args.append(self.expr())
                    self.accept(",")
                return ("call", v, targs, args)
            return ("id", v)
        raise SyntaxError(f"unexpected token {v!r}")


def _literal(s: str):
    if s.startswith(("0x", "0X")):
        u = s.endswith("u")
        n = int(s.rstrip("u"), 16)
        return U32(n) if u else n
    if s.endswith("u"):
        return U32(int(s[:-1]))
    if s.endswith("i"):
        return I32(int(s[:-1]))
    if s.endswith("f"):
        return F32(float(s[:-1]))
    if any(c in s for c in ".eE"):
        return F32(float(s))
    return int(s)


# ---------------------------------------------------------------- runtime
class Ref:
    """Pointer to an element of a storage array (for atomics)."""
    __slots__ = ("arr", "idx")

    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = idx


class Signal:
    __slots__ = ("kind", "value")

    def __init__(self, kind, value=None):
        self.kind = kind
        self.value = value


BREAK = Signal("break")
CONTINUE = Signal("continue")


def _concrete(v):
    """Concretize an abstract int for a let/var binding."""
    if type(v) is int:
        return I32(v)
    if isinstance(v, np.ndarray):
        return v.copy()
    if isinstance(v, dict):
        return {k: _concrete(x) for k, x in v.items()}
    if isinstance(v, list):
        return [_concrete(x) for x in v]
    return v


def _scalar_kind(t):
    return {"f32": F32, "i32": I32, "u32": U32, "bool": bool}.get(t)


def _vec_info(name, targs):
    if name in ("vec2f", "vec3f", "vec4f"):
        return int(name[3]), F32
    if name in ("vec2i", "vec3i", "vec4i"):
        return int(name[3]), I32
    if name in ("vec2u", "vec3u", "vec4u"):
        return int(name[3]), U32
    if name in ("vec2", "vec3", "vec4"):
        dt = _scalar_kind(targs[0][1]) if targs else None
        return int(name[3]), dt
    return None


def _convert(v, dt):
    if dt is None:
        return v
    if isinstance(v, np.ndarray):
        if dt is F32:
            return v.astype(np.float32)
        if v.dtype.kind == "f":
            return np.trunc(v).astype(np.int64).astype(dt)
        return v.astype(np.int64).astype(dt) if dt is not bool else v.astype(bool)
    if dt is F32:
        return F32(v)
    if dt is bool:
        return bool(v)
    if isinstance(v, (float, np.floating)):
        f = float(v)
        if dt is U32:
            return U32(min(max(math.trunc(f), 0), 0xFFFFFFFF))
        return I32(min(max(math.trunc(f), -2 ** 31), 2 ** 31 - 1))
    return dt(int(v) & 0xFFFFFFFF) if dt is U32 else I32(((int(v) + 2 ** 31) % 2 ** 32) - 2 ** 31)


SWZ = {"x": 0, "y": 1, "z": 2, "w": 3, "r": 0, "g": 1, "b": 2, "a": 3}


def _mix(a, b, t):
    one = F32(1.0)
    return a * (one - t) + b * t


def _clamp(e, lo, hi):
    return np.minimum(np.maximum(e, lo), hi)


def _smoothstep(e0, e1, x):
    t = _clamp((x - e0) / (e1 - e0), F32(0.0), F32(1.0))
    return t * t * (F32(3.0) - F32(2.0) * t)


def _length(v):
    if isinstance(v, np.ndarray):
        s = v[0] * v[0]
        for k in range(1, len(v)):
            s = s + v[k] * v[k]
        return np.sqrt(s)
    return np.abs(v)


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]], dtype=np.float32)


def _select(f, t, c):
    if isinstance(c, np.ndarray):
        return np.where(c, t, f).astype(np.asarray(t).dtype)
    return t if c else f


def _minmax(fn):
    def g(a, b):
        r = fn(a, b)
        if type(a) is int and type(b) is int:
            return int(r)
        return r
    return g


def _bitcast(targs, v):
    name = targs[0][1]
    if name == "f32":
        return np.array([v], dtype=np.uint32).view(np.float32)[0]
    if name == "u32":
        return np.array([v], dtype=np.float32).view(np.uint32)[0]
    raise NotImplementedError(name)


def _atomic_load(r):
    return U32(r.arr[r.idx])


def _atomic_cas(r, old, new):
    cur = U32(r.arr[r.idx])
    ok = cur == old
    if ok:
        r.arr[r.idx] = new
    return {"old_value": cur, "exchanged": bool(ok)}


def _atomic_max(r, v):
    cur = U32(r.arr[r.idx])
    r.arr[r.idx] = max(cur, U32(v))
    return cur


def _texture_store(tex, c, v):
    """textureStore on a 3D storage texture bound as an (nz, ny, nx, 4)
    array: the texel keeps the texture's precision (an rgba16float array
    holds binary16, converted with round to nearest even); stores outside
    the texture are discarded."""
    x, y, z = int(c[0]), int(c[1]), int(c[2])
    if 0 <= z < tex.shape[0] and 0 <= y < tex.shape[1] and 0 <= x < tex.shape[2]:
        tex[z, y, x] = np.asarray(v, dtype=F32).astype(tex.dtype)


def _dot(a, b):
    """Sum of the products in component order, each step rounded to f32
    (no fused multiply-add)."""
    a = np.asarray(a, dtype=F32)
    b = np.asarray(b, dtype=F32)
    r = F32(a[0] * b[0])
    for k in range(1, len(a)):
        r = F32(r + F32(a[k] * b[k]))
    return r


def _f32_unary(fn, x):
    """An f32 builtin on a scalar (kept a scalar) or a vector."""
    if isinstance(x, np.ndarray):
        return fn(x.astype(F32))
    return F32(fn(F32(x)))


class Mat3:
    """mat3x3<f32> as its three column vectors.  matrix * vector is
    c0 * v.x + c1 * v.y + c2 * v.z, summed in that order in f32."""

    def __init__(self, cols):
        self.c = [np.asarray(c, dtype=F32) for c in cols]

    def __mul__(self, v):
        v = np.asarray(v, dtype=F32)
        return (self.c[0] * v[0] + self.c[1] * v[1]) + self.c[2] * v[2]


def _normalize(v):
    v = np.asarray(v, dtype=F32)
    return v / _length(v)


def _texture_dimensions(tex, *level):
    """A 3D texture bound as an (nz, ny, nx, 4) array: vec3u(nx, ny, nz)."""
    return np.array([tex.shape[2], tex.shape[1], tex.shape[0]], dtype=U32)


def _texture_sample_level(tex, samp, uv, level):
    """textureSampleLevel with the renderer's sampler (linear filtering,
    clamp-to-edge addressing; src/render.rs:121-125), modelled exactly in
    f32: per axis p = u * n - 0.5, texels floor(p) and floor(p) + 1 clamped
    to the texture, weight p - floor(p); mixes along x, then y, then z."""
    uv = np.asarray(uv, dtype=F32)

    def ax(u, n):
        p = F32(F32(u) * F32(n)) - F32(0.5)
        f0 = np.floor(p)
        w = F32(p - f0)
        i0 = int(f0)
        return min(max(i0, 0), n - 1), min(max(i0 + 1, 0), n - 1), w

    nz, ny, nx = tex.shape[0], tex.shape[1], tex.shape[2]
    x0, x1, fx = ax(uv[0], nx)
    y0, y1, fy = ax(uv[1], ny)
    z0, z1, fz = ax(uv[2], nz)

    def t(z, y, x):
        return tex[z, y, x].astype(F32)

    def mix(a, b, w):
        return a * (F32(1.0) - w) + b * w
    c00 = mix(t(z0, y0, x0), t(z0, y0, x1), fx)
    c10 = mix(t(z0, y1, x0), t(z0, y1, x1), fx)
    c01 = mix(t(z1, y0, x0), t(z1, y0, x1), fx)
    c11 = mix(t(z1, y1, x0), t(z1, y1, x1), fx)
    return mix(mix(c00, c10, fy), mix(c01, c11, fy), fz)


def _texture_load(tex, c, level):
    """textureLoad of one texel of a 3D texture, as vec4<f32>."""
    return tex[int(c[2]), int(c[1]), int(c[0])].astype(F32)


BUILTINS: Dict[str, Callable] = {
    "textureStore": _texture_store, "textureLoad": _texture_load, "dot": _dot,
    "textureDimensions": _texture_dimensions, "textureSampleLevel": _texture_sample_level,
    "normalize": _normalize, "cos": lambda x: _f32_unary(np.cos, x),
    "sin": lambda x: _f32_unary(np.sin, x), "round": lambda x: _f32_unary(np.round, x),
    "clamp": _clamp, "min": _minmax(np.minimum), "max": _minmax(np.maximum), "mix": _mix,
    "smoothstep": _smoothstep, "select": _select, "exp": np.exp, "sqrt": np.sqrt,
    "length": _length, "cross": _cross, "floor": np.floor, "abs": np.abs,
    "all": lambda v: bool(np.all(v)), "any": lambda v: bool(np.any(v)),
    "atomicLoad": _atomic_load, "atomicCompareExchangeWeak": _atomic_cas,
    "atomicMax": _atomic_max, "workgroupBarrier": lambda: None,
}


class Module:
    """One assembled kernel: parsed declarations, globals and functions."""

    def __init__(self, src: str, overrides: Optional[Dict[str, Any]] = None,
                 replace: Optional[Dict[str, Callable]] = None):
        self.decls = Parser(src).module()
        self.structs = {}
        self.globals: Dict[str, Any] = {}
        self.bindings: Dict[int, str] = {}
        self.funcs: Dict[str, Callable] = {}
        self.fn_decls = {}
        self.replace = replace or {}
        overrides = overrides or {}
        for d in self.decls:
            if d[0] == "struct":
                self.structs[d[1]] = d[2]
            elif d[0] == "fn":
                self.fn_decls[d[1]] = d
        for d in self.decls:
            if d[0] in ("const", "override"):
                _, name, ty, init = d
                if name in overrides:
                    v = overrides[name]
                else:
                    v = self._eval_const(init)
                if ty is not None:
                    v = self._coerce(v, ty)
                self.globals[name] = _concrete(v)
            elif d[0] == "gvar":
                _, name, space, ty, init, at = d
                for a, args in at:
                    if a == "binding":
                        self.bindings[int(self._eval_const(args[0]))] = name
                if init is not None:
                    self.globals[name] = _concrete(self._eval_const(init))
                elif space == "workgroup" or space == "private":
                    self.globals[name] = self._zero(ty)
                else:
                    self.globals[name] = None
        for name, d in self.fn_decls.items():
            self.funcs[name] = self._compile_fn(d)
        for name, f in self.replace.items():
            self.funcs[name] = f

    # ----- helpers
    def _eval_const(self, e):
        f = self._expr(e, {})
        return f({})

    def _zero(self, ty):
        name, params = ty[1], ty[2]
        if name == "array":
            n = int(params[1][1])
            return [self._zero(params[0]) for _ in range(n)]
        vi = _vec_info(name, params)
        if vi:
            return np.zeros(vi[0], dtype=vi[1] if vi[1] is not bool else bool)
        if name in self.structs:
            return {m: self._zero(t) for m, t in self.structs[name]}
        k = _scalar_kind(name)
        return k(0) if k is not bool else False

    def _coerce(self, v, ty):
        name = ty[1]
        k = _scalar_kind(name)
        if k is not None and not isinstance(v, np.ndarray):
            return _convert(v, k)
        vi = _vec_info(name, ty[2])
        if vi and isinstance(v, np.ndarray):
            return _convert(v, vi[1])
        return v

    # ----- compilation to closures
    def _compile_fn(self, d):
        _, name, params, ret, body, at = d
        pnames = [p[0] for p in params]
        ptypes = [p[1] for p in params]
        run = self._stmt(body, set(pnames))
        coerce = self._coerce

        def fn(*args):
            fr = {}
            for n, t, a in zip(pnames, ptypes, args):
                fr[n] = coerce(a, t)
            s = run(fr)
            if s is not None and s.kind == "return":
                return s.value
            return None
        return fn

    def _stmt(self, s, scope):
        k = s[0]
        if k == "block":
            inner = set(scope)
            parts = [self._stmt(x, inner) for x in s[1]]

            def run(fr):
                for p in parts:
                    r = p(fr)
                    if r is not None:
                        return r
                return None
            return run
        if k == "decl":
            _, kw, name, ty, init = s
            scope.add(name)
            if init is None:
                z = self._zero(ty)

                def run(fr, z=z):
                    fr[name] = _concrete(z)
                return run
            f = self._expr(init, scope)
            co = self._coerce

            def run(fr):
                v = _concrete(f(fr))
                if ty is not None:
                    v = co(v, ty)
                fr[name] = v
            return run
        if k == "assign":
            return self._assign(s, scope)
        if k == "exprstmt":
            f = self._expr(s[1], scope)

            def run(fr):
                f(fr)
            return run
        if k == "if":
            c = self._expr(s[1], scope)
            t = self._stmt(s[2], scope)
            e = self._stmt(s[3], scope) if s[3] is not None else None

            def run(fr):
                if c(fr):
                    return t(fr)
                if e is not None:
                    return e(fr)
                return None
            return run
        if k == "for":
            inner = set(scope)
            init = self._stmt(s[1], inner) if s[1] else None
            cond = self._expr(s[2], inner) if s[2] else None
            upd = self._stmt(s[3], inner) if s[3] else None
            body = self._stmt(s[4], inner)

            def run(fr):
                if init:
                    init(fr)
                while cond is None or cond(fr):
                    r = body(fr)
                    if r is not None:
                        if r is BREAK:
                            break
                        if r is not CONTINUE:
                            return r
                    if upd:
                        upd(fr)
                return None
            return run
        if k == "loop":
            body = self._stmt(s[1], scope)

            def run(fr):
                while True:
                    r = body(fr)
                    if r is not None:
                        if r is BREAK:
                            return None
                        if r is not CONTINUE:
                            return r
            return run
        if k == "break":
            return lambda fr: BREAK
        if k == "continue":
            return lambda fr: CONTINUE
        if k == "return":
            if s[1] is None:
                return lambda fr: Signal("return", None)
            f = self._expr(s[1], scope)
            return lambda fr: Signal("return", f(fr))
        raise NotImplementedError(k)

    def _assign(self, s, scope):
        _, op, lhs, rhs = s
        r = self._expr(rhs, scope)
        binop = None if op == "=" else _BINOPS[op[:-1]]
        if lhs[0] == "id":
            name = lhs[1]
            local = name in scope
            g = self.globals

            def run(fr):
                v = r(fr)
                tgt = fr if local else g
                if binop is not None:
                    v = binop(tgt[name], v)
                old = tgt[name]
                if isinstance(old, np.ndarray) and isinstance(v, np.ndarray):
                    v = v.astype(old.dtype)
                elif isinstance(old, np.generic) and not isinstance(v, np.ndarray):
                    v = type(old)(v)
                tgt[name] = v
            return run
        if lhs[0] in ("member", "index"):
            base = self._lvalue_base(lhs[1], scope)
            if lhs[0] == "member":
                key_f = None
                mname = lhs[2]
            else:
                key_f = self._expr(lhs[2], scope)
                mname = None

            def run(fr):
                container = base(fr)
                v = r(fr)
                if mname is not None:
                    if isinstance(container, dict):
                        if binop is not None:
                            v = binop(container[mname], v)
                        container[mname] = _concrete(v)
                        return
                    idx = SWZ[mname]
                else:
                    idx = int(key_f(fr))
                if binop is not None:
                    v = binop(container[idx], v)
                if isinstance(container, np.ndarray):
                    container[idx] = v
                else:
                    old = container[idx]
                    if isinstance(old, np.generic) and not isinstance(v, np.ndarray):
                        v = type(old)(v)
                    container[idx] = _concrete(v)
            return run
        raise NotImplementedError(lhs[0])

    def _lvalue_base(self, e, scope):
        """Closure returning the mutable container an lvalue lives in."""
        if e[0] == "id":
            name = e[1]
            if name in scope:
                return lambda fr: fr[name]
            g = self.globals
            return lambda fr: g[name]
        if e[0] == "member":
            b = self._lvalue_base(e[1], scope)
            m = e[2]
            return lambda fr: b(fr)[m]
        if e[0] == "index":
            b = self._lvalue_base(e[1], scope)
            i = self._expr(e[2], scope)
            return lambda fr: b(fr)[int(i(fr))]
        raise NotImplementedError(e[0])

    def _expr(self, e, scope):
        k = e[0]
        if k == "lit":
            v = e[1]
            return lambda fr: v
        if k == "id":
            name = e[1]
            if name in scope:
                return lambda fr: fr[name]
            g = self.globals
            return lambda fr: g[name]
        if k == "bin":
            op = e[1]
            a = self._expr(e[2], scope)
            b = self._expr(e[3], scope)
            if op == "&&":
                return lambda fr: bool(a(fr)) and bool(b(fr))
            if op == "||":
                return lambda fr: bool(a(fr)) or bool(b(fr))
            f = _BINOPS[op]
            return lambda fr: f(a(fr), b(fr))
        if k == "un":
            a = self._expr(e[2], scope)
            if e[1] == "-":
                return lambda fr: -a(fr)
            if e[1] == "!":
                return lambda fr: not a(fr)
            return lambda fr: ~a(fr)
        if k == "addr":
            inner = e[1]
            assert inner[0] == "index"
            base = self._expr(inner[1], scope)
            idx = self._expr(inner[2], scope)
            return lambda fr: Ref(base(fr), int(idx(fr)))
        if k == "member":
            b = self._expr(e[1], scope)
            m = e[2]
            if m in ("old_value", "exchanged") or not all(c in SWZ for c in m):
                return lambda fr: b(fr)[m]
            if len(m) == 1:
                ix = SWZ[m]

                def get1(fr):
                    v = b(fr)
                    if isinstance(v, dict):
                        return v[m]
                    return v[ix]
                return get1
            ixs = [SWZ[c] for c in m]

            def getn(fr):
                v = b(fr)
                if isinstance(v, dict):
                    return v[m]
                return v[ixs].copy()
            return getn
        if k == "index":
            b = self._expr(e[1], scope)
            i = self._expr(e[2], scope)

            def get(fr):
                v = b(fr)[int(i(fr))]
                if isinstance(v, np.ndarray):
                    return v.copy()
                return v
            return get
        if k == "call":
            return self._call(e, scope)
        raise NotImplementedError(k)

    def _call(self, e, scope):
        _, name, targs, args = e
        fs = [self._expr(a, scope) for a in args]
        vi = _vec_info(name, targs)
        if vi is not None:
            n, dt = vi

            def ctor(fr):
                vals = [f(fr) for f in fs]
                if len(vals) == 1 and not isinstance(vals[0], np.ndarray):
                    x = vals[0]
                    d = dt or (F32 if isinstance(x, (np.floating, float)) else I32)
                    return np.full(n, x, dtype=d if d is not bool else bool)
                if len(vals) == 1 and isinstance(vals[0], np.ndarray):
                    return _convert(vals[0], dt) if dt else vals[0].copy()
                flat = []
                for x in vals:
                    if isinstance(x, np.ndarray):
                        flat.extend(list(x))
                    else:
                        flat.append(x)
                d = dt or (F32 if any(isinstance(x, np.floating) for x in flat) else I32)
                return np.array([_convert(x, d) for x in flat], dtype=d)
            return ctor
        if name in ("mat3x3f", "mat3x3"):
            return lambda fr: Mat3([f(fr) for f in fs])
        if name in ("f32", "i32", "u32", "bool"):
            dt = _scalar_kind(name)
            return lambda fr: _convert(fs[0](fr), dt)
        if name == "array":
            elem = targs[0] if targs else None

            def arr(fr):
                vals = [_concrete(f(fr)) for f in fs]
                if elem is not None:
                    vals = [self._coerce(v, elem) for v in vals]
                return vals
            return arr
        if name == "bitcast":
            return lambda fr: _bitcast(targs, fs[0](fr))
        if name in self.structs:
            members = [m for m, _ in self.structs[name]]
            return lambda fr: {m: _concrete(f(fr)) for m, f in zip(members, fs)}
        if name in BUILTINS and name not in self.fn_decls and name not in self.replace:
            bf = BUILTINS[name]
            if len(fs) == 1:
                f0 = fs[0]
                return lambda fr: bf(f0(fr))
            return lambda fr: bf(*[f(fr) for f in fs])
        funcs = self.funcs

        def callf(fr):
            return funcs[name](*[f(fr) for f in fs])
        return callf

    # ----- dispatch
    def bind(self, binding: int, value):
        self.globals[self.bindings[binding]] = value

    def dispatch(self, groups, wg=(4, 4, 4), entry="main"):
        """Run every invocation of the grid in order (gid x fastest)."""
        fn = self.funcs[entry]
        params = self.fn_decls[entry][2]
        want = []
        for pn, ty, at in params:
            b = [args for a, args in at if a == "builtin"]
            want.append(b[0][0][1] if b else None)
        nx, ny, nz = groups[0] * wg[0], groups[1] * wg[1], groups[2] * wg[2]
        for z in range(nz):
            for y in range(ny):
                for x in range(nx):
                    gid = np.array([x, y, z], dtype=np.uint32)
                    args = []
                    for w in want:
                        if w == "global_invocation_id":
                            args.append(gid)
                        elif w == "local_invocation_index":
                            args.append(U32(0))
                        else:
                            raise NotImplementedError(w)
                    fn(*args)


def _shr(a, b):
    return a >> b


def _div(a, b):
    if type(a) is int and type(b) is int:
        return int(a / b)
    rt = np.result_type(a, b)
    if np.issubdtype(rt, np.integer):  # WGSL integer division truncates toward zero
        return np.trunc(np.true_divide(a, b)).astype(rt)
    return a / b


_BINOPS = {
    "+": lambda a, b: a + b, "-": lambda a, b: a - b, "*": lambda a, b: a * b, "/": _div,
    "%": lambda a, b: np.fmod(a, b), "&": lambda a, b: a & b, "|": lambda a, b: a | b,
    "^": lambda a, b: a ^ b, "<<": lambda a, b: a << b, ">>": _shr,
    "==": lambda a, b: a == b, "!=": lambda a, b: a != b, "<": lambda a, b: a < b,
    ">": lambda a, b: a > b, "<=": lambda a, b: a <= b, ">=": lambda a, b: a >= b,
}
