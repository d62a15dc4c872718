"""Stand-in for the parts of Taichi (``ti``) and ``taichi.math`` (``tm``) that
the reference renderer's hot-path code uses -- TEST INFRASTRUCTURE ONLY.

It lets the reference's own ``@ti.func`` functions, ``@ti.dataclass`` records
and the ``cast_rays`` / ``update_camera`` kernels of ``main.py`` (lifted
unmodified from the file's syntax tree by ``make_estimator_ref.py``) run in
plain Python, so that fixtures of what the reference computes can be written
without Taichi (which is not installable offline).

Arithmetic model (``ti.init(default_fp=ti.f32)``, as ``main.py:9`` sets it):

* every float is an ``np.float32`` and every operation rounds once (IEEE
  round-to-nearest), which is what NumPy 2 does for float32 scalars combined
  with Python numbers (Python literals and module constants are "weak" and
  take the float32 type, as Taichi casts constants to ``default_fp``);
* ``ti.i32`` values are :class:`I32`, an ``int`` whose arithmetic with a
  float yields float32 (Taichi promotes i32 op f32 to f32; a plain Python int
  would promote to float64), and ``/`` between integers is float division;
* ``x ** n`` with a constant integer exponent is exponentiation by squaring
  (Taichi lowers integer powers to multiplications); the lifting pass rewrites
  ``**`` into :func:`ti_pow`;
* ``tm.min`` / ``tm.max`` are the NaN-ignoring ``minnum`` / ``maxnum`` that
  Taichi's LLVM backends emit for floats;
* ``tm.normalize(v) = v / v.norm()``, ``v.norm() = sqrt(x*x + y*y + z*z)``
  (left to right), ``tm.dot`` sums left to right, ``tm.reflect`` /
  ``tm.refract`` follow GLSL (``refract`` returns the zero vector on total
  internal reflection);
* transcendental functions are NumPy's float32 ones (Taichi's fast-math
  device intrinsics cannot be reproduced; they differ in the last bits).

Random numbers: ``ti.random()`` returns the next draw of :data:`RNG`, which
either replays a given list of draws or generates the Philox-4x32-10 stream
the oracle and the CUDA kernels use (key = (seed, pass), counter = (pixel,
draw // 4, scene, 0), draw = (word >> 8) * 2^-24), so the lifted reference
code and the oracle consume identical random numbers.
"""
import math
import types

import numpy as np

f32 = np.float32
_MASK = 0xFFFFFFFF


# --------------------------------------------------------------------- scalars
class I32:
    """A Taichi i32 value.  Integer arithmetic stays integer; mixing with a
    float gives float32 (Taichi promotes i32 op f32 to f32, where a Python int
    would promote to float64); ``/`` is float division.  Not an ``int``
    subclass: NumPy and Python's float would treat a subclass as a strong
    int64 / plain int and promote to float64 before these methods run."""

    __slots__ = ("v",)
    __array_ufunc__ = None  # NumPy defers to the reflected methods below

    def __init__(self, v):
        self.v = int(v)

    def __index__(self):
        return self.v

    def __int__(self):
        return self.v

    def __float__(self):
        return float(self.v)

    def __hash__(self):
        return hash(self.v)

    def __bool__(self):
        return self.v != 0

    def __repr__(self):
        return "I32(%d)" % self.v

    @staticmethod
    def _isf(o):
        return isinstance(o, (float, np.floating))

    @staticmethod
    def _num(o):
        return o.v if isinstance(o, I32) else o

    def _op(self, o, op, rev=False):
        if isinstance(o, Vec):
            return NotImplemented
        if self._isf(o):
            a, b = f32(self.v), f32(o)
        else:
            a, b = self.v, int(self._num(o))
        r = op(b, a) if rev else op(a, b)
        return r if isinstance(r, np.floating) else I32(r)

    def __add__(self, o):
        return self._op(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._op(o, lambda a, b: a + b, True)

    def __sub__(self, o):
        return self._op(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._op(o, lambda a, b: a - b, True)

    def __mul__(self, o):
        if isinstance(o, Vec):
            return o * f32(self.v)
        return self._op(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._op(o, lambda a, b: a * b, True)

    def __truediv__(self, o):
        return f32(self.v) / f32(self._num(o))

    def __rtruediv__(self, o):
        return f32(self._num(o)) / f32(self.v)

    def __floordiv__(self, o):
        return I32(self.v // int(self._num(o)))

    def __mod__(self, o):
        return I32(self.v % int(self._num(o)))

    def __neg__(self):
        return I32(-self.v)

    def __abs__(self):
        return I32(abs(self.v))

    def __eq__(self, o):
        return self.v == self._num(o)

    def __ne__(self, o):
        return self.v != self._num(o)

    def __lt__(self, o):
        return self.v < self._num(o)

    def __le__(self, o):
        return self.v <= self._num(o)

    def __gt__(self, o):
        return self.v > self._num(o)

    def __ge__(self, o):
        return self.v >= self._num(o)


def _is_int(x):
    return isinstance(x, (I32, int, np.integer)) and not isinstance(x, bool)


def _sc(x):
    """A scalar as Taichi holds it: i32 stays integer, everything else f32."""
    if isinstance(x, bool):
        return I32(int(x))
    if _is_int(x):
        return I32(int(x))
    return f32(x)


def ti_pow(a, b):
    """``a ** b``: integer exponents by squaring (one rounding per multiply)."""
    if isinstance(b, (int, np.integer)) and not isinstance(b, bool):
        n = int(b)
        if _is_int(a):
            return I32(int(a) ** n)
        x = f32(a)
        if n < 0:
            x, n = f32(1.0) / x, -n
        r = f32(1.0)
        first = True
        while n:
            if n & 1:
                r = x if first else r * x
                first = False
            n >>= 1
            if n:
                x = x * x
        return r
    return np.power(f32(a), f32(b))


# --------------------------------------------------------------------- vectors
class Vec:
    """An immutable small float32 vector (tm.vec2 / tm.vec3 / ti.Vector of floats).
    Immutable, so that ``+=`` rebinds and no two records share state."""

    __slots__ = ("e",)
    __array_ufunc__ = None  # float32 scalars defer to __rmul__ etc. instead of making an array

    def __init__(self, items):
        self.e = tuple(f32(v) for v in items)

    # element access
    def __getitem__(self, i):
        return self.e[int(i)]

    def __len__(self):
        return len(self.e)

    def __iter__(self):
        return iter(self.e)

    x = property(lambda s: s.e[0])
    y = property(lambda s: s.e[1])
    z = property(lambda s: s.e[2])

    def _bin(self, o, op):
        if isinstance(o, Vec):
            return Vec(op(a, b) for a, b in zip(self.e, o.e))
        o = _sc(o)
        return Vec(op(a, o) for a in self.e)

    def __add__(self, o):
        return self._bin(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._bin(o, lambda a, b: b + a)

    def __sub__(self, o):
        return self._bin(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._bin(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._bin(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._bin(o, lambda a, b: b * a)

    def __truediv__(self, o):
        return self._bin(o, lambda a, b: a / b)

    def __rtruediv__(self, o):
        return self._bin(o, lambda a, b: b / a)

    def __neg__(self):
        return Vec(-a for a in self.e)

    def __pow__(self, o):
        return Vec(ti_pow(a, o) for a in self.e)

    def sum(self):
        r = self.e[0]
        for a in self.e[1:]:
            r = r + a
        return r

    def norm_sqr(self):
        return (self * self).sum()

    def norm(self, eps=0):
        return np.sqrt(self.norm_sqr() + f32(eps)) if eps else np.sqrt(self.norm_sqr())

    def __repr__(self):
        return "Vec(%s)" % ", ".join(repr(float(a)) for a in self.e)


class MutVec(list):
    """A mutable vector (``ti.types.vector(n, ...)`` instances written element by element)."""

    def __init__(self, n, dtype, fill):
        self.dtype = dtype
        super().__init__([self._cast(fill)] * n)

    def _cast(self, v):
        return I32(int(v)) if self.dtype is i32 else f32(v)

    def __setitem__(self, i, v):
        super().__setitem__(int(i), self._cast(v))

    def __getitem__(self, i):
        return super().__getitem__(int(i))


# --------------------------------------------------------------------- types
class _DType:
    def __init__(self, name):
        self.name = name

    def __repr__(self):
        return "ti." + self.name


f32_t = _DType("f32")
i32 = _DType("i32")


class VecType:
    def __init__(self, n, dtype=None):
        self.n, self.dtype = n, dtype or f32_t

    def __call__(self, *args):
        if len(args) == 1 and self.n > 1 and not isinstance(args[0], (Vec, list, tuple)):
            if self.n > 4:  # spectral vectors are written element by element
                return MutVec(self.n, self.dtype, args[0])
            return Vec([args[0]] * self.n)
        if len(args) == 1:
            return Vec(args[0])
        return Vec(args)

    def default(self):
        return Vec([0.0] * self.n) if self.n <= 4 else MutVec(self.n, self.dtype, 0)

    def cast(self, v):
        if isinstance(v, (Vec, MutVec)):
            return v if self.n > 4 else Vec(v)
        return self(v)


class Record:
    """An instance of a ``@ti.dataclass`` / ``ti.types.struct``: fields keep
    their declared types on every assignment (Taichi casts on store)."""

    __slots__ = ("_t", "_v")

    def __init__(self, rtype, kw):
        object.__setattr__(self, "_t", rtype)
        object.__setattr__(self, "_v", {})
        for name, ft in rtype.fields.items():
            self._v[name] = _default(ft)
        for name, val in kw.items():
            if name in rtype.fields:  # Taichi ignores unknown keywords here (main.py:1006)
                setattr(self, name, val)

    def __getattr__(self, name):
        try:
            return self._v[name]
        except KeyError:
            raise AttributeError(name)

    def __setattr__(self, name, val):
        self._v[name] = _cast(self._t.fields[name], val)

    def __repr__(self):
        return "%s(%s)" % (self._t.name, ", ".join("%s=%r" % kv for kv in self._v.items()))


class RecordType:
    def __init__(self, name, fields):
        self.name, self.fields = name, dict(fields)

    def __call__(self, **kw):
        return Record(self, kw)


def _default(ft):
    if ft is f32_t:
        return f32(0.0)
    if ft is i32:
        return I32(0)
    if isinstance(ft, VecType):
        return ft.default()
    if isinstance(ft, RecordType):
        return ft()
    raise TypeError(ft)


def _cast(ft, v):
    if ft is f32_t:
        return f32(v)
    if ft is i32:
        return I32(int(v))  # float -> int truncates toward zero, as a Taichi cast does
    if isinstance(ft, VecType):
        return ft.cast(v)
    return v


def dataclass(cls):
    ann = cls.__dict__.get("__annotations__", {})
    return RecordType(cls.__name__, ann)


def cast(v, t):
    return _cast(f32_t if t is f32_t else i32, v)


# --------------------------------------------------------------------- fields
class Field:
    """A Taichi field backed by a NumPy array; reads give Taichi-typed values."""

    def __init__(self, arr, vec=False):
        self.a = arr
        self.vec = vec

    def _wrap(self, v):
        if self.vec:
            return Vec(v)
        if isinstance(v, np.ndarray):
            return v if v.ndim else _sc(v[()])
        if isinstance(v, np.integer):
            return I32(int(v))
        if isinstance(v, np.floating):
            return f32(v)
        return v

    @staticmethod
    def _key(k):
        if k is None:
            return ()
        if isinstance(k, tuple):
            return tuple(int(x) for x in k)
        return int(k)

    def __getitem__(self, k):
        return self._wrap(self.a[self._key(k)])

    def __setitem__(self, k, v):
        self.a[self._key(k)] = np.asarray(list(v) if isinstance(v, (Vec, MutVec)) else v, dtype=self.a.dtype)


class RecordField:
    """A field of records (``triangles``, ``bvh_nodes``)."""

    def __init__(self, records):
        self.r = records

    def __getitem__(self, k):
        return self.r[int(k)]


class DepositLog:
    """``block_accumulator`` for one pass: every ``+=`` is recorded as a
    separate deposit (pixel, band, value), so that tests can sum them in FP64
    and see which ones the reference made NaN."""

    def __init__(self):
        self.log = []

    def __getitem__(self, k):
        return f32(0.0)

    def __setitem__(self, k, v):
        i, j, b = (int(x) for x in k)
        self.log.append((i, j, b, float(v)))


class PixelDomain:
    """``pixels_geometry`` as the domain of the kernel's struct-for: yields
    the selected (i, j) and switches RNG to that pixel's stream first."""

    def __init__(self, pixels, width, seed, pass_idx, scene_id=0):
        self.pixels, self.width = pixels, width
        self.seed, self.pass_idx, self.scene_id = seed, pass_idx, scene_id
        self.draws = []

    def __iter__(self):
        for (i, j) in self.pixels:
            RNG.stream(self.seed, self.pass_idx, int(j) * self.width + int(i), self.scene_id)
            yield I32(int(i)), I32(int(j))
            self.draws.append(RNG.n)  # draws the pixel's path consumed


# --------------------------------------------------------------------- random
def philox4x32_10(ctr, key):
    """Philox-4x32-10 block (Salmon, Moraes, Dror, Shaw, SC'11)."""
    c0, c1, c2, c3 = (int(x) & _MASK for x in ctr)
    k0, k1 = (int(x) & _MASK for x in key)
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & _MASK
            k1 = (k1 + 0xBB67AE85) & _MASK
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        n0 = (p1 >> 32) ^ c1 ^ k0
        n2 = (p0 >> 32) ^ c3 ^ k1
        c1 = p1 & _MASK
        c3 = p0 & _MASK
        c0, c2 = n0, n2
    return c0, c1, c2, c3


class RandomSource:
    def __init__(self):
        self.mode = "list"
        self.draws = []
        self.n = 0

    def stream(self, seed, pass_idx, pixel, scene_id=0):
        self.mode = "philox"
        self.key = (seed & _MASK, pass_idx & _MASK)
        self.pix, self.scene = pixel & _MASK, scene_id & _MASK
        self.n = 0
        self.buf = None

    def replay(self, draws):
        self.mode = "list"
        self.draws = [f32(d) for d in draws]
        self.n = 0

    def next(self):
        if self.mode == "philox":
            if self.n & 3 == 0:
                self.buf = philox4x32_10((self.pix, self.n >> 2, self.scene, 0), self.key)
            x = self.buf[self.n & 3]
            self.n += 1
            return f32(x >> 8) * f32(1.0 / 16777216.0)
        if self.n >= len(self.draws):
            raise IndexError("the replayed draw list ran out after %d draws" % self.n)
        v = self.draws[self.n]
        self.n += 1
        return v


RNG = RandomSource()


# --------------------------------------------------------------------- tm
def _vmap(f, *xs):
    if any(isinstance(x, Vec) for x in xs):
        n = max(len(x) for x in xs if isinstance(x, Vec))
        cols = [x.e if isinstance(x, Vec) else (x,) * n for x in xs]
        return Vec(f(*c) for c in zip(*cols))
    return f(*xs)


def _max(a, b):
    if _is_int(a) and _is_int(b):
        return I32(max(int(a), int(b)))
    return f32(np.fmax(f32(a), f32(b)))


def _min(a, b):
    if _is_int(a) and _is_int(b):
        return I32(min(int(a), int(b)))
    return f32(np.fmin(f32(a), f32(b)))


def _dot(a, b):
    return (a * b).sum()


def _cross(a, b):
    return Vec((a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]))


def _normalize(v):
    return v / v.norm()


def _reflect(x, n):
    return x - f32(2.0) * _dot(x, n) * n


def _refract(x, n, eta):
    dxn = _dot(x, n)
    result = x * f32(0.0)
    k = f32(1.0) - eta * eta * (f32(1.0) - dxn * dxn)
    if k >= 0.0:
        result = eta * x - (eta * dxn + np.sqrt(k)) * n
    return result


def _sign(x):
    x = f32(x)
    return f32(1.0) if x > 0 else (f32(-1.0) if x < 0 else f32(0.0))


def _u(fn):
    return lambda x: _vmap(lambda a: f32(fn(f32(a))), x)


tm = types.SimpleNamespace(
    pi=math.pi,
    vec2=VecType(2), vec3=VecType(3), vec4=VecType(4),
    dot=_dot, cross=_cross, normalize=_normalize, length=lambda v: v.norm(),
    reflect=_reflect, refract=_refract,
    max=lambda a, b: _vmap(_max, a, b), min=lambda a, b: _vmap(_min, a, b),
    clamp=lambda x, lo, hi: _vmap(lambda a, l, h: _min(_max(a, l), h), x, lo, hi),
    sign=_sign,
    acos=_u(np.arccos), cos=_u(np.cos), sin=_u(np.sin), tan=_u(np.tan), log=_u(np.log), exp=_u(np.exp),
    sqrt=_u(np.sqrt), pow=lambda a, b: _vmap(ti_pow, a, b),
)


def _identity(fn):
    return fn


def _vector(items, dt=None):
    items = list(items)
    if dt is i32 or all(_is_int(v) for v in items):
        return [I32(int(v)) for v in items]  # integer vectors are written element by element
    return Vec(items)


ti = types.SimpleNamespace(
    f32=f32_t, i32=i32,
    func=_identity, kernel=_identity, dataclass=dataclass,
    types=types.SimpleNamespace(vector=lambda n, dtype=None: VecType(n, dtype),
                                struct=lambda **fields: RecordType("struct", fields)),
    Vector=_vector,
    math=tm,
    random=lambda dtype=None: RNG.next(),
    ndrange=lambda n: (I32(k) for k in range(int(n))),
    cast=cast,
    sqrt=_u(np.sqrt), exp=_u(np.exp), log=_u(np.log), cos=_u(np.cos), sin=_u(np.sin),
    abs=lambda x: _vmap(lambda a: abs(a), x),
)
