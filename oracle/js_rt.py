"""JavaScript semantics for code translated by oracle/ts2py.py.

TEST INFRASTRUCTURE ONLY.  The subset the reference's host-side builders use
(src/lib/gpu/bvh.ts): IEEE double numbers, ToInt32 / ToUint32 bitwise
operators, Math.min / max / floor with their NaN and signed-zero rules,
growable arrays, plain objects, typed arrays whose reads give doubles (a
Float32Array element read is the float widened to double, never float32
arithmetic) and whose writes convert as the ECMAScript typed-array setters do,
ArrayBuffer, Uint8Array views and DataView little/big-endian stores.
"""
from __future__ import annotations

import math
import struct

import numpy as np

Infinity = math.inf
NaN = math.nan
undefined = None


# ------------------------------------------------------------------ numbers
def to_int32(x) -> int:
    if isinstance(x, bool):
        x = int(x)
    if isinstance(x, float):
        if not math.isfinite(x):
            return 0
        x = math.trunc(x)
    n = int(x) & 0xFFFFFFFF
    return n - (1 << 32) if n & 0x80000000 else n


def to_uint32(x) -> int:
    if isinstance(x, bool):
        x = int(x)
    if isinstance(x, float):
        if not math.isfinite(x):
            return 0
        x = math.trunc(x)
    return int(x) & 0xFFFFFFFF


def js_bor(a, b):
    return to_int32(to_int32(a) | to_int32(b))


def js_band(a, b):
    return to_int32(to_int32(a) & to_int32(b))


def js_bxor(a, b):
    return to_int32(to_int32(a) ^ to_int32(b))


def js_bnot(a):
    return to_int32(~to_int32(a))


def js_shl(a, b):
    return to_int32(to_int32(a) << (to_uint32(b) & 31))


def js_shr(a, b):
    return to_int32(a) >> (to_uint32(b) & 31)


def js_ushr(a, b):
    return to_uint32(a) >> (to_uint32(b) & 31)


def js_neg(a):
    """Unary minus; -0 is a double in JavaScript (Python integers have no sign of zero)."""
    return -float(a) if a == 0 else -a


def js_mod(a, b):
    if isinstance(a, int) and isinstance(b, int) and b != 0:
        r = abs(a) % abs(b)
        return -r if a < 0 else r
    return math.fmod(a, b)


def js_div(a, b):
    if b == 0:
        if a == 0 or (isinstance(a, float) and math.isnan(a)):
            return math.nan
        neg = (a < 0) != (math.copysign(1.0, b) < 0)
        return -math.inf if neg else math.inf
    return a / b


def _is_neg_zero(x):
    return x == 0 and math.copysign(1.0, x) < 0


class _Math:
    PI = math.pi

    @staticmethod
    def min(*xs):
        r = math.inf
        for x in xs:
            if isinstance(x, float) and math.isnan(x):
                return math.nan
            if x < r or (x == r == 0 and _is_neg_zero(x)):
                r = x
        return r

    @staticmethod
    def max(*xs):
        r = -math.inf
        for x in xs:
            if isinstance(x, float) and math.isnan(x):
                return math.nan
            if x > r or (x == r == 0 and _is_neg_zero(r)):
                r = x
        return r

    @staticmethod
    def floor(x):
        if isinstance(x, float) and not math.isfinite(x):
            return x
        return math.floor(x)

    @staticmethod
    def ceil(x):
        if isinstance(x, float) and not math.isfinite(x):
            return x
        return math.ceil(x)

    @staticmethod
    def abs(x):
        return abs(x)

    @staticmethod
    def sqrt(x):
        return math.sqrt(x) if x >= 0 else math.nan


Math = _Math()


def _idx(i):
    if isinstance(i, float):
        if not i.is_integer():
            raise IndexError(f"non-integer index {i}")
        return int(i)
    return i


# ------------------------------------------------------------------ objects, arrays
class JSObj:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class JSArray(list):
    @property
    def length(self):
        return len(self)

    def push(self, *xs):
        self.extend(xs)
        return len(self)

    def slice(self, a=0, b=None):
        n = len(self)
        a = _idx(a)
        b = n if b is None else _idx(b)
        a = max(n + a, 0) if a < 0 else min(a, n)
        b = max(n + b, 0) if b < 0 else min(b, n)
        return JSArray(list.__getitem__(self, slice(a, b)))

    def __getitem__(self, i):
        if isinstance(i, slice):  # Python-side access to the contents
            return list.__getitem__(self, i)
        i = _idx(i)
        return list.__getitem__(self, i) if 0 <= i < len(self) else None

    def __setitem__(self, i, v):
        i = _idx(i)
        if i >= len(self):
            self.extend([None] * (i + 1 - len(self)))
        list.__setitem__(self, i, v)


class _ArrayCtor:
    def __call__(self, n=0):
        return JSArray([None] * _idx(n))

    @staticmethod
    def from_(obj, fn=None):
        n = _idx(obj.length)
        return JSArray([fn(None, k) if fn else None for k in range(n)])


Array = _ArrayCtor()


class ArrayBuffer:
    def __init__(self, n=0):
        self.b = bytearray(_idx(n))

    @property
    def byteLength(self):
        return len(self.b)

    def slice(self, a=0, b=None):
        out = ArrayBuffer(0)
        out.b = bytearray(self.b[_idx(a):(None if b is None else _idx(b))])
        return out


class _Typed:
    dtype = None

    def __init__(self, arg=0):
        if isinstance(arg, ArrayBuffer):
            self.a = np.frombuffer(arg.b, dtype=self.dtype)  # a view (writes reach the buffer)
        elif isinstance(arg, (int, float)):
            self.a = np.zeros(_idx(arg), self.dtype)
        elif isinstance(arg, _Typed):
            self.a = np.array([self._conv(float(x)) for x in arg.a.tolist()], self.dtype)
        else:
            self.a = np.array([self._conv(x) for x in arg], self.dtype)

    @property
    def length(self):
        return int(self.a.shape[0])

    def __len__(self):
        return self.length

    def __getitem__(self, i):
        i = _idx(i)
        return self.a[i].item() if 0 <= i < self.a.shape[0] else None

    def __setitem__(self, i, v):
        i = _idx(i)
        if 0 <= i < self.a.shape[0]:
            self.a[i] = self._conv(v)

    def set(self, src, offset=0):
        if isinstance(src, _Typed) and src.dtype == self.dtype:
            n = src.a.shape[0]
            if offset + n > self.a.shape[0]:
                raise IndexError("typed array set out of range")  # RangeError in JavaScript
            self.a[offset:offset + n] = src.a
            return
        vals = src.a if isinstance(src, _Typed) else src
        for k, v in enumerate(vals.tolist() if hasattr(vals, "tolist") else vals):
            self[offset + k] = v

    def __iter__(self):
        return iter(self.a.tolist())


class Float32Array(_Typed):
    dtype = np.float32

    @staticmethod
    def _conv(v):
        return np.float32(v)  # round to nearest, ties to even; overflow to infinity


class Float64Array(_Typed):
    dtype = np.float64

    @staticmethod
    def _conv(v):
        return float(v)


class Int32Array(_Typed):
    dtype = np.int32

    @staticmethod
    def _conv(v):
        return to_int32(v)


class Uint32Array(_Typed):
    dtype = np.uint32

    @staticmethod
    def _conv(v):
        return to_uint32(v)


class Uint8Array(_Typed):
    dtype = np.uint8

    @staticmethod
    def _conv(v):
        return to_uint32(v) & 0xFF


class DataView:
    def __init__(self, buf):
        self.buf = buf

    def _put(self, fmt, off, v, le):
        struct.pack_into(("<" if le else ">") + fmt, self.buf.b, _idx(off), v)

    def setFloat32(self, off, v, le=False):
        with np.errstate(over="ignore"):
            f = float(np.float32(v))
        self._put("f", off, f, le)

    def setUint32(self, off, v, le=False):
        self._put("I", off, to_uint32(v), le)

    def setInt32(self, off, v, le=False):
        self._put("i", off, to_int32(v), le)

    def getFloat32(self, off, le=False):
        return struct.unpack_from(("<" if le else ">") + "f", self.buf.b, _idx(off))[0]

    def getUint32(self, off, le=False):
        return struct.unpack_from(("<" if le else ">") + "I", self.buf.b, _idx(off))[0]
