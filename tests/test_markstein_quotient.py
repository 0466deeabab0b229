"""The IGR record sweep's quotient (div_markstein in sifv_kernels.cuh),
restated on the host with the C library's fused multiply-add: for
y = RN(1 / b), q0 = a y, q1 = q0 + (a - b q0) y, q = q1 + (a - b q1) y equals
the IEEE quotient a / b bit for bit whenever a is +0 or |a| and |y| lie in
[2^-450, 2^450] (the range the kernel checks before taking this path).

The device form is checked against IEEE division on the GPU by the IGR
parity tests (bit-identical sigma); this test pins the arithmetic itself on
adversarial operands: significands near 1 and near 2, numerators close to the
divisor, exact quotients, wide exponents and zeros.
"""
import ctypes
import ctypes.util
import math
import struct

import numpy as np
import pytest

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_fma = _libm.fma
_fma.restype = ctypes.c_double
_fma.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _in_range(x: float) -> bool:
    e = (_bits(x) >> 52) & 0x7FF
    return 573 <= e <= 1473


def _operand_ok(x: float) -> bool:
    return _in_range(x) or _bits(x) == 0


def markstein(a: float, b: float, y: float) -> float:
    q0 = a * y
    q1 = _fma(_fma(-q0, b, a), y, q0)
    return _fma(_fma(-q1, b, a), y, q1)


def _pairs(rng, n):
    out = []
    mant = rng.integers(0, 1 << 52, size=(n, 2), dtype=np.int64)
    exps = rng.integers(-100, 100, size=(n, 2))
    for k in range(n):
        kind = k % 6
        ma, mb = int(mant[k, 0]), int(mant[k, 1])
        ea, eb = int(exps[k, 0]), int(exps[k, 1])
        if kind == 1:
            mb = (1 << 52) - 1 - (mb & 0xFF)          # divisor significand near 2
        elif kind == 2:
            mb = mb & 0xFF                             # divisor significand near 1
        elif kind == 3:
            ma = mb ^ (ma & 0x3F)                      # numerator close to the divisor
        elif kind == 4:
            ea, eb = ea * 4, eb * 4                    # wide exponents (some out of range)
        a = struct.unpack("<d", struct.pack("<q", ((1023 + ea) << 52) | ma))[0]
        b = struct.unpack("<d", struct.pack("<q", ((1023 + eb) << 52) | mb))[0]
        if kind == 5:
            a = b * float(k % 97 + 1)                  # exact quotients
        if k & 1:
            a = -a
        out.append((a, b))
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_markstein_matches_ieee_division(seed):
    rng = np.random.default_rng(seed)
    fast = 0
    for a, b in _pairs(rng, 40000):
        y = 1.0 / b
        if not (_in_range(y) and _operand_ok(a)):
            continue
        fast += 1
        assert _bits(markstein(a, b, y)) == _bits(a / b), (a.hex(), b.hex())
    assert fast > 30000


def test_markstein_zero_numerator_sign():
    for b in (1.0, 3.5, 1e-300 * 2.0 ** 900, -2.0, -7.25):
        y = 1.0 / b
        assert _bits(markstein(0.0, b, y)) == _bits(0.0 / b)
    # -0 is outside the fast path (the kernel divides plainly): the sequence
    # would return +0 there
    assert not _operand_ok(-0.0)
    assert math.copysign(1.0, markstein(-0.0, 2.0, 0.5)) == 1.0
