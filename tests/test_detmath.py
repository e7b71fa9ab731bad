"""Portable elementary functions (detmath.h) and the Philox generator."""
import math

import numpy as np
import pytest

import hostcheck_ffi as H
from oracle_ffi import P


def _run(which, x):
    x = np.ascontiguousarray(x, float)
    y = np.zeros_like(x)
    H.load().hc_detmath(which, x.size, P(x), P(y))
    return y


def _ulps(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    sp = np.spacing(np.maximum(np.abs(b), 1e-300))
    return np.abs(a - b) / sp


@pytest.mark.parametrize("which,fn,lo,hi", [
    (0, math.exp, -700.0, 700.0),
    (0, math.exp, -1.0, 1.0),
    (1, math.log, 1e-300, 1e300),
    (1, math.log, 0.5, 2.0),
    (2, math.sin, -1e5, 1e5),
    (3, math.cos, -1e5, 1e5),
    (2, math.sin, -3.0, 3.0),
    (3, math.cos, -3.0, 3.0),
])
def test_accuracy_against_libm(which, fn, lo, hi):
    rng = np.random.default_rng(which + 7)
    if which == 1 and lo > 0 and hi / lo > 1e10:
        x = 10.0 ** rng.uniform(math.log10(lo), math.log10(hi), 20000)
    else:
        x = rng.uniform(lo, hi, 20000)
    y = _run(which, x)
    ref = np.array([fn(v) for v in x])
    if which >= 2:
        # absolute error relative to 1 for large-argument trig
        assert np.max(np.abs(y - ref)) < 4e-16 * max(1.0, abs(hi) * 1e-5) * 8
    else:
        assert np.max(_ulps(y, ref)) <= 4.0


def test_special_values():
    assert _run(0, [0.0])[0] == 1.0
    assert _run(1, [1.0])[0] == 0.0
    assert _run(0, [-800.0])[0] == 0.0
    assert math.isinf(_run(0, [800.0])[0])
    assert math.isinf(_run(1, [0.0])[0])
    assert math.isnan(_run(1, [-1.0])[0])
    assert _run(2, [0.0])[0] == 0.0
    assert _run(3, [0.0])[0] == 1.0


def _philox(ctr, key):
    import ctypes as C
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    H.load().hc_philox(c, k, o)
    return [o[i] for i in range(4)]


def test_philox_known_answers():
    # Philox4x32-10 known-answer vectors of Salmon et al. (Random123)
    assert _philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert _philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert _philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
