"""DistributedVector operations (linalg/dvector.rs:46-160) on the device.

dot / dot_smaller / sum use a fixed reduction order (not the reference's
serial loop): equal to the serial sum to rounding, and the same bits on every
call.  +=, -=, *= (scalar), inv and set / set_smaller are exact.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reductions(fv):
    rng = np.random.default_rng(4)
    for n in (1, 31, 1000, 1_000_003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        x, y = fv.DistributedVector(a), fv.DistributedVector(b)
        serial = 0.0
        for u, v in zip(a[:5000], b[:5000]):  # the reference's loop on a prefix, exact check below
            serial += u * v
        d = x.dot(y)
        exact = math.fsum(a * b)
        assert abs(d - exact) <= 1e-13 * max(1.0, math.fsum(abs(a * b)))
        assert x.dot(y) == d  # same bits on repeat
        assert abs(x.sum() - math.fsum(a)) <= 1e-13 * max(1.0, math.fsum(abs(a)))
        if n <= 5000:
            assert abs(d - serial) <= 1e-13 * max(1.0, math.fsum(abs(a * b)))
    short = fv.DistributedVector(np.arange(5.0))
    long_ = fv.DistributedVector(np.arange(9.0))
    assert short.dot_smaller(long_) == 30.0
    with pytest.raises(ValueError):
        short.dot(long_)
    assert fv.DistributedVector.from_size(0).sum() == 0.0


def test_elementwise_updates(fv):
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(10007), rng.standard_normal(10007)
    x, y = fv.DistributedVector(a.copy()), fv.DistributedVector(b)
    x += y
    assert np.array_equal(x.numpy(), a + b)
    x -= y
    assert np.array_equal(x.numpy(), (a + b) - b)
    x *= 0.37
    assert np.array_equal(x.numpy(), ((a + b) - b) * 0.37)
    z = fv.DistributedVector(b.copy()).inv()
    assert np.array_equal(z.numpy(), 1.0 / b)
    w = fv.DistributedVector.from_size(10007)
    w.set(y)
    assert np.array_equal(w.numpy(), b)
    s = fv.DistributedVector(np.zeros(20))
    s.set_smaller(fv.DistributedVector(np.arange(8.0)))
    assert np.array_equal(s.numpy(), np.concatenate([np.arange(8.0), np.zeros(12)]))
    s[3] = 7.5
    assert s[3] == 7.5 and s[4] == 4.0
