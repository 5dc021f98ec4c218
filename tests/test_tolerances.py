"""The per-array gradient check of tests/tolerances.py catches what a pooled check misses."""
import numpy as np
import pytest

from tolerances import GRAD_REL, assert_grads_close, normwise


def test_small_array_error_is_caught_per_array():
    """A 100% error in a small-magnitude SH array passes a pooled normwise check but not
    the per-array one."""
    rng = np.random.default_rng(0)
    want = rng.normal(0, 1, (28, 1000))
    want[5] *= 1e-6
    got = want.copy()
    got[5] *= 2.0
    assert normwise(got, want) <= GRAD_REL  # the pooled check is blind to it
    with pytest.raises(AssertionError, match="array 5"):
        assert_grads_close(got, want)


def test_elementwise_error_above_floor_is_caught():
    rng = np.random.default_rng(1)
    want = rng.normal(0, 1, (4, 1000))
    got = want.copy()
    i = int(np.argsort(np.abs(want[2]))[500])  # a mid-magnitude element, above the floor
    got[2, i] *= 1 + 3 * GRAD_REL
    assert normwise(got[2], want[2]) <= GRAD_REL
    with pytest.raises(AssertionError, match="array 2"):
        assert_grads_close(got, want)
    assert_grads_close(want * (1 + 0.5 * GRAD_REL), want)


def test_zero_reference_array_must_stay_zero():
    want = np.zeros((2, 10))
    want[0] = 1.0
    got = want.copy()
    got[1, 3] = 1e-9
    with pytest.raises(AssertionError, match="reference is zero"):
        assert_grads_close(got, want)
