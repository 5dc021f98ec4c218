"""The ray source's shuffle (the keyed permutation of cpx_ray_source) in the oracle: a
bijection of [0, n) for any n, different orders for different seeds."""
import numpy as np
import pytest

import ray_source_ref as RS


@pytest.mark.parametrize("n", [1, 2, 3, 5, 64, 1000, 4097, 65537])
def test_permutation_is_a_bijection(n):
    keys = RS.splitmix64_keys(12345)
    p = RS.permute(np.arange(n), n, keys)
    assert np.array_equal(np.sort(p), np.arange(n))


def test_seeds_give_different_orders_and_the_domain_is_tight():
    n = 100_000
    a = RS.permute(np.arange(n), n, RS.splitmix64_keys(1))
    b = RS.permute(np.arange(n), n, RS.splitmix64_keys(2))
    assert (a != b).mean() > 0.99
    assert (a == np.arange(n)).mean() < 0.01
    # the Feistel domain is the next even power of two: at most 4 n, so the walk stays short
    assert (1 << (2 * RS.half_bits(n))) < 4 * n
    # a batch of consecutive samples draws from all over the table
    batch = a[:4096]
    assert np.histogram(batch, bins=8, range=(0, n))[0].min() > 4096 / 8 * 0.8
