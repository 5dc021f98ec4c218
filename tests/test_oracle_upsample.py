"""Coarse-to-fine upsampling of the oracle (upsampleScene, SceneUtils.cu:262-485): properties
that hold for the reference's kernel, on the CPU."""
import numpy as np

import cpx_scenes as S
import orc


def _src(n=16, seed=2, sparse_threshold=None):
    rng = np.random.default_rng(seed)
    c, s, p = S.random_blobs(rng, 5)
    params = S.make_params(S.blob_density(n, n, n, c, s, p), 9, rng, 0.3)
    if sparse_threshold is None:
        return orc.Scene(n, n, n, 9, params), params
    occ, cage, idx, cnt, _ = orc.occupancy(params[0], n, n, n, sparse_threshold)
    comp = orc.compact(params, cage, cnt)
    return orc.Scene(n, n, n, 9, comp, sparse=True, occ=occ, index_offsets=idx, in_cage=cage), params


def test_even_vertices_copy_the_source_and_midpoints_average():
    sc, params = _src()
    n = 16
    up = orc.upsample(sc, 2 * n, 2 * n, 2 * n, threshold=-1.0)
    src = params.reshape(28, n, n, n)
    dst = up.reshape(28, 2 * n, 2 * n, 2 * n)
    assert np.array_equal(dst[:, ::2, ::2, ::2], src)
    # x-midpoints between two source vertices (y, z even): the float mean of the two
    mid = dst[:, ::2, ::2, 1:-1:2]
    want = (0.5 * src[:, :, :, :-1].astype(np.float64) + 0.5 * src[:, :, :, 1:]).astype(np.float32)
    assert np.abs(mid - want).max() <= 1e-6 * np.abs(want).max()
    # the last vertex of each axis repeats the clamped source vertex
    assert np.array_equal(dst[:, ::2, ::2, -1], src[:, :, :, -1])


def test_threshold_and_low_band():
    sc, params = _src()
    n = 16
    up = orc.upsample(sc, 2 * n, 2 * n, 2 * n, threshold=5.0)
    full = orc.upsample(sc, 2 * n, 2 * n, 2 * n, threshold=-1.0)
    below = full[0] < 5.0
    assert below.any() and (~below).any()
    assert not up[0][below].any()
    assert np.array_equal(up[0][~below], full[0][~below])
    low = orc.upsample(sc, 2 * n, 2 * n, 2 * n, threshold=-1.0, low_band_only=True, dst_sh=9)
    k = np.arange(27) % 9
    assert np.array_equal(low[1:][k == 0], full[1:][k == 0])
    assert not low[1:][k != 0].any()


def test_sparse_source_zeros_outside_its_cells():
    sc, params = _src(sparse_threshold=8.0)
    dense, _ = _src()
    n = 16
    up = orc.upsample(sc, 2 * n, 2 * n, 2 * n, threshold=-1.0)
    ref = orc.upsample(dense, 2 * n, 2 * n, 2 * n, threshold=-1.0)
    zero = ~up.any(0)
    assert zero.any() and (~zero).any()
    # where the sparse source's cell is occupied and all corners are in cage, the values agree
    agree = np.isclose(up, ref, rtol=0, atol=0).all(0)
    assert agree[~zero].mean() > 0.5
