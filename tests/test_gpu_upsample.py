"""Coarse-to-fine upsampling (cpx_grid_upsample) against the oracle and against the reference's
own objectScene::initSelfByUpsample (upsampleScene) on the same GPU: bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(n, seed):
    import cpx_scenes as S

    rng = np.random.default_rng(seed)
    c, s, p = S.random_blobs(rng, 6)
    return S.make_params(S.blob_density(n, n, n, c, s, p), 9, rng, 0.3)


@pytest.mark.parametrize("low_band", [False, True])
def test_upsample_matches_reference_and_oracle(cuda, low_band):
    import cpx
    import orc
    import refharness as R

    n = 24
    params = _params(n, 3)
    src = cpx.ObjectScene(n, n, n, 9)
    src.upload_params(params)
    dst = cpx.ObjectScene(2 * n, 2 * n, 2 * n, 1 if low_band else 9)
    dst.init_by_upsample(src, threshold=2.0, low_band_only=low_band)
    got = dst.download_params()
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params)
    # the reference's low-band refinement: lowBandOnly with a one-coefficient target (its dense
    # path takes the kernel's low-band flag from src.sh_dim != targetSH_dim)
    want = ref.upsample(2.0, low_band_only=low_band, target_sh=1 if low_band else None)
    ref.close()
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    osc = orc.Scene(n, n, n, 9, params)
    assert np.array_equal(got, orc.upsample(osc, 2 * n, 2 * n, 2 * n, 2.0, low_band_only=low_band))


def test_sparse_source_and_sparse_target(cuda):
    """A sparse source (zeros in its unoccupied cells) against the reference; then the target
    made sparse as the reference's initSelfByUpsample does, and marched."""
    import torch

    import cpx
    import refharness as R

    n = 24
    params = _params(n, 4)
    src = cpx.ObjectScene(n, n, n, 9)
    src.upload_params(params)
    src.prune_self(6.0)
    src.make_sparse()
    dst = cpx.ObjectScene(2 * n, 2 * n, 2 * n, 9)
    dst.init_by_upsample(src, threshold=1.0)
    got = dst.download_params()
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params, sparse_threshold=6.0)
    want = ref.upsample(1.0)
    ref.close()
    assert np.array_equal(got, want)
    assert (got[0] == 0).mean() > 0.3
    # the reference's sparse target: prune the dense target and compact it
    occ, cage, idx, cnt = dst.prune_self(1.0)
    dst.make_sparse()
    assert dst.actual_grid_nums == cnt > 0
    compact = dst.download_params()
    assert np.array_equal(compact, got[:, cage.astype(bool)])
    # a second refinement from the sparse target into a sparse target of its own occupancy
    fine = cpx.ObjectScene(4 * n, 4 * n, 4 * n, 9)
    fine.init_by_upsample(dst, threshold=1.0)
    assert fine.download_params()[0].max() > 0
