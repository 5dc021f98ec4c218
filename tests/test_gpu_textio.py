"""The reference's text checkpoint (objectScene::saveSelf / initFromFile, SceneUtils.cu:703-790,
1246-1300) and image format (Image::initSelfFromFile): the files cpx_grid_save_text writes equal
the reference's own saveSelf output byte for byte; cpx_grid_load_text gives the parameters the
reference's initFromFile loads; cpx_image_load_text reads what the reference's reader reads."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(n, seed):
    import cpx_scenes as S

    rng = np.random.default_rng(seed)
    c, s, p = S.random_blobs(rng, 4)
    return S.make_params(S.blob_density(n, n, n, c, s, p), 9, rng, 0.3)


def _files(d):
    return sorted(os.listdir(d))


def _same_files(a, b, skip=()):
    assert _files(a) == _files(b)
    for f in _files(a):
        if f in skip:
            continue
        with open(os.path.join(a, f), "rb") as fa, open(os.path.join(b, f), "rb") as fb:
            assert fa.read() == fb.read(), f


@pytest.mark.parametrize("band,hierarchy", [(2, False), (1, True), (0, False)])
def test_dense_checkpoint_files_equal_the_reference(cuda, tmp_path, band, hierarchy):
    import cpx
    import refharness as R

    n = 20
    params = _params(n, band + 3)
    ours, theirs = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    theirs.mkdir()
    sc = cpx.ObjectScene(n, n, n, 9)
    sc.upload_params(params)
    cpx.save_text(sc, ours, band, hierarchy_mode=hierarchy)
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params)
    ref.save_text(theirs, band, hierarchy_mode=hierarchy)
    ref.close()
    # a dense scene never pruned writes its occupancy buffer uninitialised: not compared
    _same_files(ours, theirs, skip=("occupancy.txt",))


def test_dense_checkpoint_loads_as_the_reference_loads(cuda, tmp_path):
    import cpx
    import refharness as R

    n = 20
    params = _params(n, 9)
    d = tmp_path / "ckpt"
    d.mkdir()
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params)
    ref.save_text(d, 1)  # 4 coefficients per channel
    ref.close()
    want = R.load_text(d, n, n, n, 0.5, 4, 9)
    sc = cpx.ObjectScene(n, n, n, 9)
    cpx.load_text(sc, d, 4)
    got = sc.download_params()
    assert np.array_equal(got, want)
    # the values are the 6-decimal text of the originals
    assert np.abs(got[0] - params[0]).max() <= 5e-7 * max(1.0, np.abs(params[0]).max())
    assert not got[5:10].any() and not got[14:19].any()  # coefficients 4..8 were not in the files


def test_sparse_checkpoint_files_equal_the_reference(cuda, tmp_path):
    import cpx
    import refharness as R

    n = 20
    params = _params(n, 11)
    ours, theirs = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    theirs.mkdir()
    sc = cpx.ObjectScene(n, n, n, 9)
    sc.upload_params(params)
    sc.prune_self(1.0)
    sc.make_sparse()
    cpx.save_text(sc, ours, 2)
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params, sparse_threshold=1.0)
    ref.save_text(theirs, 2)
    ref.close()
    _same_files(ours, theirs)
    with open(os.path.join(ours, "sparse_inCageInfo_band2.txt")) as f:
        assert int(f.read()) == sc.actual_grid_nums


def test_image_text_reads_as_the_reference_reads(cuda, tmp_path):
    import cpx
    import refharness as R

    w, h = 41, 29
    rng = np.random.default_rng(2)
    prefix = str(tmp_path / "view")
    planes = [rng.integers(0, 256, w * h) for _ in range(3)]
    mask = np.zeros((h, w), np.int64)
    mask[3:20, 5:33] = 255
    for name, p in zip(("red", "green", "blue", "mask"), planes + [mask.reshape(-1)]):
        with open(prefix + "_%s.txt" % name, "w") as f:
            for r in range(h):
                f.write("".join("%d " % v for v in p[r * w:(r + 1) * w]) + "\n")
    img, box, pix = cpx.load_image_text(prefix, w, h)
    rimg, rbox, rpix = R.image_load_text(prefix, w, h)
    for a, b in zip(img, rimg):
        assert np.array_equal(a, b)
    assert box == rbox and np.array_equal(pix, rpix)
