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


def _sparse_scene(n, seed, thr=1.0):
    import cpx

    params = _params(n, seed)
    sc = cpx.ObjectScene(n, n, n, 9)
    sc.upload_params(params)
    occ, cage, idx, cnt = sc.prune_self(thr)
    sc.make_sparse()
    return sc, params, occ, cage, idx, cnt


def test_sparse_checkpoint_round_trip(cuda, tmp_path):
    """cpx_grid_save_text then cpx_grid_load_text_sparse: the same occupancy tables, the same
    compact parameters (as their 6-decimal text), and the same march."""
    import cpx

    n = 24
    sc, params, occ, cage, idx, cnt = _sparse_scene(n, 12)
    d = tmp_path / "ckpt"
    d.mkdir()
    cpx.save_text(sc, d, 2)
    want = sc.download_params()
    back = cpx.ObjectScene(n, n, n, 9)
    cpx.load_text_sparse(back, d, 9)
    assert back.sparse and back.actual_grid_nums == cnt
    occ2, cage2, idx2 = back.occupancy_tables()
    assert np.array_equal(occ2, occ) and np.array_equal(cage2, cage) and np.array_equal(idx2, idx)
    got = back.download_params()
    assert np.abs(got - want).max() <= 5e-7 * max(1.0, np.abs(want).max())
    # reloading the files of the reloaded grid gives identical bits
    d2 = tmp_path / "ckpt2"
    d2.mkdir()
    cpx.save_text(back, d2, 2)
    _same_files(d, d2)
    # both grids march the same (the loaded values are the text's)
    import cpx_scenes as S
    import torch

    cams = [S.look_at_camera(p, n, 48, 48) for p in S.fibonacci_sphere(4, 4.0)]
    rng = np.random.default_rng(1)
    pix = S.sample_pixels(rng, 4, 48, 48, 256)
    imgs = [tuple(rng.integers(0, 256, 48 * 48, dtype=np.uint8) for _ in range(3)) + (None,) for _ in range(4)]
    outs = []
    for g in (sc, back):
        g.upload_params(got)
        r = cpx.Rays(256)
        r.initial_self(g, [cpx.Camera.make(**c) for c in cams], imgs, pix, 48, 48)
        cpx.RenderUtils.renderRays(r, g)
        outs.append(r.download(fields=cpx.RAY_OUTPUTS))
        r.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k
    del torch


def test_sparse_checkpoint_of_the_reference_loads(cuda, tmp_path):
    """A sparse checkpoint written by the reference's own saveSelf loads into the grid the
    reference saved: occupancy, in-cage count and index offsets bit-exact, compact parameters
    as their text."""
    import cpx
    import refharness as R

    n = 20
    params = _params(n, 14)
    d = tmp_path / "ref"
    d.mkdir()
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params, sparse_threshold=1.0)
    ref.save_text(d, 2)
    rocc, rcage, ridx = ref.occupancy()
    rparams = ref.params()
    cnt = ref.in_cage_count
    ref.close()
    sc = cpx.ObjectScene(n, n, n, 9)
    cpx.load_text_sparse(sc, d, 9)
    assert sc.sparse and sc.actual_grid_nums == cnt
    got = sc.download_params()
    assert np.abs(got - rparams).max() <= 5e-7 * max(1.0, np.abs(rparams).max())
    occ, cage, idx = sc.occupancy_tables()
    assert np.array_equal(occ, rocc) and np.array_equal(idx, ridx) and np.array_equal(cage, rcage)


def test_inconsistent_sparse_checkpoint_is_refused(cuda, tmp_path):
    import cpx

    n = 20
    sc, *_ = _sparse_scene(n, 15)
    d = tmp_path / "ckpt"
    d.mkdir()
    cpx.save_text(sc, d, 2)
    with open(d / "sparse_inCageInfo_band2.txt", "w") as f:
        f.write("%d" % (sc.actual_grid_nums + 1))
    with pytest.raises(cpx.CpxError) as ei:
        cpx.load_text_sparse(cpx.ObjectScene(n, n, n, 9), d, 9)
    assert ei.value.name == "CPX_ERR_INVALID_ARGUMENT"
