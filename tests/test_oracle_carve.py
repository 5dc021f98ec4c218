"""Silhouette carving and the bounding-box search (RenderUtils::bbox_silhouette,
RenderUtils.cu:181-478) in the oracle: properties that hold for the reference's kernels."""
import numpy as np

import cpx_scenes as S
import orc


def _scene(n=32, seed=4, cams=4, img=48):
    rng = np.random.default_rng(seed)
    c, s, p = S.random_blobs(rng, 4)
    dens = S.blob_density(n, n, n, c, s, p)
    params = S.make_params(dens, 9, rng, 0.3)
    sc = orc.Scene(n, n, n, 9, params, step=0.5)
    views = [S.look_at_camera(e, n, img, img, fov_deg=45.0) for e in S.fibonacci_sphere(cams, 4.0)]
    images = []
    for cam in views:
        out = orc.render_image(sc, cam, (0, n - 1, 0, n - 1, 0, n - 1), img, img, False)
        # silhouettes: the mask plane; colour planes black (the reference tests any of the four)
        z = np.zeros(img * img, np.uint8)
        images.append((z, z, z, out["mask"]))
    return n, params, views, images, img


def _carve(n, params, views, images, img, radius):
    d = params[0].copy()
    lr = np.ones(n ** 3, np.float32)
    for cam, im in zip(views, images):
        orc.carve_silhouette(d, lr, n, n, n, S.projection_matrix(cam), im, img, img, radius)
    return d, lr


def test_dense_content_survives_and_empty_space_goes():
    n, params, views, images, img = _scene()
    d, lr = _carve(n, params, views, images, img, 0)
    core = params[0] > 20.0  # well inside the blobs: every view's silhouette covers them
    assert core.sum() > 20
    assert np.all(d[core] == params[0][core]) and np.all(lr[core] == 1.0)
    carved = lr == 0
    assert 0.3 < carved.mean() < 0.99
    assert np.all(d[carved] == 0) and np.all(d[~carved] == params[0][~carved])


def test_a_wider_radius_keeps_more():
    n, params, views, images, img = _scene()
    _, lr0 = _carve(n, params, views, images, img, 0)
    _, lr1 = _carve(n, params, views, images, img, 1)
    assert np.all(lr1[lr0 == 1] == 1) and (lr1 == 1).sum() > (lr0 == 1).sum()


def test_blank_images_carve_everything():
    n, params, views, _, img = _scene()
    z = np.zeros(img * img, np.uint8)
    d, lr = _carve(n, params, views, [(z, z, z, z)] * len(views), img, 2)
    assert not lr.any() and not d.any()
    box, ratio = orc.bbox(lr, n, n, n)
    assert box == (n, -1, n, -1, n, -1) and ratio == 0.0


def test_bbox_of_a_known_block_and_the_last_slice_quirk():
    W, H, D = 20, 18, 16
    lr = np.zeros((D, H, W), np.float32)
    lr[5:8, 4:13, 3:11] = 1.0
    # a column whose only kept vertex is the last depth slice does not count (the search stops
    # on it and takes it for the column's end, RenderUtils.cu:266-285)
    lr[D - 1, 0, 0] = 1.0
    box, ratio = orc.bbox(lr.reshape(-1), W, H, D)
    assert box == (3, 10, 4, 12, 5, 7)
    # the scale ratio counts every kept vertex, the quirk's one included: it is the farthest
    far = np.sqrt((0 - H / 2) ** 2 + (0 - W / 2) ** 2 + (D - 1 - D / 2) ** 2)
    assert abs(ratio - far / W * 2) < 1e-12
