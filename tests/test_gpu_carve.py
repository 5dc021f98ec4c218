"""Silhouette carving and the bounding-box search (cpx_carve_silhouette, cpx_grid_bbox) against
the reference's own RenderUtils::bbox_silhouette (RenderUtils.cu:181-478) on the same GPU and
against the oracle: the carved parameters bit for bit, the box exactly, the scale ratio to
the last bit against the reference's kernel (within 1e-15 relative against the oracle)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed=6, n=40, cams=5, img=56):
    import cpx
    import cpx_scenes as S

    rng = np.random.default_rng(seed)
    c, s, p = S.random_blobs(rng, 5)
    params = S.make_params(S.blob_density(n, n, n, c, s, p), 9, rng, 0.3)
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(params)
    views = [S.look_at_camera(e, n, img, img, fov_deg=45.0) for e in S.fibonacci_sphere(cams, 4.0)]
    images = []
    for k, cam in enumerate(views):
        out = cpx.RenderUtils.renderImage(scene, cpx.Camera.make(**cam), img, img, whiteBG=False)
        rgb8 = out["rgb8"].cpu().numpy()
        mask = out["mask"].cpu().numpy()
        # the first view tests the colour planes (mask blank), the others the mask alone
        z = np.zeros(img * img, np.uint8)
        images.append((np.where(mask > 0, rgb8[0], 0).astype(np.uint8), z, z, z) if k == 0 else (z, z, z, mask))
    scene.close()
    return n, params, views, images, img


@pytest.mark.parametrize("radius", [0, 2])
def test_carving_matches_reference_kernel_and_oracle(cuda, radius):
    import cpx
    import cpx_scenes as S
    import orc
    import refharness as R

    n, params, views, images, img = _case()
    proj = [S.projection_matrix(c) for c in views]
    ours = cpx.ObjectScene(n, n, n, 9)
    ours.upload_params(params)
    sr = cpx.RenderUtils.bbox_silhouette(proj, images, ours, img, img, radius, isGettingScaleRatio=True)
    got = ours.download_params()
    box = ours.bbox

    ref = R.RefScene(n, n, n, 9, 2, 0.5, params)
    want_box, want_sr = ref.bbox_silhouette(proj, images, img, img, radius, get_scale=True)
    want = ref.params()
    want_lr = ref.adaptive_lr()
    ref.close()
    assert np.array_equal(got, want)
    assert box == want_box
    assert sr == want_sr
    assert 0.1 < (want_lr == 0).mean() < 0.99

    d = params[0].copy()
    lr = np.ones(n ** 3, np.float32)
    for P, im in zip(proj, images):
        orc.carve_silhouette(d, lr, n, n, n, P, im, img, img, radius)
    assert np.array_equal(lr, want_lr)
    assert np.array_equal(d, got[0])
    obox, osr = orc.bbox(lr, n, n, n)
    assert obox == box and abs(osr - sr) <= 1e-15 * sr


def test_mixed_grid_carves_its_density_and_box_becomes_the_ray_box(cuda):
    import cpx
    import cpx_scenes as S

    n, params, views, images, img = _case(seed=7)
    proj = [S.projection_matrix(c) for c in views]
    a = cpx.ObjectScene(n, n, n, 9)
    b = cpx.ObjectScene(n, n, n, 9, precision="bf16")
    for sc in (a, b):
        sc.upload_params(params)
        cpx.RenderUtils.bbox_silhouette(proj, images, sc, img, img, 1)
    pa, pb = a.download_params(), b.download_params()
    assert np.array_equal(pa[0], pb[0])
    assert a.bbox == b.bbox and a.bbox != (0, n - 1, 0, n - 1, 0, n - 1)  # a proper sub-box
    # the box is the grid's ray box now: rays from the same camera start and end inside it
    cam = views[1]
    rays = cpx.Rays(img * img)
    z = np.zeros(img * img, np.uint8)
    rays.initial_self(a, [cpx.Camera.make(**cam)], [(z, z, z, None)], [np.arange(img * img, dtype=np.int32)], img, img)
    geo = rays.download(fields=("ox", "oy", "oz", "dx", "dy", "dz", "near", "far"))
    hit = geo["near"] <= geo["far"]
    assert hit.any() and not hit.all()
    pts = np.stack([geo["ox"] + geo["near"] * geo["dx"], geo["oy"] + geo["near"] * geo["dy"],
                    geo["oz"] + geo["near"] * geo["dz"]], 1)[hit]
    lo = np.array(a.bbox[0::2], np.float64) - 1e-3
    hi = np.array(a.bbox[1::2], np.float64) + 1e-3
    assert np.all(pts >= lo) and np.all(pts <= hi)
