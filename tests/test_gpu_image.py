"""Held-out view render (cpx_render_image) against the oracle and against the reference's own
image kernel (RenderUtils::renderImage, RenderUtils.cu:1720-1810) on the same GPU.

Tolerances: colour within 1e-5 absolute, expected depth within 1e-5 relative; the bytes
(rgb8, mask) are conversions of those floats, compared exactly against the reference's kernel
and within one count of the oracle (a float that lands on a rounding boundary may convert
either way when the host's exp differs from the device's in the last place)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RGB_ABS = 1e-5
DEPTH_REL = 1e-5


def _case(seed=0, n=64, sparse=None):
    import cpx_scenes as S

    rng = np.random.default_rng(seed)
    centres, sigmas, peaks = S.random_blobs(rng, 8)
    dens = S.blob_density(n, n, n, centres, sigmas, peaks)
    params = S.make_params(dens, 9, rng, 0.3)
    cams = [S.look_at_camera(p, n, 96, 80) for p in S.fibonacci_sphere(3, 4.0)]
    return {"n": n, "params": params, "cams": cams, "bbox": (0, n - 1, 0, n - 1, 0, n - 1)}


def _ours(case, sparse_threshold=None):
    import cpx

    n = case["n"]
    scene = cpx.ObjectScene(n, n, n, 9, step_size=0.5)
    scene.upload_params(case["params"])
    if sparse_threshold is not None:
        scene.prune_self(sparse_threshold)
        scene.make_sparse()
    return scene


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def _close(a, b):
    assert np.abs(a["rgb"] - b["rgb"]).max() <= RGB_ABS
    assert np.abs(a["depth"].astype(np.float64) - b["depth"]).max() <= DEPTH_REL * max(np.abs(b["depth"]).max(), 1.0)


@pytest.mark.parametrize("white", [True, False])
def test_image_matches_reference_kernel(cuda, white):
    import cpx
    import refharness as R

    case = _case(seed=1)
    n = case["n"]
    scene = _ours(case)
    ref = R.RefScene(n, n, n, 9, 2, 0.5, case["params"])
    for cam in case["cams"]:
        got = _host(cpx.RenderUtils.renderImage(scene, cpx.Camera.make(**cam), 96, 80, whiteBG=white))
        want = ref.render_image(cam, 96, 80, white)
        _close(got, want)
        assert np.array_equal(got["rgb8"], want["rgb8"])
        assert np.array_equal(got["mask"], want["mask"])
        assert got["mask"].max() > 0
    ref.close()


def test_oracle_image_pinned_to_reference(cuda):
    """The oracle's image path against the reference's kernel (pins the CPU restatement)."""
    import orc
    import refharness as R

    case = _case(seed=2)
    n = case["n"]
    ref = R.RefScene(n, n, n, 9, 2, 0.5, case["params"])
    osc = orc.Scene(n, n, n, 9, case["params"], step=0.5)
    for cam in case["cams"]:
        want = ref.render_image(cam, 96, 80, True)
        got = orc.render_image(osc, cam, case["bbox"], 96, 80, True)
        _close(got, want)
        assert np.abs(got["rgb8"].astype(int) - want["rgb8"]).max() <= 1
        assert np.mean(got["rgb8"] == want["rgb8"]) > 0.999
        assert np.abs(got["mask"].astype(int) - want["mask"]).max() <= 1
    ref.close()


def test_image_matches_oracle(cuda):
    import cpx
    import orc

    case = _case(seed=3)
    n = case["n"]
    scene = _ours(case)
    osc = orc.Scene(n, n, n, 9, case["params"], step=0.5)
    for cam in case["cams"]:
        got = _host(cpx.RenderUtils.renderImage(scene, cpx.Camera.make(**cam), 96, 80))
        want = orc.render_image(osc, cam, case["bbox"], 96, 80, True)
        _close(got, want)
        assert np.abs(got["rgb8"].astype(int) - want["rgb8"]).max() <= 1
        assert np.abs(got["mask"].astype(int) - want["mask"]).max() <= 1


def test_sparse_image_matches_reference_kernel(cuda):
    import cpx
    import refharness as R

    case = _case(seed=4)
    n = case["n"]
    scene = _ours(case, sparse_threshold=1.0)
    ref = R.RefScene(n, n, n, 9, 2, 0.5, case["params"], sparse_threshold=1.0)
    for cam in case["cams"]:
        got = _host(cpx.RenderUtils.renderImage(scene, cpx.Camera.make(**cam), 96, 80))
        want = ref.render_image(cam, 96, 80, True)
        _close(got, want)
        assert np.array_equal(got["rgb8"], want["rgb8"])
        assert np.array_equal(got["mask"], want["mask"])
    ref.close()


def test_partial_outputs_and_image_error(cuda):
    import torch

    import cpx

    case = _case(seed=5, n=32)
    scene = _ours(case)
    cam = cpx.Camera.make(**case["cams"][0])
    full = cpx.RenderUtils.renderImage(scene, cam, 96, 80)
    only = cpx.RenderUtils.renderImage(scene, cam, 96, 80, outputs=("rgb",))
    assert set(only) == {"rgb"}
    assert torch.equal(only["rgb"], full["rgb"])
    gen = torch.Generator(device="cpu").manual_seed(0)
    other = torch.rand(full["rgb"].shape, generator=gen).to(full["rgb"].device)
    mse = cpx.image_mse(full["rgb"], other)
    want = float(((full["rgb"].double() - other.double()) ** 2).mean())
    assert abs(mse - want) <= 1e-12 * max(want, 1.0)
    assert abs(cpx.image_psnr(full["rgb"], other) - 10 * np.log10(1 / want)) < 1e-9
    with pytest.raises(ValueError):
        cpx.image_mse(full["rgb"], full["rgb"][:1])
