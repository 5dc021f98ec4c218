"""One whole training step of the CUDA path against the reference's own kernels, live on
the same GPU, at the two plain-FP32 sizes:

* the 128^3 plain case exactly (8 blobs, 16 Fibonacci views at 200x200, 4096 rays, one
  forward + backward + TV (lambda 1e-3, type 0, 6 neighbours) + Adam (0.1, 0.01));
* the 256^3 grid of the full-size tests with a 512-ray batch from 800x800 views.

The reference runs through oracle/_ref/libcpxref.so: its unmodified
SparseVolumeRadianceField sources built for sm_100a, called through
RenderUtils::renderRays (RenderUtils.cu:1961-1971), renderRays_withGradients_RGB
(RenderUtils.cu:2258-2278), addVarianceLoss (RenderUtils.cu:2815-2851) and
Optimizer::updateRGBScene (Optimizer.cu:451-479).

Bit-exact: ray fields, accumulated density and weight of every ray, and the sample counts
(against the oracle, which the CPU suite pins to the reference's golden outputs: the
reference's kernels do not report counts).  RGB within 1e-5 absolute, losses within
255e-5.  Gradients within 1e-4 relative per parameter array, and elementwise above the
floor of tests/tolerances.py.  TV + Adam: fed the reference's own gradients, the fused
sweep's parameters and moments equal the reference's within float rounding; after the
whole step (each arm on its own gradients) the parameters agree wherever the gradient is
not at rounding level, since at t = 1 a parameter moves by lr * sign(g).
"""
import numpy as np
import pytest

from tolerances import RGB_ABS, assert_grads_close, grad_report

pytestmark = pytest.mark.gpu

MASK_COEF = 1.0
HUBER = 0.1
LAM = 1e-3
LR, SH_LR = 0.1, 0.01


def _ref_available():
    import refharness

    return refharness.available()


def _rows_close(got, want, atol_of):
    """Row by row (parameter arrays of up to 16.8 M floats): the worst |got - want| - atol."""
    worst = -np.inf
    for k in range(want.shape[0]):
        a = got[k].astype(np.float64)
        b = want[k].astype(np.float64)
        worst = max(worst, float((np.abs(a - b) - atol_of(b)).max()))
    return worst


def _step_against_reference(cuda, n, params_host, cams, images, pix, img, oracle_sub):
    """Both arms on identical inputs, compared stage by stage (forward, backward, TV + Adam)."""
    import torch

    import cpx
    import orc
    import refharness as R

    ref = R.RefScene(n, n, n, 9, 2, 0.5, params_host)
    ref.optimizer_init()
    ref.rays_init(cams, img, img, images, pix, True)
    nr = ref.n_rays
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(params_host)
    rays = cpx.Rays(nr)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cams], images, pix, img, img)
    try:
        # ray set-up (_rays::initialSelf, Rays.cu:187-240)
        got, want = rays.download(), ref.rays_download()
        for k in ("ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b"):
            assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), k

        # forward (renderRays)
        ref.render_forward(0, nr)
        rf = ref.rays_download()
        cpx.RenderUtils.renderRays(rays, scene)
        scene.check()
        fwd = rays.download(fields=cpx.RAY_OUTPUTS)
        counts = scene.last_sample_counts(nr)
        assert np.array_equal(fwd["acc_density"].view(np.uint32), rf["acc_density"].view(np.uint32))
        assert np.array_equal(fwd["acc_weights"].view(np.uint32), rf["acc_weights"].view(np.uint32))
        for c in "rgb":
            assert np.abs(fwd[f"acc_{c}"] - rf[f"acc_{c}"]).max() <= RGB_ABS
        osc = orc.Scene(n, n, n, 9, params_host, step=0.5)
        orays = orc.RaySet(oracle_sub.size, True, **{k: got[k][oracle_sub] for k in (
            "ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b")})
        assert np.array_equal(orc.render_forward(osc, orays), counts[oracle_sub])
        del osc, orays

        # backward (renderRays_withGradients_RGB)
        ref_losses = ref.render_backward(0, nr, MASK_COEF, HUBER)
        ref_grads = ref.grads()
        losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
        cpx.RenderUtils.renderRays_withGradients_RGB(scene, rays, losses, maskRayLossCoefficient=MASK_COEF,
                                                     huberDelta=HUBER)
        scene.check()
        assert np.abs(losses.cpu().numpy() - ref_losses).max() <= 255 * RGB_ABS
        grads = scene.download_grads()
        report = grad_report(grads, ref_grads)
        print("per-array gradient error (array, normwise, elementwise above floor, n):",
              [(k, f"{a:.2e}", f"{b:.2e}", m) for k, a, b, m in report])
        assert_grads_close(grads, ref_grads)
        del grads

        # the whole step, each arm on its own gradients (addVarianceLoss + updateRGBScene)
        ref.tv(LAM, LAM, 0, 6)
        ref.adam(LR, SH_LR, 1)
        p_ref = ref.params()
        m_ref, v_ref = ref.moments()
        cpx.Optimizer.varianceAndUpdate(scene, LAM, LAM, LR, SH_LR, 1)
        ulps = 4 * np.spacing(np.float32(np.abs(params_host).max()))
        p = scene.download_params()
        moved_same = np.mean([np.isclose(p[k], p_ref[k], rtol=0, atol=1e-4 * SH_LR + ulps).mean()
                              for k in range(p.shape[0])])
        assert moved_same > 0.999, moved_same
        m, _ = scene.download_moments()
        assert_grads_close(m, m_ref, what="first moment")
        del p, m

        # TV + Adam alone: our fused sweep fed the reference's gradients
        scene.upload_params(params_host)
        zeros = np.zeros_like(params_host)
        scene.upload_moments(zeros, zeros)
        del zeros
        scene.upload_grads(ref_grads)
        cpx.Optimizer.varianceAndUpdate(scene, LAM, LAM, LR, SH_LR, 1)
        p = scene.download_params()
        assert _rows_close(p, p_ref, lambda b: 1e-6 * LR + ulps) <= 0.0
        del p
        m, v = scene.download_moments()
        m_top, v_top = np.abs(m_ref).max(), np.abs(v_ref).max()
        assert _rows_close(m, m_ref, lambda b: 1e-6 * m_top) <= 0.0
        assert _rows_close(v, v_ref, lambda b: 1e-6 * v_top) <= 0.0
        return nr, counts
    finally:
        ref.close()
        scene.close()
        rays.close()


@pytest.mark.skipif("not _ref_available()")
def test_plain128_training_step_against_reference(cuda):
    import cpx_scenes as S

    cfg = S.small_config(seed=0)
    n = cfg["W"]
    nr, counts = _step_against_reference(cuda, n, cfg["params"], cfg["cams"], cfg["images"], cfg["pix"],
                                         cfg["img_w"], np.arange(0, 4096, 8))
    assert nr == 4096 and counts.mean() > 100


@pytest.mark.skipif("not _ref_available()")
def test_plain256_subsample_training_step_against_reference(cuda):
    import torch

    import cpx_scenes as S

    n, img, n_cams, n_rays = 256, 800, 16, 512
    rng = np.random.default_rng(21)
    c, s, p = S.random_blobs(rng, 64)
    dens = S.blob_density(n, n, n, c, s, p, device=cuda) * 0.6
    params = torch.empty((28, n ** 3), dtype=torch.float32, device=cuda)
    params[0] = dens
    params[1:].normal_(0.0, 0.3, generator=torch.Generator(device=cuda).manual_seed(3))
    host = params.cpu().numpy()
    del params, dens
    eyes = S.upper_hemisphere(n_cams, 4.0, rng)
    cams = [S.look_at_camera(e, n, img, img) for e in eyes]
    images = [tuple(rng.integers(0, 256, img * img, dtype=np.uint8) for _ in range(3)) +
              (np.full(img * img, 255, np.uint8),) for _ in range(n_cams)]
    pix = S.sample_pixels(rng, n_cams, img, img, n_rays)
    nr, counts = _step_against_reference(cuda, n, host, cams, images, pix, img, np.arange(0, n_rays, 16))
    assert nr == n_rays and counts.mean() > 200
