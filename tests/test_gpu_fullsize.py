"""Properties of the CUDA path at the full plain-FP32 size (256^3 grid, SH band 2,
8192-ray batches from 800x800 views), where the oracle cannot run the whole batch:
a ray subsample is checked against the oracle, the rest through size-independent
properties (determinism, the provable sample bound, the sweep's update formula)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 256
R = 8192


@pytest.fixture(scope="module")
def big(cuda):
    import torch

    import cpx
    import cpx_scenes as S

    rng = np.random.default_rng(21)
    c, s, p = S.random_blobs(rng, 64)
    params = torch.empty((28, N ** 3), dtype=torch.float32, device=cuda)
    params[0] = S.blob_density(N, N, N, c, s, p, device=cuda) * 0.6
    params[1:].normal_(0.0, 0.3, generator=torch.Generator(device=cuda).manual_seed(3))
    scene = cpx.ObjectScene(N, N, N, 9)
    scene.upload_params_device(params)
    eyes = S.upper_hemisphere(100, 4.0, rng)
    pix = S.sample_pixels(rng, 100, 800, 800, R)
    imgs = [tuple(rng.integers(0, 256, 640000, dtype=np.uint8) for _ in range(3)) + (None,) for _ in range(100)]
    rays = cpx.Rays(R)
    rays.initial_self(scene, [cpx.Camera.make(**S.look_at_camera(e, N, 800, 800)) for e in eyes], imgs, pix, 800, 800)
    host = params.cpu().numpy()
    return scene, rays, host


def test_forward_is_deterministic_and_bounded(big):
    import cpx

    scene, rays, _ = big
    cpx.RenderUtils.renderRays(rays, scene)
    c1 = scene.last_sample_counts(R)
    o1 = rays.download(fields=cpx.RAY_OUTPUTS)
    cpx.RenderUtils.renderRays(rays, scene)
    scene.check()
    c2 = scene.last_sample_counts(R)
    o2 = rays.download(fields=cpx.RAY_OUTPUTS)
    assert np.array_equal(c1, c2)
    for k in o1:
        assert np.array_equal(o1[k], o2[k])
    geo = rays.download(fields=("near", "far"))
    bound = np.floor((geo["far"].astype(np.float64) - geo["near"] + 1.0) / 0.5) + 2
    hit = geo["near"] <= geo["far"]
    assert np.all(c1[hit] <= bound[hit]) and c1.mean() > 200


def test_ray_subsample_matches_oracle(big, cuda):
    import torch

    import cpx
    import orc

    scene, rays, host = big
    losses = torch.zeros(R, dtype=torch.float64, device=cuda)
    scene.upload_grads(np.zeros_like(host))
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=1.0, huberDelta=0.1)
    counts = scene.last_sample_counts(R)
    out = rays.download()
    sub = np.arange(0, R, 64)  # 128 rays
    orays = orc.RaySet(sub.size, True, **{k: out[k][sub] for k in ("ox", "oy", "oz", "dx", "dy", "dz", "near",
                                                                   "far", "mask", "r", "g", "b")})
    osc = orc.Scene(N, N, N, 9, host, step=0.5)
    oc = orc.render_forward(osc, orays)
    assert np.array_equal(oc, counts[sub])
    for c in "rgb":
        assert np.abs(orays[f"acc_{c}"] - out[f"acc_{c}"][sub]).max() <= 1e-5
    assert np.abs(orays["acc_w"] - out["acc_weights"][sub]).max() <= 1e-5
    ol, _, _ = orc.render_backward(osc, orays, 1.0, 0.1)
    assert np.abs(ol - losses.cpu().numpy()[sub]).max() <= 255e-5


def test_sweep_update_formula_on_sampled_vertices(big):
    """Adam with TV off: every updated parameter follows Optimizer.cu:374-413 exactly in form."""
    import cpx

    scene, rays, host = big
    rng = np.random.default_rng(5)
    g = rng.normal(0, 1e-2, host.shape).astype(np.float32)
    m = rng.normal(0, 1e-3, host.shape).astype(np.float32)
    v = rng.uniform(0, 1e-4, host.shape).astype(np.float32)
    scene.upload_params(host)
    scene.upload_grads(g)
    scene.upload_moments(m, v)
    t = 9
    cpx.Optimizer.updateRGBScene(scene, 0.3, 1.0, t)
    p1 = scene.download_params()
    m1, v1 = scene.download_moments()
    assert not scene.download_grads().any()
    idx = rng.integers(0, N ** 3, 20000)
    gd, md, vd, pd = (a[:, idx].astype(np.float64) for a in (g, m, v, host))
    mm = 0.9 * md + 0.1 * gd
    vv = 0.999 * vd + 0.001 * gd * gd
    lr = np.array([0.3] + [1.0] * 27)[:, None]
    step = lr * (mm / (1 - 0.9 ** t)) / (np.sqrt(vv / (1 - 0.999 ** t)) + 1e-6)
    want = pd - step
    want[0] = np.maximum(want[0], 0)
    assert np.abs(m1[:, idx] - mm).max() <= 1e-6 * np.abs(mm).max()
    assert np.abs(v1[:, idx] - vv).max() <= 1e-6 * np.abs(vv).max()
    assert np.abs(p1[:, idx] - want).max() <= 1e-5 * np.abs(step).max() + 4 * np.spacing(np.float32(64))
    scene.upload_params(host)
    scene.upload_moments(np.zeros_like(host), np.zeros_like(host))


def test_fused_tv_adam_equals_tv_then_adam(big):
    import cpx

    scene, rays, host = big
    rng = np.random.default_rng(6)
    g = rng.normal(0, 1e-3, host.shape).astype(np.float32)
    outs = []
    for fused in (True, False):
        scene.upload_params(host)
        scene.upload_grads(g)
        scene.upload_moments(np.zeros_like(host), np.zeros_like(host))
        if fused:
            cpx.Optimizer.varianceAndUpdate(scene, 1e-4, 1e-5, 0.3, 1.0, 3)
        else:
            cpx.RenderUtils.addVarianceLoss(scene, 1e-4, 1e-5, 0, 6)
            cpx.Optimizer.updateRGBScene(scene, 0.3, 1.0, 3)
        outs.append(scene.download_params())
    d = np.abs(outs[0] - outs[1])
    assert (d <= 1e-6 + 4 * np.spacing(np.float32(64))).mean() > 0.9999
    scene.upload_params(host)
