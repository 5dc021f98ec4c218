"""The touched-vertex maps: the backward marks the vertices it scatters into and the optimizer
sweep reads and clears gradient records only there.  A grid whose sweeps read every record
(after cpx_grid_upload_grads) must end bit-identical to one that uses the maps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(cfg, precision):
    import cpx

    n = cfg["W"]
    out = []
    for _ in range(2):
        scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"], precision=precision, sr_seed=5)
        scene.upload_params(cfg["params"])
        nr = sum(len(p) for p in cfg["pix"])
        rays = cpx.Rays(nr, white_bg=True)
        rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                          cfg["img_w"], cfg["img_h"])
        out.append((scene, rays))
    return out


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_touched_maps_equal_full_sweeps(cuda, precision):
    """Grid b marches and sweeps with its maps; grid a receives b's gradients by upload (so
    its sweep reads every record) and sweeps too.  The float atomics of the scatter are not
    bit-deterministic across runs, so a takes b's gradients instead of marching itself."""
    import torch

    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=21, n=48, n_cams=6, img=64, n_rays=1536)
    (a, ra), (b, rb) = _pair(cfg, precision)
    nr = rb.total_rays
    n_act = a.actual_grid_nums
    lb = torch.zeros(nr, dtype=torch.float64, device=cuda)
    half = nr // 2
    for t, (s0, ln) in enumerate(((0, half), (half, nr - half), (0, nr)), start=1):
        cpx.RenderUtils.renderRays_forwardBackward(b, rb, lb, None, s0, ln, 1.0, 0.1)
        g = b.download_grads()
        count = b.touched_count()
        marked = np.abs(g).sum(0) != 0
        assert 0 < marked.sum() <= count < n_act
        a.upload_grads(g)
        cpx.Optimizer.varianceAndUpdate(a, 1e-3, 1e-3, 0.1, 0.01, t)
        cpx.Optimizer.varianceAndUpdate(b, 1e-3, 1e-3, 0.1, 0.01, t)
        assert np.array_equal(a.download_params(), b.download_params()), t
    a.check()
    b.check()
    ma, va = a.download_moments()
    mb, vb = b.download_moments()
    assert np.array_equal(ma, mb) and np.array_equal(va, vb)
    assert not b.download_grads().any()
    assert b.touched_count() == 0  # the next batch's map starts clear


def test_standalone_tv_marks_every_vertex(cuda):
    """A standalone TV pass writes gradients of vertices no ray touched: the next sweep must
    read them all."""
    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=22, n=32, n_cams=2, img=32, n_rays=64)
    n = cfg["W"]
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(cfg["params"])
    cpx.RenderUtils.addVarianceLoss(scene, 1e-3, 1e-3, 0, 6)
    assert scene.touched_count() == n ** 3
    g = scene.download_grads()
    assert g.any()
    cpx.Optimizer.updateRGBScene(scene, 0.1, 0.01, 1)
    assert not scene.download_grads().any()


@pytest.mark.parametrize("dims", [(37, 45, 70), (16, 8, 33), (64, 64, 64)])
def test_plane_window_sweep_equals_row_sweep(cuda, dims):
    """The FP32 dense sweep that walks z with a tile's x-y plane on chip and the sweep that runs a
    block per row give the same parameters, moments and gradients bit for bit, two steps in a
    row, on grids whose sides are not multiples of the 16 x 8 tile or of the 32-plane z chunk,
    with an adaptive learning rate.  (Sweeps that read gradients through the touched maps equal
    sweeps that read every record: test_touched_maps_equal_full_sweeps.)"""
    import cpx
    import cpx_scenes as S

    W, H, D = dims
    rng = np.random.default_rng(W * 131 + D)
    params = S.make_params(rng.uniform(0.0, 30.0, W * H * D).astype(np.float32), 9, rng, 0.3)
    grads = [rng.normal(0, 1e-2, params.shape).astype(np.float32) for _ in range(2)]
    m0 = rng.normal(0, 1e-3, params.shape).astype(np.float32)
    v0 = rng.uniform(0, 1e-4, params.shape).astype(np.float32)
    alr = (rng.random(W * H * D) > 0.2).astype(np.float32)
    outs = []
    for opt in (cpx.OPT_PLANE_SWEEP, 0):
        sc = cpx.ObjectScene(W, H, D, 9)
        sc.set_options(opt)
        sc.upload_params(params)
        sc.set_adaptive_lr(alr)
        sc.upload_moments(m0, v0)
        res = []
        for t, g in enumerate(grads):
            sc.upload_grads(g)
            cpx.Optimizer.varianceAndUpdate(sc, 1e-3, 2e-3, 0.3, 1.0, 4 + t)
            res += [sc.download_params(), *sc.download_moments(), sc.download_grads()]
        sc.check()
        outs.append(res)
        sc.close()
    assert not np.array_equal(outs[0][0], params)
    for a, b in zip(*outs):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_split_sweep_trains_as_the_single_sweep(cuda):
    """CPX_OPT_SPLIT_SWEEP: the vertices no placed sample reaches are swept beside the shading
    and the rest after it.  Four training steps match the single sweep's: the first step's batch
    MSE exactly (same parameters before it), the parameters and moments after the fourth within
    float-atomics noise on 99.9% of the values."""
    import torch

    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=43, n=48, n_cams=6, img=64, n_rays=2048)
    n = cfg["W"]
    step = dict(mask_coef=1.0, huber_delta=0.1, lam_density=1e-4, lam_sh=1e-5, lr=0.05, sh_lr=0.2)
    runs = []
    for opt in (cpx.OPT_SPLIT_SWEEP, 0):
        scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"])
        scene.set_options(opt)
        scene.upload_params(cfg["params"])
        rays = cpx.Rays(2048, white_bg=True)
        rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                          cfg["img_w"], cfg["img_h"])
        losses = torch.zeros(512, dtype=torch.float64, device=cuda)
        mses = []
        for k in range(4):
            mses.append(cpx.train_step(scene, rays, losses, start=(k % 4) * 512, length=512, timestep=k + 1, **step))
        scene.check()
        runs.append((mses, scene.download_params(), *scene.download_moments()))
        scene.close()
        rays.close()
    (ms, ps, ms1, vs), (mp, pp, mp1, vp) = runs
    assert ms[0] == mp[0]
    assert all(abs(a - b) <= 1e-4 * b for a, b in zip(ms, mp))
    assert not np.array_equal(pp, cfg["params"])
    for got, want, tol in ((ps, pp, 1e-4 * step["lr"]), (ms1, mp1, 1e-6), (vs, vp, 1e-9)):
        assert np.mean(np.abs(got - want) <= tol + 1e-4 * np.abs(want)) >= 0.999
