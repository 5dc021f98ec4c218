"""Parity of the CUDA path (through the C ABI) with the oracle and with the reference.

Tolerances (stated by the hot-path contract): rendered RGB within 1e-5 absolute,
density and SH gradients within 1e-4 relative (per parameter array, normwise and
elementwise above a floor: tests/tolerances.py), ray/AABB hits, sample counts and
occupancy index lists bit-exact.  Against the
reference's own kernels on the same GPU (same libm), the accumulated density and
weight of every ray are bit-exact too."""
import numpy as np
import pytest

from tolerances import RGB_ABS, assert_grads_close, normwise

pytestmark = pytest.mark.gpu

MASK_COEF = 1.0
HUBER = 0.1


def build(cfg, sparse_threshold=None):
    """Our grid + rays and the oracle's, from one synthetic config."""
    import cpx
    import orc

    n, sh = cfg["W"], cfg["sh_dim"]
    scene = cpx.ObjectScene(n, n, n, sh, step_size=cfg["step"])
    scene.upload_params(cfg["params"])
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr, white_bg=True)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                      cfg["img_w"], cfg["img_h"])
    orays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, orays, off)
        off += len(pix)
    if sparse_threshold is None:
        osc = orc.Scene(n, n, n, sh, cfg["params"], step=cfg["step"])
    else:
        occ, cage, idx, cnt = scene.prune_self(sparse_threshold)
        scene.make_sparse()
        comp = orc.compact(cfg["params"], cage, cnt)
        osc = orc.Scene(n, n, n, sh, comp, step=cfg["step"], sparse=True, occ=occ, index_offsets=idx,
                        in_cage=cage)
    return scene, rays, osc, orays


@pytest.fixture(scope="module")
def plain128(cuda):
    import cpx_scenes as S

    cfg = S.small_config(seed=0)
    scene, rays, osc, orays = build(cfg)
    return cfg, scene, rays, osc, orays


def test_rays_bit_exact(plain128):
    cfg, scene, rays, osc, orays = plain128
    got = rays.download()
    for k, ok in (("ox", "ox"), ("oy", "oy"), ("oz", "oz"), ("dx", "dx"), ("dy", "dy"), ("dz", "dz"),
                  ("near", "near_t"), ("far", "far_t"), ("mask", "mask"), ("r", "r"), ("g", "g"), ("b", "b")):
        assert np.array_equal(got[k].view(np.uint8), orays[ok].view(np.uint8)), k


def test_forward_matches_oracle(plain128):
    import cpx
    import orc

    cfg, scene, rays, osc, orays = plain128
    nr = rays.total_rays
    cpx.RenderUtils.renderRays(rays, scene)
    scene.check()
    counts = scene.last_sample_counts(nr)
    ocounts = orc.render_forward(osc, orays)
    assert np.array_equal(counts, ocounts)
    assert counts.mean() > 100
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    assert np.abs(out["acc_density"] - orays["acc_den"]).max() <= 1e-5 * np.abs(orays["acc_den"]).max()
    assert np.abs(out["acc_weights"] - orays["acc_w"]).max() <= 1e-5
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - orays[f"acc_{c}"]).max() <= RGB_ABS


def test_backward_matches_oracle(plain128, cuda):
    import cpx
    import orc
    import torch

    cfg, scene, rays, osc, orays = plain128
    nr = rays.total_rays
    cpx.RenderUtils.renderRays(rays, scene)
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    for k, ok in (("acc_density", "acc_den"), ("acc_weights", "acc_w"), ("acc_r", "acc_r"), ("acc_g", "acc_g"),
                  ("acc_b", "acc_b")):
        orays.a[ok][:] = out[k]  # the oracle backward reads the same forward outputs
    scene.upload_grads(np.zeros((28, scene.actual_grid_nums), np.float32))
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_withGradients_RGB(scene, rays, losses, maskRayLossCoefficient=MASK_COEF,
                                                 huberDelta=HUBER)
    scene.check()
    grads = scene.download_grads()
    ol, og, oc = orc.render_backward(osc, orays, MASK_COEF, HUBER)
    assert np.array_equal(scene.last_sample_counts(nr), oc)
    assert np.abs(losses.cpu().numpy() - ol).max() <= 255 * RGB_ABS
    assert_grads_close(grads, og)


def test_fused_forward_backward_equals_separate(plain128, cuda):
    import cpx
    import torch

    cfg, scene, rays, osc, orays = plain128
    nr = rays.total_rays
    zero = np.zeros((28, scene.actual_grid_nums), np.float32)
    l1 = torch.zeros(nr, dtype=torch.float64, device=cuda)
    l2 = torch.zeros_like(l1)
    scene.upload_grads(zero)
    cpx.RenderUtils.renderRays(rays, scene)
    cpx.RenderUtils.renderRays_withGradients_RGB(scene, rays, l1, maskRayLossCoefficient=MASK_COEF, huberDelta=HUBER)
    out1 = rays.download(fields=cpx.RAY_OUTPUTS)
    g1 = scene.download_grads()
    scene.upload_grads(zero)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, l2, maskRayLossCoefficient=MASK_COEF, huberDelta=HUBER)
    out2 = rays.download(fields=cpx.RAY_OUTPUTS)
    g2 = scene.download_grads()
    assert torch.equal(l1, l2)
    for k in out1:
        assert np.array_equal(out1[k], out2[k])
    assert_grads_close(g2, g1, rel=1e-5)  # atomic accumulation order only


def test_fused_march_equals_two_stage(plain128, cuda):
    """The fused march (placement and shading overlapped in one launch) and the two-launch
    march give the same forward outputs bit for bit, and gradients equal up to the order of
    the float atomics."""
    import cpx
    import torch

    cfg, scene, rays, osc, orays = plain128
    nr = rays.total_rays
    zero = np.zeros((28, scene.actual_grid_nums), np.float32)
    outs = []
    for opt in (cpx.OPT_FUSED_MARCH, 0):
        scene.set_options(opt)
        losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
        scene.upload_grads(zero)
        cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=MASK_COEF,
                                                   huberDelta=HUBER)
        scene.check()
        outs.append((rays.download(fields=cpx.RAY_OUTPUTS), losses.cpu().numpy(), scene.download_grads(),
                     scene.last_sample_counts(nr)))
    scene.set_options(0)
    (o1, l1, g1, c1), (o2, l2, g2, c2) = outs
    assert np.array_equal(c1, c2)
    for k in o1:
        assert np.array_equal(o1[k].view(np.uint32), o2[k].view(np.uint32)), k
    assert np.array_equal(l1, l2)
    assert_grads_close(g1, g2, rel=1e-5)


@pytest.mark.parametrize("typ,nb", [(0, 6), (0, 3), (0, 26), (1, 6), (2, 6)])
def test_tv_matches_oracle(plain128, typ, nb):
    import cpx
    import orc

    cfg, scene, rays, osc, orays = plain128
    rng = np.random.default_rng(7)
    g0 = rng.normal(0, 1e-3, (28, scene.actual_grid_nums)).astype(np.float32)
    scene.upload_grads(g0)
    cpx.RenderUtils.addVarianceLoss(scene, 1e-3, 2e-3, typ, nb)
    got = scene.download_grads()
    want = g0.copy()
    orc.tv_grad(osc, want, 1e-3, 2e-3, typ, nb)
    # type 0 is a deterministic per-vertex sum; types 1 and 2 add each cell's share to its corners
    # with float atomics, whose order varies
    assert_grads_close(got - g0, want - g0, rel=1e-5 if typ == 0 else 1e-4, what="TV gradient")


def test_adam_matches_oracle(plain128):
    import cpx
    import orc

    cfg, scene, rays, osc, orays = plain128
    n = scene.actual_grid_nums
    rng = np.random.default_rng(8)
    g0 = rng.normal(0, 1e-2, (28, n)).astype(np.float32)
    m0 = rng.normal(0, 1e-3, (28, n)).astype(np.float32)
    v0 = rng.uniform(0, 1e-4, (28, n)).astype(np.float32)
    alr = (rng.random(n) > 0.1).astype(np.float32)
    for fused in (False, True):
        scene.upload_params(cfg["params"])
        scene.upload_grads(g0)
        scene.upload_moments(m0, v0)
        scene.set_adaptive_lr(alr)
        if fused:
            cpx.Optimizer.varianceAndUpdate(scene, 1e-3, 2e-3, 0.1, 0.01, 7)
        else:
            cpx.Optimizer.updateRGBScene(scene, 0.1, 0.01, 7)
        p = scene.download_params()
        m, v = scene.download_moments()
        g = scene.download_grads()
        o = orc.Scene(cfg["W"], cfg["H"], cfg["D"], 9, cfg["params"], step=0.5, adaptive_lr=alr)
        og, om, ov = g0.copy(), m0.copy(), v0.copy()
        if fused:
            orc.tv_grad(o, og, 1e-3, 2e-3, 0, 6)
        orc.adam(o, og, om, ov, 0.1, 0.01, 7)
        step_want = o.params - cfg["params"]
        assert np.abs(p - o.params).max() <= 1e-6 * np.abs(step_want).max() + 4 * np.spacing(np.float32(60.0))
        assert normwise(m, om) <= 1e-6 and normwise(v, ov) <= 1e-6
        assert not g.any()
        assert np.all(p[0] >= 0)
    scene.set_adaptive_lr(np.ones(n, np.float32))
    scene.upload_params(cfg["params"])


def test_occupancy_and_sparse_march_match_oracle(cuda):
    import cpx
    import cpx_scenes as S
    import orc
    import torch

    cfg = S.small_config(seed=4, n=96, n_cams=8, img=160, n_rays=2048)
    scene, rays, osc, orays = build(cfg, sparse_threshold=8.0)
    occ, cage, idx, cnt, _ = orc.occupancy(cfg["params"][0], 96, 96, 96, 8.0)
    assert scene.actual_grid_nums == cnt and scene.sparse
    assert np.array_equal(np.asarray(osc.occ), occ) and np.array_equal(np.asarray(osc.index_offsets), idx)
    assert np.array_equal(scene.download_params(), osc.params)
    nr = rays.total_rays
    cpx.RenderUtils.renderRays(rays, scene)
    counts = scene.last_sample_counts(nr)
    assert np.array_equal(counts, orc.render_forward(osc, orays))
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - orays[f"acc_{c}"]).max() <= RGB_ABS
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_withGradients_RGB(scene, rays, losses, maskRayLossCoefficient=MASK_COEF,
                                                 huberDelta=HUBER)
    for k, ok in (("acc_density", "acc_den"), ("acc_weights", "acc_w"), ("acc_r", "acc_r"), ("acc_g", "acc_g"),
                  ("acc_b", "acc_b")):
        orays.a[ok][:] = out[k]
    ol, og, _ = orc.render_backward(osc, orays, MASK_COEF, HUBER)
    g = scene.download_grads()
    assert_grads_close(g, og)
    # TV type 0 on the sparse grid (index 0 reads as the vertex itself) fused with Adam
    g32 = og.astype(np.float32)
    scene.upload_grads(g32)
    cpx.Optimizer.varianceAndUpdate(scene, 1e-3, 1e-3, 0.1, 0.01, 1)
    p = scene.download_params()
    want = g32.copy()
    orc.tv_grad(osc, want, 1e-3, 1e-3, 0, 6)
    orc.adam(osc, want, np.zeros_like(want), np.zeros_like(want), 0.1, 0.01, 1)
    assert np.abs(p - osc.params).max() <= 1e-5 * 0.1 + 4 * np.spacing(np.float32(60.0))


@pytest.mark.parametrize("sh_dim", [1, 4])
def test_lower_sh_bands(cuda, sh_dim):
    import cpx
    import cpx_scenes as S
    import orc
    import torch

    cfg = S.small_config(seed=9, n=48, n_cams=4, img=64, n_rays=512, sh_dim=sh_dim)
    scene, rays, osc, orays = build(cfg)
    nr = rays.total_rays
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=MASK_COEF, huberDelta=HUBER)
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    orc.render_forward(osc, orays)
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - orays[f"acc_{c}"]).max() <= RGB_ABS
    ol, og, _ = orc.render_backward(osc, orays, MASK_COEF, HUBER)
    assert_grads_close(scene.download_grads(), og)


def test_jitter_offsets_match_oracle(cuda):
    """Per-sample offsets (SolidStrategy 0); positions use offset[sample index]."""
    import cpx
    import cpx_scenes as S
    import orc

    cfg = S.small_config(seed=10, n=48, n_cams=4, img=64, n_rays=512)
    scene, rays, _, orays = build(cfg)
    rng = np.random.default_rng(3)
    offs = [rng.normal(0, 0.06, 300) for _ in range(3)]
    scene.set_sample_offsets(*offs)
    osc = orc.Scene(48, 48, 48, 9, cfg["params"], step=0.5, offsets=offs)
    cpx.RenderUtils.renderRays(rays, scene)
    counts = scene.last_sample_counts(rays.total_rays)
    assert np.array_equal(counts, orc.render_forward(osc, orays))
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - orays[f"acc_{c}"]).max() <= RGB_ABS


def test_hierarchy_strategy_restricts_bands(cuda):
    """hierarchyStrategy: gradients and updates only for band `optimizing_band`
    (RenderUtils.cu:1117-1126, Optimizer.cu:394-398)."""
    import cpx
    import cpx_scenes as S
    import orc
    import torch

    cfg = S.small_config(seed=11, n=40, n_cams=4, img=64, n_rays=400)
    n = 40
    scene = cpx.ObjectScene(n, n, n, 9, optimizing_band=1, hierarchy_strategy=True)
    scene.upload_params(cfg["params"])
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"], 64, 64)
    orays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], 64, *img, True, pix, orays, off)
        off += len(pix)
    osc = orc.Scene(n, n, n, 9, cfg["params"], step=0.5, band=1, hierarchy=True)
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=MASK_COEF, huberDelta=HUBER)
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    orc.render_forward(osc, orays)
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - orays[f"acc_{c}"]).max() <= RGB_ABS
    _, og, _ = orc.render_backward(osc, orays, MASK_COEF, HUBER)
    g = scene.download_grads()
    assert_grads_close(g, og)
    k = (np.arange(27) % 9)
    assert not g[1:][(k < 1) | (k >= 4)].any()  # only band 1 (k = 1..3) receives SH gradients


def test_golden_inputs_bit_exact_against_reference(cuda):
    """Our kernels on the inputs of tests/golden/ref_dense.npz: accumulated density and
    weights equal the reference kernels' bit for bit (same GPU, same libm); RGB and
    gradients within tolerance."""
    import cpx
    import make_ref_golden as G
    import torch
    from conftest import GOLDEN

    ref = np.load(GOLDEN / "ref_dense.npz")
    case = G.dense_case()
    n = case["n"]
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(case["params"])
    scene.set_adaptive_lr(case["adaptive"])
    nr = sum(len(p) for p in case["pix"])
    rays = cpx.Rays(nr)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in case["cams"]], case["images"], case["pix"],
                      case["img"], case["img"])
    got = rays.download()
    for k in ("ox", "dx", "dy", "dz", "near", "far", "r", "g", "b", "mask"):
        assert np.array_equal(got[k].view(np.uint8), ref[f"ray_{k}"].view(np.uint8)), k
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=G.MASK_COEF,
                                               huberDelta=G.HUBER)
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    assert np.array_equal(out["acc_density"], ref["fwd_acc_density"])
    assert np.array_equal(out["acc_weights"], ref["fwd_acc_weights"])
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - ref[f"fwd_acc_{c}"]).max() <= RGB_ABS
    assert np.abs(losses.cpu().numpy() - ref["losses"]).max() <= 255 * RGB_ABS
    g = scene.download_grads()
    assert_grads_close(g, ref["grad_bwd"])
    cpx.Optimizer.varianceAndUpdate(scene, 1e-3, 1e-3, 0.1, 0.01, 1)
    p = scene.download_params()
    # at t=1 a parameter moves by ~lr*sign(g): compare where |g| is not at rounding level
    moved_same = np.isclose(p, ref["params_adam"], rtol=0, atol=1e-4 * 0.1 + 4 * np.spacing(np.float32(60.0)))
    assert moved_same.mean() > 0.999


def test_sparse_golden_bit_exact_against_reference(cuda):
    import cpx
    import make_ref_golden as G
    from conftest import GOLDEN

    ref = np.load(GOLDEN / "ref_sparse.npz")
    case = G.sparse_case()
    n = case["n"]
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(case["params"])
    occ, cage, idx, cnt = scene.prune_self(case["threshold"])
    assert np.array_equal(occ, ref["occupancy"]) and np.array_equal(cage, ref["in_cage"])
    assert np.array_equal(idx, ref["index_offsets"]) and cnt == int(ref["in_cage_count"][0])
    scene.make_sparse()
    nr = sum(len(p) for p in case["pix"])
    rays = cpx.Rays(nr)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in case["cams"]], case["images"], case["pix"],
                      case["img"], case["img"])
    cpx.RenderUtils.renderRays(rays, scene)
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    assert np.array_equal(out["acc_density"], ref["fwd_acc_density"])
    assert np.array_equal(out["acc_weights"], ref["fwd_acc_weights"])
    for c in "rgb":
        assert np.abs(out[f"acc_{c}"] - ref[f"fwd_acc_{c}"]).max() <= RGB_ABS


def test_train_step_matches_oracle_step(cuda):
    """One full batch (forward+backward, TV 6, Adam) against the oracle's sequence."""
    import cpx
    import cpx_scenes as S
    import orc
    import torch

    cfg = S.small_config(seed=12, n=64, n_cams=6, img=96, n_rays=1024)
    scene, rays, osc, orays = build(cfg)
    nr = rays.total_rays
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    mse = cpx.train_step(scene, rays, losses, mask_coef=MASK_COEF, huber_delta=HUBER, lam_density=1e-3,
                         lam_sh=1e-3, lr=0.1, sh_lr=0.01, timestep=1)
    p = scene.download_params()
    orc.render_forward(osc, orays)
    ol, og, _ = orc.render_backward(osc, orays, MASK_COEF, HUBER)
    assert abs(mse - orc.mse(ol)) <= 1e-4 * orc.mse(ol)
    g = og.astype(np.float32)
    orc.tv_grad(osc, g, 1e-3, 1e-3, 0, 6)
    orc.adam(osc, g, np.zeros_like(g), np.zeros_like(g), 0.1, 0.01, 1)
    # at t=1 each parameter moves by ~lr*sign(g); a gradient near zero can flip the sign
    # under a 1e-4 relative gradient difference, so compare the moved fraction
    moved_same = np.isclose(p, osc.params, rtol=0, atol=1e-3 * 0.01 + 4 * np.spacing(np.float32(60.0)))
    assert moved_same.mean() > 0.999


def test_edge_cases(cuda):
    import cpx
    import torch

    n = 16
    scene = cpx.ObjectScene(n, n, n, 9)
    params = np.zeros((28, n ** 3), np.float32)
    params[0] = 20.0
    scene.upload_params(params)
    rays = cpx.Rays(4)
    o = np.array([-5.0, 7.5, 7.5], np.float32)
    rays.upload(ox=[o[0]] * 4, oy=[o[1]] * 4, oz=[o[2]] * 4, dx=[1, 1, 1, 1], dy=[0, 0, 0, 0], dz=[0, 0, 0, 0],
                near=[5.0, 9.0, 5.0, 5.0], far=[20.0, 1.0, 20.0, 5.0], mask=[255] * 4, r=[0] * 4, g=[0] * 4,
                b=[0] * 4)
    losses = torch.zeros(4, dtype=torch.float64, device=cuda)
    # empty batch is a no-op
    cpx.RenderUtils.renderRays(rays, scene, len=0)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=1.0, huberDelta=0.1)
    scene.check()
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    counts = scene.last_sample_counts(4)
    assert counts[1] == 0 and out["acc_r"][1] == 0 and losses[1].item() == 0  # near > far: no background
    assert counts[3] == 0 and out["acc_r"][3] == 1.0                         # near == far: background only
    assert counts[0] > 0 and counts[0] == counts[2]
    # NaN parameters: the reference's loss becomes 255 and the ray adds no gradient
    params[0] = np.nan
    scene.upload_params(params)
    scene.upload_grads(np.zeros_like(params))
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=1.0, huberDelta=0.1)
    assert losses[0].item() == 255.0
    # a sample index outside the table is reported, not read
    bad = torch.tensor([0, 7], dtype=torch.int32, device=cuda)
    cpx.RenderUtils.renderRays(rays, scene, sampleIndex=bad, len=2)
    with pytest.raises(cpx.CpxError) as ei:
        scene.check()
    assert ei.value.name == "CPX_ERR_INVALID_ARGUMENT"
    # a ray far longer than the grid box stops at the sample bound and is reported
    params[0] = 0.0
    scene.upload_params(params)
    rays.upload(near=[0.0], far=[1e7])
    cpx.RenderUtils.renderRays(rays, scene, len=1)
    with pytest.raises(cpx.CpxError) as ei:
        scene.check()
    assert ei.value.name == "CPX_ERR_ITERATION_CAP"
    scene.check()  # the flag is cleared once reported
    with pytest.raises(cpx.CpxError):
        cpx.RenderUtils.renderRays(rays, scene, startSampleIndex=2, len=3)  # beyond the table
