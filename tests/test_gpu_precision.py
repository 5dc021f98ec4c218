"""The mixed storage forms (16-bit SH and Adam moments, FP32 density, gradients and march,
stochastic rounding) against the FP64 host oracle, and against the FP32 form.

Error bounds written here: with SH values that bfloat16 represents exactly, the FP32 march
agrees with the FP64 oracle to 1e-4 in colour and 2e-3 normwise in the gradients (the march
itself is the only difference); with arbitrary values the SH rounding adds at most 4e-3
(bfloat16) / 1e-3 (half) to the colour.  Set CPX_REPORT_DIR to write the error table."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASK_COEF = 1.0
HUBER = 0.1


def bf16_rn(x):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (b.astype(np.uint32) << 16).view(np.float32)


def to_storage(params, precision):
    """The parameter values a grid of `precision` holds after an upload of `params`."""
    out = np.array(params, np.float32, copy=True)
    if precision == "bf16":
        out[1:] = bf16_rn(out[1:])
    elif precision == "fp16":
        out[1:] = out[1:].astype(np.float16).astype(np.float32)
    return out


def make(cfg, precision, params=None, sparse_threshold=None):
    import cpx

    n = cfg["W"]
    scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"], precision=precision, sr_seed=7)
    scene.upload_params(cfg["params"] if params is None else params)
    scene.occupancy_tables = None
    if sparse_threshold is not None:
        scene.occupancy_tables = scene.prune_self(sparse_threshold)
        scene.make_sparse()
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr, white_bg=True)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                      cfg["img_w"], cfg["img_h"])
    return scene, rays


def oracle(cfg, params):
    """The oracle's dense scene of `params` and its copy of the rays (bit-exact with ours)."""
    import orc

    n = cfg["W"]
    nr = sum(len(p) for p in cfg["pix"])
    orays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, orays, off)
        off += len(pix)
    return orc.Scene(n, n, n, 9, params, step=cfg["step"]), orays


def normwise(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def run_fb(scene, rays):
    import torch

    import cpx

    nr = rays.total_rays
    losses = torch.zeros(nr, dtype=torch.float64, device="cuda")
    scene.upload_grads(np.zeros((28, scene.actual_grid_nums), np.float32))
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, maskRayLossCoefficient=MASK_COEF,
                                               huberDelta=HUBER)
    scene.check()
    out = rays.download(fields=cpx.RAY_OUTPUTS)
    pred = np.stack([out["acc_r"], out["acc_g"], out["acc_b"]], 1)
    return pred, out["acc_weights"], losses.cpu().numpy(), scene.download_grads()


@pytest.fixture(scope="module")
def case():
    import cpx_scenes as S

    return S.small_config(seed=11, n=64, n_cams=8, img=96, n_rays=2048)


def moments_storage(m, v, precision):
    """The moments a grid of `precision` holds after an upload of (m, v): bfloat16 (nearest), or
    for "fp16full" half of m * 2^8 and of sqrt(v) * 2^8 (nearest), read back as m and v."""
    if precision != "fp16full":
        return bf16_rn(m), bf16_rn(v)
    k = np.float32(256.0)
    hm = (np.asarray(m, np.float32) * k).astype(np.float16).astype(np.float32) / k
    r = (np.sqrt(np.asarray(v, np.float32)) * k).astype(np.float16).astype(np.float32) / k
    return hm, (r * r).astype(np.float32)


@pytest.mark.parametrize("precision", ["bf16", "fp16", "fp16full"])
def test_upload_rounds_to_nearest_and_downloads_exactly(cuda, case, precision):
    import cpx

    n = case["W"]
    scene = cpx.ObjectScene(n, n, n, 9, precision=precision)
    scene.upload_params(case["params"])
    got = scene.download_params()
    assert np.array_equal(got, to_storage(case["params"], "fp16" if precision == "fp16full" else precision))
    m = np.random.default_rng(0).normal(0, 1e-3, case["params"].shape).astype(np.float32)
    v = (m * m).astype(np.float32)
    scene.upload_moments(m, v)
    gm, gv = scene.download_moments()
    wm, wv = moments_storage(m, v, precision)
    assert np.array_equal(gm, wm) and np.array_equal(gv, wv)


def test_half_moments_hold_adam_closer_than_bfloat16(cuda):
    """Thirty Adam steps on the same gradient sequence (no TV) in the three 16-bit forms against
    FP64 Adam from the same starting values, gradients spanning 1e-6 .. 1e-1.  Moment errors
    are measured against the gradient scale sqrt(v) (what Adam divides by): the half-moment form
    ("fp16full") keeps both moments within a few half ulps (median below 2^-10, 99th percentile
    below 2^-7), the first moment at least 4x and the second at least 3x closer than the bfloat16
    moments of "bf16" and "fp16" (bfloat16 holds v itself, whose relative error is twice its
    root's, so the root gains less from half's three extra mantissa bits); every
    form's parameters stay within its 16-bit storage error of FP64 Adam (stochastic rounding
    at each of the 30 write-backs: a random walk of a few ulps)."""
    import cpx

    n = 32
    rng = np.random.default_rng(5)
    params = rng.normal(0.0, 0.3, (28, n ** 3)).astype(np.float32)
    params[0] = np.abs(params[0]) + 0.5
    scale = 10.0 ** rng.uniform(-6, -1, (28, n ** 3))
    grads = [(rng.normal(0.0, 1.0, (28, n ** 3)) * scale).astype(np.float32) for _ in range(30)]
    lr, sh_lr = 1e-2, 1e-3
    rel = {}
    for precision in ("bf16", "fp16", "fp16full"):
        p64 = to_storage(params, "fp16" if precision == "fp16full" else precision).astype(np.float64)
        m64 = np.zeros_like(p64)
        v64 = np.zeros_like(p64)
        lrs = np.array([[lr]] + [[sh_lr]] * 27)
        for t, g in enumerate(grads, start=1):
            g = g.astype(np.float64)
            m64 = 0.9 * m64 + 0.1 * g
            v64 = 0.999 * v64 + 0.001 * g * g
            p64 = p64 - lrs * (m64 / (1 - 0.9 ** t)) / (np.sqrt(v64 / (1 - 0.999 ** t)) + 1e-6)
            p64[0] = np.maximum(p64[0], 0.0)
        scene = cpx.ObjectScene(n, n, n, 9, precision=precision, sr_seed=9)
        scene.upload_params(params)
        for t, g in enumerate(grads, start=1):
            scene.upload_grads(g)
            cpx.Optimizer.updateRGBScene(scene, lr, sh_lr, timeStep=t)
        m, v = scene.download_moments()
        post = scene.download_params()
        scene.close()
        s64 = np.sqrt(v64)
        em = np.abs(m - m64) / s64
        ev = np.abs(np.sqrt(v) - s64) / s64
        rel[precision] = (float(np.median(em)), float(np.percentile(em, 99)), float(np.median(ev)),
                          float(np.percentile(ev, 99)))
        u = 2.0 ** -7 if precision == "bf16" else 2.0 ** -10  # 16-bit spacing of |p| in [1, 2)
        err = np.abs(post[1:] - p64[1:])
        assert err.max() < 20 * u + 30 * sh_lr * 0.05 and err.mean() < 4 * u, (precision, err.max(), err.mean())
        assert np.abs(post[0] - p64[0]).max() < 30 * lr * 0.05, precision
    med_m, p99_m, med_v, p99_v = rel["fp16full"]
    assert med_m < 2.0 ** -10 and p99_m < 2.0 ** -7 and med_v < 2.0 ** -10 and p99_v < 2.0 ** -7, rel
    for other in ("bf16", "fp16"):
        assert med_m < rel[other][0] / 4 and med_v < rel[other][2] / 3, rel


@pytest.mark.parametrize("precision", ["bf16", "fp16", "fp16full"])
def test_fp32_march_against_fp64_oracle(cuda, case, precision):
    """SH values exactly representable in 16 bits: the remaining difference to the FP64
    oracle is the FP32 march alone (the oracle marching as the FP32 march does: empty cells
    at the density clamp jumped, rays ended below transmittance 1e-4)."""
    import orc

    params = to_storage(case["params"], "fp16" if precision == "fp16full" else precision)
    scene, rays = make(case, precision, params)
    pred, accw, losses, grad = run_fb(scene, rays)
    osc, orays = oracle(case, params)
    pred64, accw64, losses64, grad64, _ = orc.fp64_step(osc, orays, MASK_COEF, HUBER, skip_empty=True,
                                                        t_stop=orc.MIXED_T_STOP)
    assert np.abs(pred - pred64).max() < 1e-4
    assert np.abs(accw - accw64).max() < 1e-4
    assert normwise(grad[0], grad64[0]) < 2e-3
    assert normwise(grad[1:], grad64[1:]) < 2e-3


def test_mixed_image_equals_fp32_image_of_rounded_values(cuda, case):
    """The image path reads 16-bit SH exactly: a BF16 grid renders the same bytes as an FP32
    grid holding the bfloat16-rounded values."""
    import cpx

    params = to_storage(case["params"], "bf16")
    n = case["W"]
    a = cpx.ObjectScene(n, n, n, 9, precision="bf16")
    a.upload_params(case["params"])
    b = cpx.ObjectScene(n, n, n, 9)
    b.upload_params(params)
    cam = cpx.Camera.make(**case["cams"][0])
    ia = cpx.RenderUtils.renderImage(a, cam, 96, 96)
    ib = cpx.RenderUtils.renderImage(b, cam, 96, 96)
    for k in ("rgb", "rgb8", "depth", "mask"):
        assert np.array_equal(ia[k].cpu().numpy(), ib[k].cpu().numpy()), k


def test_stochastic_rounding_keeps_small_steps(cuda):
    """Adam steps far below half a bfloat16 spacing survive on average: 27 x 2^18 SH values at
    1.0 get one step of 1e-4 (bfloat16 numbers just below 1.0 are 2^-8 apart); the mean lands
    at 1 - 1e-4 within 4 sigma."""
    import cpx

    n = 64
    scene = cpx.ObjectScene(n, n, n, 9, precision="bf16", sr_seed=3)
    params = np.ones((28, n ** 3), np.float32)
    scene.upload_params(params)
    scene.upload_grads(np.ones((28, n ** 3), np.float32))
    cpx.Optimizer.updateRGBScene(scene, 0.1, 1e-4, timeStep=1)
    got = scene.download_params()[1:].astype(np.float64)
    vals = np.unique(got)
    assert set(vals.tolist()) <= {1.0, 1.0 - 2.0 ** -8}  # the two neighbours below 1.0 and 1.0
    p = 1e-4 / 2.0 ** -8
    sigma = 2.0 ** -8 * np.sqrt(p * (1 - p) / got.size)
    assert abs(got.mean() - (1.0 - 1e-4)) < 4 * sigma
    # the same step rounded to nearest would leave every value at 1.0
    assert (got < 1.0).mean() > 0.5 * p


@pytest.mark.parametrize("precision", ["bf16", "fp16", "fp16full"])
def test_step_errors_against_fp64_oracle(cuda, case, precision):
    """One full batch (forward, backward, TV type 0 / 6, Adam) on arbitrary values: the error
    table of the mixed form and of the FP32 form against the FP64 oracle."""
    import orc

    import cpx

    params = case["params"]
    osc, orays = oracle(case, params)
    lam, lr, sh_lr = 1e-3, 0.1, 0.01
    pred64, accw64, losses64, grad64, post64 = orc.fp64_step(osc, orays, MASK_COEF, HUBER, lam_d=lam, lam_sh=lam,
                                                             lr=lr, sh_lr=sh_lr)
    table = {}
    for form in ("fp32", precision):
        scene, rays = make(case, form, params)
        pred, accw, losses, grad = run_fb(scene, rays)
        scene.upload_grads(grad)
        cpx.Optimizer.varianceAndUpdate(scene, lam, lam, lr, sh_lr, 1)
        post = scene.download_params()
        moved = np.abs(post64 - params) > 1e-3 * np.array([[lr]] + [[sh_lr]] * 27)
        # at t = 1 Adam moves a parameter by lr * g / (|g| + 1e-6): where |g| is near the
        # epsilon the step length follows small gradient differences, and where a gradient is
        # at rounding level its sign may differ; the post-step values are compared where the
        # FP64 gradient (with TV) is well above the epsilon and the step directions agree
        g64 = np.abs(post64 - params) >= 0.99 * np.array([[lr]] + [[sh_lr]] * 27)
        agree = (np.sign(post - params) == np.sign(post64 - params)) & g64
        table[form] = {
            "rgb_max_abs": float(np.abs(pred - pred64).max()),
            "rgb_mean_abs": float(np.abs(pred - pred64).mean()),
            "loss_max_abs": float(np.abs(losses - losses64).max()),
            "grad_density_normwise": normwise(grad[0], grad64[0]),
            "grad_sh_normwise": normwise(grad[1:], grad64[1:]),
            "post_density_max_abs": float(np.abs(post[0] - post64[0]).max()),
            "post_sh_max_abs": float(np.abs(post[1:] - post64[1:]).max()),
            "post_sh_max_abs_same_direction": float(np.abs(post[1:] - post64[1:])[agree[1:]].max()),
            "post_sign_agreement": float(np.mean(np.sign(post - params)[moved] == np.sign(post64 - params)[moved])),
        }
    e32, e16 = table["fp32"], table[precision]
    assert e32["rgb_max_abs"] < 2e-5 and e32["grad_sh_normwise"] < 1e-4
    bound = 4e-3 if precision == "bf16" else 1e-3
    assert e16["rgb_max_abs"] < bound
    assert e16["grad_density_normwise"] < 0.05 and e16["grad_sh_normwise"] < 0.05
    # post-step SH: within one 16-bit ulp of the value (|SH| < 2 here) plus the step's error
    assert e16["post_sh_max_abs_same_direction"] < (2.0 ** -6 if precision == "bf16" else 2.0 ** -9) + 1e-3
    assert e16["post_sh_max_abs"] <= 2 * sh_lr + 2.0 ** -6
    assert e16["post_sign_agreement"] > 0.97
    rep = os.environ.get("CPX_REPORT_DIR")
    if rep:
        os.makedirs(rep, exist_ok=True)
        with open(os.path.join(rep, f"precision_errors_{precision}.json"), "w") as f:
            json.dump({"case": "64^3 dense, 2048 rays, seed 11", "errors_vs_fp64": table}, f, indent=1)


def test_sparse_mixed_form_against_fp64_oracle(cuda, case):
    import orc

    params = to_storage(case["params"], "bf16")
    scene, rays = make(case, "bf16", params, sparse_threshold=2.0)
    occ, cage, idx, cnt = scene.occupancy_tables
    n = case["W"]
    comp = orc.compact(params, cage, cnt)
    osc = orc.Scene(n, n, n, 9, comp, step=case["step"], sparse=True, occ=occ, index_offsets=idx, in_cage=cage)
    _, orays = oracle(case, params)
    pred, accw, losses, grad = run_fb(scene, rays)
    # the FP32 march jumps over empty cells and bricks of a sparse grid in whole steps
    pred64, accw64, _, grad64, _ = orc.fp64_step(osc, orays, MASK_COEF, HUBER, skip_empty=True,
                                                   t_stop=orc.MIXED_T_STOP)
    assert np.abs(pred - pred64).max() < 1e-4
    assert normwise(grad[1:], grad64[1:]) < 2e-3


def test_dense_empty_jumps_and_early_stop_against_fp64_oracle(cuda, case):
    """A dense mixed grid whose empty space lies below the empty-density bound: the FP32 march
    jumps over those cells and stops rays behind opaque content, exactly as the FP64 oracle
    with the same map and stop; the march without them (options) is the plain FP32 march, and
    the two differ by less than 5e-4 in colour (1e-4 from the stop, the rest from the skipped
    samples' optical depth, 1.2e-6 each) while the jumping march keeps far fewer samples."""
    import orc

    import cpx

    params = to_storage(case["params"], "bf16")
    params[0] = np.maximum(params[0] * 4.0 - 6.0, 0.0)  # opaque blob cores, empty space at the clamp
    scene, rays = make(case, "bf16", params)
    pred, accw, losses, grad = run_fb(scene, rays)
    n_jump = scene.last_sample_counts(rays.total_rays)
    osc, orays = oracle(case, params)
    pred64, accw64, _, grad64, _ = orc.fp64_step(osc, orays, MASK_COEF, HUBER, skip_empty=True,
                                                   t_stop=orc.MIXED_T_STOP)
    assert np.abs(pred - pred64).max() < 1e-4
    assert np.abs(accw - accw64).max() < 1e-4
    assert normwise(grad[0], grad64[0]) < 2e-3
    assert normwise(grad[1:], grad64[1:]) < 2e-3
    scene.set_options(cpx.OPT_NO_EMPTY_SKIP | cpx.OPT_NO_EARLY_STOP)
    pred_full, _, _, _ = run_fb(scene, rays)
    n_full = scene.last_sample_counts(rays.total_rays)
    assert np.abs(pred - pred_full).max() < 5e-4
    assert n_jump.sum() < 0.8 * n_full.sum()
    assert np.all(n_jump <= n_full)


def test_mixed_training_tracks_fp32_training(cuda, case):
    """Twenty batches of the same rays in both forms: the batch MSE of the mixed form stays
    within 2% of the FP32 form's."""
    import torch

    import cpx

    curves = {}
    for form in ("fp32", "bf16"):
        scene, rays = make(case, form)
        nr = rays.total_rays
        losses = torch.zeros(nr, dtype=torch.float64, device="cuda")
        curve = []
        for t in range(1, 21):
            curve.append(cpx.train_step(scene, rays, losses, timestep=t, lam_density=1e-3, lam_sh=1e-3, lr=0.1,
                                        sh_lr=0.01))
        curves[form] = np.array(curve)
    assert curves["fp32"][-1] < curves["fp32"][0]
    assert np.all(np.abs(curves["bf16"] - curves["fp32"]) <= 0.02 * curves["fp32"])


@pytest.mark.parametrize("dims", [(37, 30, 45), (66, 17, 9), (5, 4, 40), (33, 9, 5), (65, 2, 6)])
def test_dense_cell_map_is_bit_exact(cuda, dims):
    """The dense empty-space map the mixed march jumps by, bit for bit against the oracle's
    (a cell is open unless all eight corner densities are at or below 0): after an upload and
    after a sweep that moves densities across 0, on uneven grids whose cell counts leave a
    ragged last word, whose cell rows are shorter than a word (W = 5) or exactly one (W = 33),
    or one vertex longer than two words (W = 65).  The FP32 form's march keeps no map."""
    import orc

    import cpx

    W, H, D = dims
    n = W * H * D
    rng = np.random.default_rng(W * 1000 + H)
    params = rng.normal(0.0, 0.05, (28, n)).astype(np.float32)
    dens = rng.normal(0.0, 1.0, n).astype(np.float32)
    dens[rng.random(n) < 0.9] = 0.0  # mostly at the clamp: about two thirds of the cells empty
    params[0] = dens
    scene = cpx.ObjectScene(W, H, D, 9, precision="bf16", sr_seed=3)
    scene.upload_params(params)
    got = scene.cell_map()
    want = orc.dense_open_cells(dens, W, H, D)
    assert 0.1 < want.mean() < 0.9
    assert np.array_equal(got, want)
    grads = rng.normal(0.0, 1.0, params.shape).astype(np.float32)
    scene.upload_grads(grads)
    cpx.Optimizer.varianceAndUpdate(scene, 1e-4, 1e-5, 0.3, 0.1, 1)
    after = scene.download_params()[0]
    assert np.mean((after > 0) != (dens > 0)) > 0.05  # the sweep moved densities across 0
    assert np.array_equal(scene.cell_map(), orc.dense_open_cells(after, W, H, D))
    fp32 = cpx.ObjectScene(W, H, D, 9, precision="fp32")
    fp32.upload_params(params)
    with pytest.raises(cpx.CpxError):
        fp32.cell_map()


def test_sparse_adam_updates_touched_vertices_only(cuda, case):
    """CPX_OPT_SPARSE_ADAM on a BF16 grid with non-zero moments everywhere: after one batch of
    512 rays and the fused TV + Adam sweep, every vertex the batch gave a gradient has new
    moments, every vertex whose moments did not change kept its parameters bit for bit (dense
    Adam would move them through their moments), and most of the 64^3 grid is such a vertex."""
    import torch

    import cpx

    scene, rays = make(case, "bf16")
    scene.set_options(cpx.OPT_SPARSE_ADAM)
    rng = np.random.default_rng(2)
    shape = (28, scene.actual_grid_nums)
    scene.upload_moments(rng.normal(0, 1e-3, shape).astype(np.float32),
                         rng.uniform(1e-8, 1e-6, shape).astype(np.float32))
    p0 = scene.download_params()
    m0, v0 = scene.download_moments()
    losses = torch.zeros(512, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, None, 0, 512, MASK_COEF, HUBER)
    scene.check()
    hit = np.any(scene.download_grads() != 0, axis=0)
    cpx.Optimizer.varianceAndUpdate(scene, 1e-3, 1e-3, 0.1, 0.01, 1)
    scene.check()
    p1 = scene.download_params()
    m1, v1 = scene.download_moments()
    moved = np.any(m1 != m0, axis=0) | np.any(v1 != v0, axis=0)
    assert hit.sum() > 0 and np.all(moved[hit])
    assert np.array_equal(p1[:, ~moved].view(np.uint32), p0[:, ~moved].view(np.uint32))
    assert (~moved).mean() > 0.5
    scene.close()
    rays.close()
