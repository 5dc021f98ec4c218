"""Size-independent properties of the oracle (the CPU restatement of the reference)."""
import numpy as np
import pytest

import cpx_scenes as S
import orc


@pytest.fixture(scope="module")
def small():
    cfg = S.small_config(seed=5, n=32, n_cams=4, img=40, n_rays=300)
    n = cfg["W"]
    nr = sum(len(p) for p in cfg["pix"])
    rays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, rays, off)
        off += len(pix)
    scene = orc.Scene(n, n, n, 9, cfg["params"], step=0.5)
    return cfg, scene, rays


def test_sample_count_bound(small):
    """Every step is >= step - w and the weights sum to <= 1, so the march takes at most
    (far - near + 1)/step + 1 samples (RenderUtils.cu:1674-1705)."""
    cfg, scene, rays = small
    counts = orc.render_forward(scene, rays)
    hit = rays["near_t"] <= rays["far_t"]
    bound = np.floor((rays["far_t"].astype(np.float64) - rays["near_t"] + 1.0) / 0.5) + 2
    assert np.all(counts[hit] <= bound[hit])
    assert np.all(counts[~hit] == 0)
    assert counts.max() > 20


def test_forward_outputs_are_composites(small):
    cfg, scene, rays = small
    orc.render_forward(scene, rays)
    w = rays["acc_w"]
    assert np.all(w >= 0) and np.all(w <= 1 + 1e-6)
    for c in ("acc_r", "acc_g", "acc_b"):
        assert np.all(rays[c] >= -1e-6) and np.all(rays[c] <= 1 + 1e-5)


def test_missed_rays_have_no_background_and_zero_loss():
    """near > far: zero outputs, no white background, loss 0 (RenderUtils.cu:1943, 2145)."""
    rays = orc.RaySet(1, True, near=5.0, far=1.0, dx=1.0, mask=255, r=10, g=20, b=30)
    params = np.ones((28, 8 ** 3), np.float32)
    scene = orc.Scene(8, 8, 8, 9, params)
    assert orc.render_forward(scene, rays)[0] == 0
    assert rays["acc_r"][0] == 0 and rays["acc_w"][0] == 0
    losses, grad, _ = orc.render_backward(scene, rays, 1.0, 0.1)
    assert losses[0] == 0 and not grad.any()


def test_backward_replays_forward_samples(small):
    cfg, scene, rays = small
    c1 = orc.render_forward(scene, rays)
    _, grad, c2 = orc.render_backward(scene, rays, 1.0, 0.1)
    assert np.array_equal(c1, c2)
    assert np.abs(grad).max() > 0


def test_gradient_matches_finite_difference():
    """d(loss)/d(SH band-0) at the vertex with the largest gradient against a central
    difference of the rendered colour (Huber inactive, mask term off)."""
    rng = np.random.default_rng(0)
    n = 8
    params = np.zeros((28, n ** 3), np.float32)
    params[0] = 18.0 + rng.normal(0, 1, n ** 3).astype(np.float32)
    params[1:] = rng.normal(0, 0.5, (27, n ** 3)).astype(np.float32)
    o = np.array([-3.0, 3.3, 3.1], np.float32)
    d = np.array([1.0, 0.05, 0.1], np.float32)
    d /= np.linalg.norm(d)
    fields = dict(ox=o[0], oy=o[1], oz=o[2], dx=d[0], dy=d[1], dz=d[2], near=3.5, far=9.5, mask=0,
                  r=20, g=230, b=140)

    def colour(p):
        rays = orc.RaySet(1, True, **fields)
        orc.render_forward(orc.Scene(n, n, n, 9, p), rays)
        return np.array([rays["acc_r"][0], rays["acc_g"][0], rays["acc_b"][0]], np.float64)

    rays = orc.RaySet(1, True, **fields)
    sc = orc.Scene(n, n, n, 9, params)
    orc.render_forward(sc, rays)
    _, grad, _ = orc.render_backward(sc, rays, 0.0, 1.0)
    res = colour(params) - np.array([20, 230, 140]) / 255.0
    v = int(np.argmax(np.abs(grad[1])))
    got, want = [], []
    for k in (1, 10, 19):  # the band-0 SH coefficient of each channel
        h = 5e-2
        p1 = params.copy(); p1[k, v] += h
        p0 = params.copy(); p0[k, v] -= h
        dcol = (colour(p1) - colour(p0)) / (2 * h)
        got.append(grad[k, v])
        want.append(0.6667 * np.dot(res, dcol))  # the reference scales by 2/3 (RenderUtils.cu:2213)
    got, want = np.array(got), np.array(want)
    assert np.abs(got - want).max() <= 2e-3 * np.abs(want).max()


def test_tv_vanishes_on_constant_field():
    n = 10
    params = np.full((28, n ** 3), 0.7, np.float32)
    sc = orc.Scene(n, n, n, 9, params)
    for typ, nb in ((0, 3), (0, 6), (0, 26), (1, 6)):
        g = np.zeros_like(params)
        orc.tv_grad(sc, g, 1e-3, 1e-3, typ, nb)
        assert np.abs(g).max() <= 1e-3 * 1e-6  # lambda times a few float ulps of the mean


def test_adam_first_step_is_signed_lr():
    """At t=1 the bias-corrected step is lr * g/(|g| + eps) (Optimizer.cu:374-413)."""
    n = 4
    rng = np.random.default_rng(1)
    params = rng.normal(5.0, 1.0, (28, n ** 3)).astype(np.float32)
    grad = rng.normal(0, 1, params.shape).astype(np.float32)
    m = np.zeros_like(params)
    v = np.zeros_like(params)
    sc = orc.Scene(n, n, n, 9, params)
    orc.adam(sc, grad.copy(), m, v, 0.1, 0.01, 1)
    step = params - sc.params
    lr = np.array([0.1] + [0.01] * 27)[:, None]
    expect = lr * grad / (np.abs(grad) + 1e-6)
    mask = np.ones_like(step, bool)
    mask[0] = params[0] - expect[0] > 0  # density is clamped at 0
    assert np.allclose(step[mask], expect[mask], rtol=1e-5, atol=2e-6)  # ulp of params ~5


def test_occupancy_index_is_exclusive_prefix_of_in_cage():
    n = 12
    rng = np.random.default_rng(2)
    dens = rng.uniform(0, 10, n ** 3).astype(np.float32)
    occ, cage, idx, cnt, dropped = orc.occupancy(dens, n, n, n, 8.5)
    assert cnt == int(cage.sum())
    ex = np.cumsum(cage) - cage
    assert np.array_equal(idx[cage == 1], ex[cage == 1].astype(np.uint32))
    assert not idx[cage == 0].any()
    # occupancy: any corner strictly above the threshold
    d = dens.reshape(n, n, n)
    corners = np.stack([d[z:n - 1 + z, y:n - 1 + y, x:n - 1 + x] for z in (0, 1) for y in (0, 1) for x in (0, 1)])
    assert np.array_equal(occ.reshape(n - 1, n - 1, n - 1), (corners > 8.5).any(0).astype(np.uint8))


def test_occupancy_x_face_flag_quirk():
    """The x = W-1 face flag lands at depth*W*H + H*W + col + 1 (SceneUtils.cu:872), i.e. at
    vertex (W-1, 0, depth+1); for the last cell layer that is (W-1, 0, D-1), still in range."""
    n = 6
    dens = np.zeros(n ** 3, np.float32)
    v = 2 * n * n + 3 * n + (n - 1)  # vertex (x=W-1, y=3, z=2)
    dens[v] = 100.0
    occ, cage, idx, cnt, dropped = orc.occupancy(dens, n, n, n, 8.0)
    assert cage[2 * n * n + 3 * n + (n - 2)] == 1   # min corner of an occupied cell
    assert cage[v] == 0                              # never flagged by the x-face rule
    assert cage[3 * n * n + (n - 1)] == 1            # ...which flags (W-1, 0, z+1) instead
    dens2 = np.zeros(n ** 3, np.float32)
    dens2[(n - 1) * n * n + 2 * n + (n - 1)] = 100.0  # occupies cells at z = D-2, x = W-2
    _, cage2, _, _, dropped2 = orc.occupancy(dens2, n, n, n, 8.0)
    assert dropped2 == 0 and cage2[(n - 1) * n * n + (n - 1)] == 1


def test_fp64_oracle_agrees_with_the_reference_restatement(small):
    """The all-FP64 oracle (the yardstick of the mixed forms) computes the same step as the
    pinned restatement of the reference, up to the reference's float rounding."""
    cfg, scene, rays = small
    orc.render_forward(scene, rays)
    losses32, grad32, _ = orc.render_backward(scene, rays, 1.0, 0.1)
    pred64, accw64, losses64, grad64, post = orc.fp64_step(scene, rays, 1.0, 0.1, lam_d=1e-3, lam_sh=1e-3,
                                                           lr=0.1, sh_lr=0.01)
    pred32 = np.stack([rays["acc_r"], rays["acc_g"], rays["acc_b"]], 1)
    assert np.abs(pred64 - pred32).max() < 2e-5
    assert np.abs(accw64 - rays["acc_w"]).max() < 2e-5
    assert np.abs(losses64 - losses32).max() < 255 * 2e-5
    for blk in (slice(0, 1), slice(1, None)):
        err = np.abs(grad64[blk] - grad32[blk]).max() / np.abs(grad64[blk]).max()
        assert err < 1e-4, (blk, err)
    # Adam from zero moments moves every updated parameter by about lr * sign(g) at t = 1
    moved = np.abs(post - scene.params)
    assert np.isfinite(post).all() and moved[0].max() <= 0.1 + 1e-9 and moved[1:].max() <= 0.01 + 1e-9


def test_empty_space_jumps_keep_the_sample_sequence():
    """The FP32 march's jumps over empty cells and bricks move by whole steps, so in the FP64
    oracle a sparse march with jumps equals the step-by-step march up to rounding."""
    cfg = S.small_config(seed=8, n=48, n_cams=4, img=40, n_rays=400)
    n = cfg["W"]
    occ, cage, idx, cnt, _ = orc.occupancy(cfg["params"][0], n, n, n, 4.0)
    assert 0 < occ.mean() < 0.5
    comp = orc.compact(cfg["params"], cage, cnt)
    sc = orc.Scene(n, n, n, 9, comp, step=0.5, sparse=True, occ=occ, index_offsets=idx, in_cage=cage)
    nr = sum(len(p) for p in cfg["pix"])
    rays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, rays, off)
        off += len(pix)
    a = orc.fp64_step(sc, rays, 1.0, 0.1)
    b = orc.fp64_step(sc, rays, 1.0, 0.1, skip_empty=True)
    assert np.abs(a[0] - b[0]).max() < 1e-9
    assert np.abs(a[3] - b[3]).max() <= 1e-9 * np.abs(a[3]).max()
    assert np.abs(a[0] - 1.0).max() > 0.05  # the rays see the blobs


def test_early_stop_bounds_the_colour_change():
    """Ending a ray once its transmittance is below t_stop changes its colour and accumulated
    weight by at most t_stop (all that the rest of the ray could add, against the white
    background it would otherwise show); with t_stop 0 nothing changes."""
    cfg = S.small_config(seed=9, n=48, n_cams=4, img=40, n_rays=400)
    n = cfg["W"]
    params = cfg["params"].copy()
    params[0] *= 4.0  # opaque blobs: many rays end well before their far bound
    sc = orc.Scene(n, n, n, 9, params, step=0.5)
    nr = sum(len(p) for p in cfg["pix"])
    rays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, rays, off)
        off += len(pix)
    full = orc.fp64_step(sc, rays, 1.0, 0.1)
    same = orc.fp64_step(sc, rays, 1.0, 0.1, t_stop=0.0)
    # (the oracle's threads add gradients in any order: equal up to that rounding)
    assert np.array_equal(full[0], same[0])
    assert np.abs(full[3] - same[3]).max() <= 1e-12 * np.abs(full[3]).max()
    stop = orc.fp64_step(sc, rays, 1.0, 0.1, t_stop=orc.MIXED_T_STOP)
    assert np.abs(full[0] - stop[0]).max() <= orc.MIXED_T_STOP
    assert np.abs(full[1] - stop[1]).max() <= orc.MIXED_T_STOP
    assert (full[1] > 1 - orc.MIXED_T_STOP).mean() > 0.05  # some rays do end early
    # the gradients change only through the samples past the stop and the loss they shift
    assert np.linalg.norm(full[3] - stop[3]) <= 1e-2 * np.linalg.norm(full[3])


def test_dense_empty_cells_change_little():
    """On a dense grid the FP32 march jumps over cells whose eight corner densities are all at
    or below EMPTY_DENSITY (0, the optimizer's clamp): each such sample would add at most
    softplus(-13) * step to the optical depth; with empty space at the clamp the image moves
    by less than 2e-4 while the empty cells are skipped."""
    cfg = S.small_config(seed=10, n=48, n_cams=4, img=40, n_rays=400)
    n = cfg["W"]
    params = cfg["params"].copy()
    params[0] = np.maximum(params[0] - 6.0, 0.0)  # empty space at the clamp, blob cores above it
    sc = orc.Scene(n, n, n, 9, params, step=0.5)
    cells = orc.dense_open_cells(params[0], n, n, n)
    assert 0.01 < cells.mean() < 0.6
    nr = sum(len(p) for p in cfg["pix"])
    rays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(cfg["cams"], cfg["images"], cfg["pix"]):
        orc.rays_from_camera(cam, cfg["bbox"], cfg["img_w"], *img, True, pix, rays, off)
        off += len(pix)
    full = orc.fp64_step(sc, rays, 1.0, 0.1)
    jump = orc.fp64_step(sc, rays, 1.0, 0.1, skip_empty=True)
    assert np.abs(full[0] - jump[0]).max() < 2e-4
    assert np.abs(full[1] - jump[1]).max() < 2e-4
    assert np.abs(full[0] - 1.0).max() > 0.05  # the rays see the blobs
    # the gradients agree on the vertices of open cells; the skipped ones lose tiny terms
    assert np.linalg.norm(full[3] - jump[3]) <= 2e-3 * np.linalg.norm(full[3])
