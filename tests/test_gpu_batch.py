"""Batched multi-scene training (cpx_batch_*): one batched iteration equals cpx_train_step on
every scene alone with start = (i % pool) * len and timestep i + 1.

The forward of a step is deterministic, so the per-scene MSE of the first step is compared to
1e-12 relative (only the order of the final double sum differs).  The gradient scatter uses
float atomics whose order varies between runs, so parameters and moments after several
steps are compared with a tolerance: 99.9 % of the values within 1e-4 * lr + 1e-5 * |value|
and none further than one Adam step (lr) away; a wrong ray batch, scene or timestep moves
nearly every value by a sizeable fraction of lr and fails the first bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LR = 0.05
SH_LR = 0.2
STEP_KW = dict(lr=LR, sh_lr=SH_LR, lam_density=1e-4, lam_sh=1e-5, huber_delta=0.1, mask_coef=1.0)


def _scene(seed, n, n_rays, precision="fp32", sparse=False):
    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=seed, n=n, n_cams=4, img=48, n_rays=n_rays)
    scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"], precision=precision, sr_seed=seed + 1)
    scene.upload_params(cfg["params"])
    if sparse:
        scene.prune_self(1.0)
        scene.make_sparse()
    rays = cpx.Rays(n_rays, white_bg=True)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                      cfg["img_w"], cfg["img_h"])
    return scene, rays


# (seed, grid edge, ray table, rays per batch, sparse): uneven grids and batch lengths; the
# second scene's table holds two batches, so iteration 2 wraps to its first batch
SPECS = [(31, 32, 1536, 512, False), (32, 48, 1536, 768, True), (33, 40, 1200, 1200, False)]


def _twins(precision):
    solo = [_scene(s, n, nr, precision, sp) for s, n, nr, _, sp in SPECS]
    bat = [_scene(s, n, nr, precision, sp) for s, n, nr, _, sp in SPECS]
    return solo, bat


def _close(a, b, what):
    tol = 1e-4 * LR + 1e-5 * np.abs(a)
    d = np.abs(a - b)
    assert np.mean(d <= tol) >= 0.999, (what, float(np.mean(d <= tol)), float(d.max()))
    assert d.max() <= SH_LR, (what, float(d.max()))


def _solo_step(scene, rays, length, it):
    import torch

    import cpx

    pool = rays.total_rays // length
    losses = torch.zeros(length, dtype=torch.float64, device="cuda")
    return cpx.train_step(scene, rays, losses, start=(it % pool) * length, length=length, timestep=it + 1, **STEP_KW)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_batch_equals_per_scene_steps(cuda, precision):
    import cpx

    solo, bat = _twins(precision)
    lens = [sp[3] for sp in SPECS]
    batch = cpx.Batch([(sc, r, n) for (sc, r), n in zip(bat, lens)], **STEP_KW)
    assert batch.info()["total_rays"] == sum(lens)
    for it in range(3):
        want = np.array([_solo_step(sc, r, n, it) for (sc, r), n in zip(solo, lens)])
        batch.step(graphs=False)
        got = batch.mse()
        rel = 1e-12 if it == 0 else 1e-4
        assert np.all(np.abs(got - want) <= rel * np.abs(want)), (it, got, want)
    batch.check()
    assert batch.info()["iteration"] == 3
    for (a, _), (b, _) in zip(solo, bat):
        _close(a.download_params(), b.download_params(), "params")
        ma, va = a.download_moments()
        mb, vb = b.download_moments()
        _close(ma, mb, "m")
        # a 16-bit moment rounds stochastically: a gradient that differs in its last float bit
        # can land on the neighbouring bfloat16 value (2^-8 relative)
        vrel = 1e-3 if precision == "fp32" else 1e-2
        assert np.mean(np.abs(va - vb) <= vrel * np.abs(va) + 1e-12) >= 0.999
        assert b.touched_count() == 0  # the next batch's map starts clear
    batch.close()


def test_graph_replay_equals_eager(cuda):
    """Two identical batches, one stepped eagerly and one by graph replay: the first step's
    MSE is identical, later ones agree to float-atomics noise, and so do the grids."""
    import cpx

    lens = [sp[3] for sp in SPECS]
    e_sc = [_scene(s, n, nr, "fp32", sp) for s, n, nr, _, sp in SPECS]
    g_sc = [_scene(s, n, nr, "fp32", sp) for s, n, nr, _, sp in SPECS]
    eager = cpx.Batch([(sc, r, n) for (sc, r), n in zip(e_sc, lens)], **STEP_KW)
    graph = cpx.Batch([(sc, r, n) for (sc, r), n in zip(g_sc, lens)], **STEP_KW)
    for it in range(5):
        eager.step(graphs=False)
        graph.step(graphs=True)
        a, b = eager.mse(), graph.mse()
        if it == 0:
            assert np.array_equal(a, b)
        assert np.all(np.abs(a - b) <= 1e-4 * np.abs(a)), it
    eager.check()
    graph.check()
    assert graph.info()["iteration"] == 5
    for (a, _), (b, _) in zip(e_sc, g_sc):
        _close(a.download_params(), b.download_params(), "params")
    eager.close()
    graph.close()


def test_graph_follows_outside_changes(cuda):
    """A grid stepped outside the batch (its buffers flip) and gradients uploaded by hand
    (every record is read) both leave the captured graphs stale: the batch notices and the
    result matches an eager twin given the same outside work."""
    import cpx

    lens = [sp[3] for sp in SPECS]
    e_sc = [_scene(s, n, nr, "fp32", sp) for s, n, nr, _, sp in SPECS]
    g_sc = [_scene(s, n, nr, "fp32", sp) for s, n, nr, _, sp in SPECS]
    eager = cpx.Batch([(sc, r, n) for (sc, r), n in zip(e_sc, lens)], **STEP_KW)
    graph = cpx.Batch([(sc, r, n) for (sc, r), n in zip(g_sc, lens)], **STEP_KW)
    for it in range(6):
        if it == 2:
            for sc_list in (e_sc, g_sc):  # one scene steps alone: its parity flips
                sc, r = sc_list[1]
                _solo_step(sc, r, lens[1], 0)
        if it == 4:
            for sc_list in (e_sc, g_sc):  # hand-made gradients on scene 0
                sc = sc_list[0][0]
                g = np.full((sc.n_arrays, sc.actual_grid_nums), 1e-3, np.float32)
                sc.upload_grads(g)
        eager.step(graphs=False)
        graph.step(graphs=True)
        a, b = eager.mse(), graph.mse()
        assert np.all(np.abs(a - b) <= 1e-4 * np.abs(a)), it
    eager.check()
    graph.check()
    for (a, _), (b, _) in zip(e_sc, g_sc):
        _close(a.download_params(), b.download_params(), "params")
    eager.close()
    graph.close()


def test_autotune_keeps_training(cuda):
    import cpx

    lens = [sp[3] for sp in SPECS]
    sc = [_scene(s, n, nr, "bf16", sp) for s, n, nr, _, sp in SPECS]
    batch = cpx.Batch([(s, r, n) for (s, r), n in zip(sc, lens)], **STEP_KW)
    first = None
    for _ in range(2):
        batch.step()
        first = batch.mse() if first is None else first
    best = batch.autotune(steps_per_trial=2)
    assert best["place_block"] in (64, 128, 256, 512)
    assert best["shade_warps"] in (2, 4, 8) and best["grab"] in (1, 2, 4, 8)
    assert batch.tuning == best
    assert batch.info()["iteration"] > 2 + 2 * 3
    for _ in range(3):
        batch.step()
    batch.check()
    assert np.all(batch.mse() < first)  # every scene kept training
    batch.set_tuning(64, 8, 2)
    batch.step()
    batch.check()
    with pytest.raises(cpx.CpxError):
        batch.set_tuning(48, 4, 1)
    batch.close()


def test_batch_rejects_mixed_forms(cuda):
    import cpx

    a = _scene(41, 24, 256, "fp32")
    b = _scene(42, 24, 256, "bf16")
    with pytest.raises(cpx.CpxError):
        cpx.Batch([(a[0], a[1], 128), (b[0], b[1], 128)], **STEP_KW)
    with pytest.raises(cpx.CpxError):
        cpx.Batch([(a[0], a[1], 512)], **STEP_KW)  # more rays per batch than the table holds
    with pytest.raises(cpx.CpxError):
        cpx.Batch([(a[0], a[1], 128), (a[0], a[1], 128)], **STEP_KW)


@pytest.mark.parametrize("warps,spl", [(2, 2), (2, 4), (4, 2)])
def test_samples_per_step_equals_one_sample_per_lane(cuda, warps, spl):
    """Shading chunks of 32 * samples_per_step samples (one vertex table per chunk) give the
    forward of one sample per lane exactly (first-step MSE to 1e-12) and the same training
    within float-atomics noise after three steps."""
    import cpx

    lens = [sp[3] for sp in SPECS]
    runs = []
    for tuning in ((64, warps, 1, 1), (64, warps, 1, spl)):
        sc = [_scene(s, n, nr, "fp32", sp) for s, n, nr, _, sp in SPECS]
        batch = cpx.Batch([(s, r, n) for (s, r), n in zip(sc, lens)], **STEP_KW)
        batch.set_tuning(*tuning)
        assert batch.tuning["samples_per_step"] == tuning[3]
        mses = []
        for _ in range(3):
            batch.step(graphs=False)
            mses.append(batch.mse())
        batch.check()
        runs.append((mses, [s.download_params() for s, _ in sc]))
        batch.close()
    (m1, p1), (m2, p2) = runs
    assert np.all(np.abs(m1[0] - m2[0]) <= 1e-12 * np.abs(m1[0]))
    for a, b in zip(p1, p2):
        _close(a, b, "params")
