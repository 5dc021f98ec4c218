"""cpx_train_step_ahead: a training step that places the next batch's samples beside its
optimizer sweep.  The batch a step shades from a placement done in advance must equal a fresh
march of that batch on the same parameters bit for bit (sample counts, accumulated density and
weight, per-ray losses; RGB within 1e-5), and training must follow cpx_train_step within float
atomics noise.  A change of what placement reads (here: new parameters) makes the next step
place the batch itself."""
import numpy as np
import pytest

from tolerances import RGB_ABS

pytestmark = pytest.mark.gpu

STEP = dict(mask_coef=1.0, huber_delta=0.1, lam_density=1e-4, lam_sh=1e-5, lr=0.05, sh_lr=0.2)
N_BATCH = 512


def _grid_and_rays(cfg):
    import cpx

    n = cfg["W"]
    scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"])
    scene.upload_params(cfg["params"])
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr, white_bg=True)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                      cfg["img_w"], cfg["img_h"])
    return scene, rays


def _fresh_march(params, cfg, b, cuda):
    """Forward + backward of batch b on `params` by the plain path (placement done on the spot)."""
    import torch

    import cpx

    scene, rays = _grid_and_rays(cfg)
    scene.upload_params(params)
    losses = torch.zeros(N_BATCH, dtype=torch.float64, device=cuda)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, None, b * N_BATCH, N_BATCH, 1.0, 0.1)
    scene.check()
    out = rays.download(b * N_BATCH, N_BATCH, fields=cpx.RAY_OUTPUTS)
    counts = scene.last_sample_counts(N_BATCH)
    scene.close()
    rays.close()
    return out, counts, losses.cpu().numpy()


def test_step_ahead_shades_the_batch_a_fresh_march_would(cuda):
    import torch

    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=41, n=48, n_cams=6, img=64, n_rays=4 * N_BATCH)
    scene, rays = _grid_and_rays(cfg)
    twin, twin_rays = _grid_and_rays(cfg)
    losses = torch.zeros(N_BATCH, dtype=torch.float64, device=cuda)
    twin_losses = torch.zeros_like(losses)
    for k in range(4):
        b, nb = k % 4, (k + 1) % 4
        before = scene.download_params()
        mse = cpx.train_step_ahead(scene, rays, losses, start=b * N_BATCH, length=N_BATCH, next_rays=rays,
                                   next_start=nb * N_BATCH, next_length=N_BATCH, timestep=k + 1, **STEP)
        scene.check()
        got = rays.download(b * N_BATCH, N_BATCH, fields=cpx.RAY_OUTPUTS)
        counts = scene.last_sample_counts(N_BATCH)
        want, want_counts, want_losses = _fresh_march(before, cfg, b, cuda)
        assert np.array_equal(counts, want_counts), k
        assert np.array_equal(got["acc_density"].view(np.uint32), want["acc_density"].view(np.uint32)), k
        assert np.array_equal(got["acc_weights"].view(np.uint32), want["acc_weights"].view(np.uint32)), k
        for c in "rgb":
            assert np.abs(got[f"acc_{c}"] - want[f"acc_{c}"]).max() <= RGB_ABS
        assert np.array_equal(losses.cpu().numpy(), want_losses), k
        # the plain step on a twin grid trains the same way (float atomics aside)
        twin_mse = cpx.train_step(twin, twin_rays, twin_losses, start=b * N_BATCH, length=N_BATCH,
                                  timestep=k + 1, **STEP)
        assert abs(mse - twin_mse) <= (1e-12 if k == 0 else 1e-4) * twin_mse
    p, q = scene.download_params(), twin.download_params()
    tol = 1e-4 * STEP["lr"] + 1e-5 * np.abs(q)
    assert np.mean(np.abs(p - q) <= tol) >= 0.999
    # new parameters: the batch placed in advance is stale, the next step places it again
    changed = p.copy()
    changed[0] *= 0.5
    scene.upload_params(changed)
    cpx.train_step_ahead(scene, rays, losses, start=0, length=N_BATCH, next_rays=rays, next_start=N_BATCH,
                         next_length=N_BATCH, timestep=5, **STEP)
    scene.check()
    want, want_counts, _ = _fresh_march(changed, cfg, 0, cuda)
    assert np.array_equal(scene.last_sample_counts(N_BATCH), want_counts)
    assert np.array_equal(rays.download(0, N_BATCH, fields=("acc_density",))["acc_density"], want["acc_density"])
    for h in (scene, rays, twin, twin_rays):
        h.close()


def test_step_ahead_falls_back_where_it_does_not_apply(cuda):
    """A mixed-precision grid (or no next batch) runs the plain step."""
    import torch

    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=42, n=32, n_cams=4, img=48, n_rays=2 * N_BATCH)
    n = cfg["W"]
    for precision in ("fp32", "bf16"):
        scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"], precision=precision)
        scene.upload_params(cfg["params"])
        rays = cpx.Rays(2 * N_BATCH, white_bg=True)
        rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"], 48, 48)
        losses = torch.zeros(N_BATCH, dtype=torch.float64, device=cuda)
        nxt = rays if precision == "bf16" else None
        mse = cpx.train_step_ahead(scene, rays, losses, start=0, length=N_BATCH, next_rays=nxt,
                                   next_start=N_BATCH, next_length=N_BATCH, timestep=1, **STEP)
        scene.check()
        assert np.isfinite(mse) and mse > 0
        scene.close()
        rays.close()
