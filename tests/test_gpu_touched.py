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
