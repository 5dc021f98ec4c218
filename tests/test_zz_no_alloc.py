"""cpx_render_forward_backward_noalloc: the march for callers that cannot allocate device
memory while they run (their allocator owns the device memory, or their loop may not
allocate once started).  It must give the same results as cpx_render_forward_backward,
twice in a row on the same fixed scratch, without taking device memory.

This file is collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

from tolerances import RGB_ABS, assert_grads_close

pytestmark = pytest.mark.gpu


def _noalloc():
    import cpx

    fn = cpx._lib.cpx_render_forward_backward_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_float,
                   C.c_void_p]
    fn.restype = C.c_int
    return fn


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    import torch

    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=31, n=64, n_cams=6, img=96, n_rays=1024)
    n = cfg["W"]
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(cfg["params"])
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"], 96, 96)
    zero = np.zeros((28, n ** 3), np.float32)

    # the allocating entry point
    ref_losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    scene.upload_grads(zero)
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, ref_losses, maskRayLossCoefficient=1.0, huberDelta=0.1)
    scene.check()
    ref_out = rays.download(fields=cpx.RAY_OUTPUTS)
    ref_grad = scene.download_grads()

    fn = _noalloc()
    # first call on this device looks up the scratch array's device address
    losses = torch.zeros(nr, dtype=torch.float64, device=cuda)
    scene.upload_grads(zero)
    assert fn(scene.handle, rays.handle, losses.data_ptr(), None, 0, nr, 1.0, 0.1, None) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for call in range(2):
        scene.upload_grads(zero)
        losses.zero_()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        assert fn(scene.handle, rays.handle, losses.data_ptr(), None, 0, nr, 1.0, 0.1, None) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20), "the call took device memory"
        out = rays.download(fields=cpx.RAY_OUTPUTS)
        grad = scene.download_grads()
        for k in ("acc_density", "acc_weights"):
            assert np.array_equal(out[k], ref_out[k]), (call, k)
        for c in "rgb":
            assert np.abs(out[f"acc_{c}"] - ref_out[f"acc_{c}"]).max() <= RGB_ABS
        assert np.abs(losses.cpu().numpy() - ref_losses.cpu().numpy()).max() <= 255 * RGB_ABS
        assert_grads_close(grad, ref_grad)
    assert torch.cuda.mem_get_info()[0] >= free_before - (2 << 20)


def test_noalloc_rejects_batches_beyond_its_fixed_size(cuda):
    import torch

    import cpx

    n = 256
    scene = cpx.ObjectScene(n, n, n, 9)   # ~890 sample slots per ray
    rays = cpx.Rays(4096)
    losses = torch.zeros(4096, dtype=torch.float64, device=cuda)
    fn = _noalloc()
    rc = fn(scene.handle, rays.handle, losses.data_ptr(), None, 0, 4096, 1.0, 0.1, None)
    assert cpx.STATUS[rc] == "CPX_ERR_INVALID_ARGUMENT"
    assert b"fixed scratch" in cpx._lib.cpx_last_error()
