"""The ray source (cpx_ray_source_*): rays generated per batch on the device equal the table
cpx_rays_init_camera builds (itself bit-exact with the reference's _rays::initialSelf, see
test_gpu_parity) field for field; the shuffled order is the oracle's keyed permutation;
training on generated batches equals training on the table's rows in the same order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b")


def _setup(mask_rays=True, white_bg=True, seed=3):
    import cpx
    import cpx_scenes as S

    cfg = S.small_config(seed=seed, n=40, n_cams=5, img=48, n_rays=3000)
    n = cfg["W"]
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(cfg["params"])
    cams = [cpx.Camera.make(**c) for c in cfg["cams"]]
    pix = cfg["pix"] if mask_rays else [np.arange(48 * 48, dtype=np.int32)] * len(cams)
    table = cpx.Rays(sum(len(p) for p in pix), white_bg=white_bg)
    table.initial_self(scene, cams, cfg["images"], pix, 48, 48)
    src = cpx.RaySource(cams, cfg["images"], 48, 48, pixel_lists=pix if mask_rays else None, white_bg=white_bg)
    return cfg, scene, table, src


def _fields(rays, n):
    return rays.download(0, n, fields=FIELDS)


@pytest.mark.parametrize("mask_rays", [True, False])
def test_identity_source_equals_the_ray_table(cuda, mask_rays):
    import cpx

    cfg, scene, table, src = _setup(mask_rays)
    n = len(src)
    assert n == table.total_rays
    out = cpx.Rays(n, white_bg=True)
    # in uneven batches
    start = 0
    for ln in (1, 700, 1, n - 702):
        batch = cpx.Rays(ln, white_bg=True)
        src.generate(scene, start, ln, batch)
        a, b = _fields(batch, ln), table.download(start, ln, fields=FIELDS)
        for k in FIELDS:
            assert np.array_equal(a[k], b[k]), (k, start)
        start += ln
    src.check()


def test_shuffled_order_is_the_oracle_permutation(cuda):
    import cpx
    import ray_source_ref as RS

    cfg, scene, table, src = _setup()
    n = len(src)
    src.shuffle(2024)
    keys, hb = src.keys()
    assert keys == RS.splitmix64_keys(2024) and hb == RS.half_bits(n)
    perm = RS.permute(np.arange(n), n, keys, hb)
    batch = cpx.Rays(n, white_bg=True)
    src.generate(scene, 0, n, batch)
    src.check()
    got = _fields(batch, n)
    want = table.download(0, n, fields=FIELDS)
    for k in FIELDS:
        assert np.array_equal(got[k], want[k][perm]), k
    # another epoch, another order; the identity comes back on request
    src.shuffle(2025)
    src.generate(scene, 0, n, batch)
    assert not np.array_equal(_fields(batch, n)["dx"], got["dx"])
    src.shuffle(0, shuffled=False)
    src.generate(scene, 0, 512, batch)
    assert np.array_equal(_fields(batch, 512)["dx"], want["dx"][:512])


def test_training_on_generated_batches_equals_the_gathered_table(cuda):
    """One batch from the source against the same rays gathered from the table by index (the
    reference's sample-index path): the forward is identical, so the batch MSE is too."""
    import torch

    import cpx
    import ray_source_ref as RS

    cfg, scene, table, src = _setup()
    n = len(src)
    src.shuffle(7)
    keys, hb = src.keys()
    perm = RS.permute(np.arange(n), n, keys, hb)
    L = 1024
    batch = cpx.Rays(L, white_bg=True)
    src.generate(scene, 1000, L, batch)
    losses = torch.zeros(L, dtype=torch.float64, device=cuda)
    a = cpx.train_step(scene, batch, losses, start=0, length=L, timestep=1)
    scene2 = cpx.ObjectScene(cfg["W"], cfg["W"], cfg["W"], 9)
    scene2.upload_params(cfg["params"])
    idx = torch.from_numpy(perm[1000:1000 + L].astype(np.int32)).to(cuda)
    b = cpx.train_step(scene2, table, losses, start=0, length=L, sample_index=idx, timestep=1)
    assert a == b
    assert np.array_equal(scene.download_params(), scene2.download_params()) or \
        np.abs(scene.download_params() - scene2.download_params()).max() < 1e-4  # float-atomics order


def test_out_of_range_batches_are_refused(cuda):
    import cpx

    cfg, scene, table, src = _setup()
    n = len(src)
    batch = cpx.Rays(64, white_bg=True)
    with pytest.raises(cpx.CpxError):
        src.generate(scene, n - 10, 64, batch)
    with pytest.raises(cpx.CpxError):
        src.generate(scene, 0, 65, batch)
    black = cpx.Rays(64, white_bg=False)
    with pytest.raises(cpx.CpxError):
        src.generate(scene, 0, 64, black)
