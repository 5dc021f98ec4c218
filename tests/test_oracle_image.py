"""Held-out view render of the oracle (RenderUtils::renderImage, RenderUtils.cu:1720-1810):
properties that hold for the reference's image kernel, checked on the CPU."""
import numpy as np
import pytest

import cpx_scenes as S
import orc


def _scene(n=32, density=None, sh_dc=None, seed=3):
    rng = np.random.default_rng(seed)
    if density is None:
        centres, sigmas, peaks = S.random_blobs(rng, 6)
        dens = S.blob_density(n, n, n, centres, sigmas, peaks)
    else:
        dens = np.full(n ** 3, density, np.float32)
    params = S.make_params(dens, 9, rng, 0.3)
    if sh_dc is not None:
        params[1:] = 0.0
        params[1::9] = sh_dc
    return orc.Scene(n, n, n, 9, params, step=0.5), (0, n - 1, 0, n - 1, 0, n - 1)


def test_pixel_column_uses_modulo_height():
    """The reference takes a pixel's column as p % height (RenderUtils.cu:1727): in a
    8-wide, 4-high image the first row repeats its first four pixels."""
    scene, bbox = _scene()
    cam = S.look_at_camera(np.array([0.0, -4.0, 0.5]), 32, 8, 4, fov_deg=20.0)
    out = orc.render_image(scene, cam, bbox, 8, 4, True)
    rgb = out["rgb"]
    assert np.array_equal(rgb[:, 0:4], rgb[:, 4:8])
    assert np.array_equal(out["depth"][0:4], out["depth"][4:8])
    assert out["mask"].max() > 0


def test_rays_that_miss_the_box():
    """near > far: bytes 255, float colour 1 on a white background else 0, depth and mask 0.
    (The slab test does not ask for t > 0, so a camera looking away from the box still sees
    it behind itself; these rays run parallel to the box, beside it.)"""
    scene, bbox = _scene()
    cam = S.look_at_camera(np.array([0.0, -4.0, 0.0]), 32, 16, 16, fov_deg=10.0, target_world=(4.0, -4.0, 0.0))
    for white in (True, False):
        out = orc.render_image(scene, cam, bbox, 16, 16, white)
        assert np.all(out["rgb8"] == 255)
        assert np.all(out["rgb"] == (1.0 if white else 0.0))
        assert np.all(out["depth"] == 0) and np.all(out["mask"] == 0)


def test_transparent_scene_is_background():
    scene, bbox = _scene(density=-200.0)
    cam = S.look_at_camera(np.array([0.0, -4.0, 0.0]), 32, 24, 24)
    out = orc.render_image(scene, cam, bbox, 24, 24, False)
    assert np.all(out["rgb8"] == 255)
    assert np.all(out["mask"] == 0)
    assert np.abs(out["rgb"]).max() < 1e-6


def test_opaque_constant_colour():
    """An opaque field of SH DC value c renders sigmoid(0.1 c) where the rays hit the box;
    bytes and mask follow the reference's conversions."""
    scene, bbox = _scene(density=200.0, sh_dc=np.float32(8.0))
    cam = S.look_at_camera(np.array([0.0, -4.0, 0.0]), 32, 24, 24, fov_deg=10.0)
    out = orc.render_image(scene, cam, bbox, 24, 24, False)
    col = 1.0 / (1.0 + np.exp(-0.8))
    assert out["mask"].min() >= 254
    assert np.abs(out["rgb"] - col).max() < 1e-4
    assert np.all(np.abs(out["rgb8"].astype(int) - int(col * 255 + 0.5)) <= 1)
    # the expected depth lies inside the box along the ray, close to its entry point
    assert np.all(out["depth"] > 0)


def test_bytes_follow_the_float_image():
    """rgb8 = (int)((c + 1 - acc) * 255 + 0.5) of the plain composite c whatever the background,
    mask = (u8)(acc * 255), and the white background adds 1 - acc to every channel."""
    scene, bbox = _scene(seed=9)
    cam = S.look_at_camera(np.array([1.0, -3.5, 1.5]), 32, 40, 40)
    white = orc.render_image(scene, cam, bbox, 40, 40, True)
    plain = orc.render_image(scene, cam, bbox, 40, 40, False)
    assert np.array_equal(white["rgb8"], plain["rgb8"])
    assert np.array_equal(white["mask"], plain["mask"])
    assert np.array_equal(white["depth"], plain["depth"])
    bg = white["rgb"].astype(np.float64) - plain["rgb"]
    assert np.abs(bg[0] - bg[1]).max() < 1e-6 and np.abs(bg[0] - bg[2]).max() < 1e-6
    acc = 1.0 - bg[0]
    m = plain["mask"].astype(np.float64)
    assert np.all(acc >= m / 255 - 1e-6) and np.all(acc < (m + 1) / 255 + 1e-6)
    est = np.floor((plain["rgb"] + bg[0]) * 255 + 0.5)
    assert np.abs(est - plain["rgb8"]).max() <= 1
    assert (plain["mask"] > 0).any() and (plain["mask"] < 255).any()
