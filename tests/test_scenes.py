"""Synthetic workload conventions: voxel-space cameras, pixel-centre rays, blob fields."""
import numpy as np

import cpx_scenes as S


def test_world_box_maps_onto_vertex_range():
    assert np.allclose(S.world_to_voxel([-1.5, 0.0, 1.5], 128), [0.0, 63.5, 127.0])


def test_look_at_camera_is_orthonormal_and_centred():
    cam = S.look_at_camera([0.3, -4.0, 1.0], 64, 200, 100)
    R = cam["c2w"][:3, :3]
    assert np.allclose(R.T @ R, np.eye(3), atol=1e-12)
    assert np.isclose(np.linalg.det(R), 1.0)
    # optical axis (third column) points at the box centre
    to_centre = S.world_to_voxel([0, 0, 0], 64) - cam["centre"][:3]
    assert np.allclose(R[:, 2], to_centre / np.linalg.norm(to_centre))
    assert np.allclose(cam["principle"], [100.0, 50.0])
    assert np.isclose(cam["alpha"][0], 100.0 / np.tan(np.radians(20.0)))


def test_centre_pixel_ray_of_oracle_hits_box_centre():
    import orc

    n = 64
    cam = S.look_at_camera([0.0, 0.0, 4.0], n, 200, 200)
    rays = orc.RaySet(1, True)
    img = np.zeros(200 * 200, np.uint8)
    # pixel (row 99, col 99) has its centre at (99.5, 99.5), half a pixel off the axis
    orc.rays_from_camera(cam, (0, n - 1, 0, n - 1, 0, n - 1), 200, img, img, img, None, True,
                         np.array([99 * 200 + 99], np.int32), rays, 0)
    d = np.array([rays["dx"][0], rays["dy"][0], rays["dz"][0]], np.float64)
    assert abs(np.linalg.norm(d) - 1) < 1e-6
    mid = cam["centre"][:3] + d * (rays["near_t"][0] + rays["far_t"][0]) / 2
    assert np.linalg.norm(mid - (n - 1) / 2) < 0.5


def test_blob_field_matches_closed_form():
    centres = np.array([[0.1, -0.2, 0.3]])
    sig = np.array([0.25])
    dens = S.blob_density(16, 12, 10, centres, sig, np.array([50.0])).reshape(10, 12, 16)
    z, y, x = 7, 3, 11
    p = np.array([x / S.voxel_scale(16), y / S.voxel_scale(12), z / S.voxel_scale(10)]) - 1.5
    expect = 50.0 * np.exp(-np.sum((p - centres[0]) ** 2) / (2 * 0.25 ** 2))
    assert np.isclose(dens[z, y, x], expect, rtol=1e-5)


def test_packed_rays_roundtrip():
    rng = np.random.default_rng(0)
    f = [rng.random(5).astype(np.float32) for _ in range(8)]
    b = [rng.integers(0, 256, 5).astype(np.uint8) for _ in range(4)]
    p = S.pack_rays(*f, *b)
    assert p.shape == (5, 9) and p.dtype == np.uint32
    for i in range(8):
        assert np.array_equal(p[:, i].view(np.float32), f[i])
    assert np.array_equal(p[:, 8] & 0xff, b[0]) and np.array_equal(p[:, 8] >> 24, b[3])


def test_small_config_is_seeded():
    a = S.small_config(seed=3, n=16, n_cams=2, img=16, n_rays=64)
    b = S.small_config(seed=3, n=16, n_cams=2, img=16, n_rays=64)
    assert np.array_equal(a["params"], b["params"])
    assert all(np.array_equal(x, y) for x, y in zip(a["pix"], b["pix"]))
    assert sum(len(p) for p in a["pix"]) == 64
