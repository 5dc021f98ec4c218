"""Seeded synthetic workloads for the training path (no dataset needed).

The reference trains on NeRF-Blender images, which are not part of this
project; its conventions are kept instead (SparseVolumeRadianceField/
CameraUtils.cu:45-106, 365-377; Rays.cu:22-75):

* the world box [-1.5, 1.5]^3 maps linearly onto voxel index space [0, n-1]
  per axis, and cameras live in voxel space;
* cameras look at the box centre in OpenCV convention (x right, y down,
  z forward), described by the device fields getBound reads: focal lengths,
  principal point, camera-to-world matrix and centre;
* rays start at pixel centres (col + 0.5, row + 0.5).

Parameters are planar float32 [1 + 3*sh_dim][W*H*D] in z-y-x order, the
reference's totalVariableGPUPtrs order (density, then R/G/B SH blocks).
"""
from __future__ import annotations

import math

import numpy as np

WORLD_HALF = 1.5


def voxel_scale(n: int) -> float:
    """Voxels per world unit for an axis of n vertices."""
    return (n - 1) / (2.0 * WORLD_HALF)


def world_to_voxel(p, n: int):
    return (np.asarray(p, np.float64) + WORLD_HALF) * voxel_scale(n)


def look_at_camera(eye_world, n_vox: int, img_w: int, img_h: int, fov_deg: float = 40.0,
                   target_world=(0.0, 0.0, 0.0)):
    """Pinhole camera at eye_world looking at target_world, in the voxel space of an
    n_vox^3 grid.  Returns dict(alpha, principle, c2w (4x4), centre (4,))."""
    eye = world_to_voxel(eye_world, n_vox)
    tgt = world_to_voxel(target_world, n_vox)
    f = tgt - eye
    f /= np.linalg.norm(f)
    up = np.array([0.0, 0.0, 1.0])
    if abs(np.dot(f, up)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    c2w = np.eye(4)
    c2w[:3, 0] = r
    c2w[:3, 1] = d
    c2w[:3, 2] = f
    c2w[:3, 3] = eye
    focal = (img_w / 2.0) / math.tan(math.radians(fov_deg) / 2.0)
    return {
        "alpha": np.array([focal, focal]),
        "principle": np.array([img_w / 2.0, img_h / 2.0]),
        "c2w": c2w,
        "centre": np.array([eye[0], eye[1], eye[2], 1.0]),
    }


def projection_matrix(cam) -> np.ndarray:
    """The camera's 3x4 world-to-pixel matrix K [I|0] w2c (Camera::formulateProjectionMat's
    product), consistent with getBound's pixel rays: a point on pixel (row, col)'s centre ray
    projects to (col + 0.5, row + 0.5)."""
    ax, ay = cam["alpha"]
    px, py = cam["principle"]
    K = np.array([[ax, 0.0, px], [0.0, ay, py], [0.0, 0.0, 1.0]])
    w2c = np.linalg.inv(np.asarray(cam["c2w"], np.float64))
    return K @ w2c[:3, :]


def fibonacci_sphere(n: int, radius: float):
    i = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * i / n)
    theta = math.pi * (1 + 5 ** 0.5) * i
    return radius * np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], 1)


def upper_hemisphere(n: int, radius: float, rng):
    v = rng.normal(size=(n, 3))
    v[:, 2] = np.abs(v[:, 2])
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return radius * v


def random_blobs(rng, n, centre_range=1.0, sigma_range=(0.1, 0.3), peak=50.0):
    centres = rng.uniform(-centre_range, centre_range, size=(n, 3))
    sigmas = rng.uniform(sigma_range[0], sigma_range[1], size=n)
    peaks = np.full(n, float(peak))
    return centres, sigmas, peaks


def blob_density(W, H, D, centres, sigmas, peaks, device=None):
    """Sum of isotropic Gaussian blobs sampled at the vertices, float32 [W*H*D] (z-y-x).

    Uses torch on `device` when given (large grids), numpy otherwise."""
    axes = [np.arange(n) / voxel_scale(n) - WORLD_HALF for n in (W, H, D)]
    if device is not None:
        import torch

        out = torch.zeros((D, H, W), dtype=torch.float32, device=device)
        ax = [torch.as_tensor(a, dtype=torch.float64, device=device) for a in axes]
        for c, s, p in zip(centres, sigmas, peaks):
            gx = torch.exp(-((ax[0] - c[0]) ** 2) / (2 * s * s)).float()
            gy = torch.exp(-((ax[1] - c[1]) ** 2) / (2 * s * s)).float()
            gz = torch.exp(-((ax[2] - c[2]) ** 2) / (2 * s * s)).float()
            out += float(p) * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
        return out.reshape(-1)
    out = np.zeros((D, H, W), np.float32)
    for c, s, p in zip(centres, sigmas, peaks):
        g = [np.exp(-((a - ci) ** 2) / (2 * s * s)).astype(np.float32) for a, ci in zip(axes, c)]
        # restrict to the 4-sigma box of the blob
        sl = []
        for gi in g:
            nz = np.nonzero(gi > 1e-7)[0]
            sl.append(slice(nz[0], nz[-1] + 1) if nz.size else slice(0, 0))
        out[sl[2], sl[1], sl[0]] += np.float32(p) * (
            g[2][sl[2], None, None] * g[1][None, sl[1], None] * g[0][None, None, sl[0]])
    return out.reshape(-1)


def make_params(density, sh_dim, rng, sh_std):
    """Planar parameters: density row + 3*sh_dim rows of N(0, sh_std)."""
    n = density.size
    params = np.empty((1 + 3 * sh_dim, n), np.float32)
    params[0] = density
    params[1:] = rng.normal(0.0, sh_std, size=(3 * sh_dim, n)).astype(np.float32)
    return params


def sample_pixels(rng, n_cams, img_w, img_h, n_rays):
    """n_rays random (camera, pixel) pairs, grouped per camera: list of pixel-index arrays."""
    cam = rng.integers(0, n_cams, size=n_rays)
    pix = rng.integers(0, img_w * img_h, size=n_rays)
    return [np.sort(pix[cam == i]).astype(np.int32) for i in range(n_cams)]


def small_config(seed=0, n=128, n_cams=16, img=200, n_rays=4096, sh_dim=9, n_blobs=8):
    """The CPU-runnable plain case: dense n^3 blob scene, SH ~ N(0, 0.3), cameras on a
    Fibonacci sphere r=4, img x img at fov 40 deg, n_rays random rays, step 0.5, white
    background; ground-truth colours are seeded random bytes."""
    rng = np.random.default_rng(seed)
    centres, sigmas, peaks = random_blobs(rng, n_blobs)
    dens = blob_density(n, n, n, centres, sigmas, peaks)
    params = make_params(dens, sh_dim, rng, 0.3)
    cams = [look_at_camera(p, n, img, img) for p in fibonacci_sphere(n_cams, 4.0)]
    images = [tuple(rng.integers(0, 256, size=img * img, dtype=np.uint8) for _ in range(3)) +
              (np.full(img * img, 255, np.uint8),) for _ in range(n_cams)]
    pix = sample_pixels(rng, n_cams, img, img, n_rays)
    return {
        "W": n, "H": n, "D": n, "sh_dim": sh_dim, "step": 0.5, "params": params, "cams": cams,
        "images": images, "pix": pix, "img_w": img, "img_h": img, "white_bg": True,
        "bbox": (0, n - 1, 0, n - 1, 0, n - 1),
    }


def pack_rays(ox, oy, oz, dx, dy, dz, near, far, r, g, b, mask):
    """Packed ray records for cpx_rays_upload_packed: uint32 [n, 9]."""
    n = len(ox)
    out = np.empty((n, 9), np.uint32)
    for i, a in enumerate((ox, oy, oz, dx, dy, dz, near, far)):
        out[:, i] = np.asarray(a, np.float32).view(np.uint32)
    out[:, 8] = (np.asarray(r, np.uint32) | (np.asarray(g, np.uint32) << 8) |
                 (np.asarray(b, np.uint32) << 16) | (np.asarray(mask, np.uint32) << 24))
    return out
