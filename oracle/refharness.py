"""ctypes wrapper of oracle/_ref/libcpxref.so: the reference's own CUDA kernels.

TEST INFRASTRUCTURE ONLY.  libcpxref.so is the reference's unmodified sources
(SparseVolumeRadianceField/*.cu) built for sm_100a plus the ref_harness.cu
shim; it runs on a GPU only.  Used to pin parity (golden fixtures, GPU parity
tests) and as the reference arm of bench.py.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

REF_DIR = pathlib.Path(__file__).resolve().parent / "_ref"
LIB_PATH = REF_DIR / "libcpxref.so"

_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `make -C {LIB_PATH.parent.parent} ref` where the "
                              "reference sources are present")
        _lib = C.CDLL(str(LIB_PATH))
        _setup(_lib)
    return _lib


_vp = C.c_void_p


def _setup(L):
    def s(name, args, res=C.c_int):
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res

    s("ref_device_sync", [])
    s("ref_scene_create_dense", [C.c_int] * 5 + [C.c_float, _vp, _vp, C.POINTER(_vp)])
    s("ref_scene_create_sparse", [C.c_int] * 5 + [C.c_float, _vp, C.c_float, C.POINTER(_vp),
                                                  C.POINTER(C.c_uint32)])
    s("ref_download_occupancy", [_vp, _vp, _vp, _vp])
    s("ref_set_offsets", [_vp, _vp, _vp, _vp, C.c_int])
    s("ref_optimizer_init", [_vp, C.c_int])
    s("ref_rays_create", [_vp, C.c_int, C.c_int] + [_vp] * 12)
    s("ref_rays_init", [_vp, C.c_int, _vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int])
    s("ref_rays_count", [_vp])
    s("ref_render_image", [_vp] * 5 + [C.c_int] * 3 + [_vp] * 4)
    s("ref_upsample", [_vp, C.c_float, C.c_int, C.c_int, _vp])
    s("ref_bbox_silhouette", [_vp, C.c_int, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                              C.POINTER(C.c_double)])
    s("ref_adaptive_lr", [_vp, _vp])
    s("ref_save_text", [_vp, C.c_char_p, C.c_int, C.c_int, C.c_int])
    s("ref_load_text", [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, _vp])
    s("ref_image_load_text", [C.c_char_p, C.c_int, C.c_int, _vp, _vp, _vp, C.POINTER(C.c_int)])
    s("ref_rays_download", [_vp] + [_vp] * 17)
    s("ref_render_forward", [_vp, C.c_int, C.c_int])
    s("ref_render_backward", [_vp, C.c_int, C.c_int, C.c_double, C.c_float, _vp])
    s("ref_tv", [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int])
    s("ref_adam", [_vp, C.c_double, C.c_double, C.c_int])
    s("ref_train_step", [_vp, C.c_int, C.c_int, C.c_double, C.c_float, C.c_double, C.c_double, C.c_int,
                         C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _vp, _vp])
    s("ref_n_active", [_vp], C.c_int64)
    s("ref_sample_offsets", [_vp, C.c_uint, _vp, C.POINTER(C.c_int)])
    s("ref_max_sample_point", [_vp])
    L.ref_rand_values.argtypes = [C.c_uint, _vp, C.c_int]
    L.ref_rand_values.restype = None
    s("ref_params", [_vp, _vp, C.c_int])
    s("ref_grads", [_vp, _vp, C.c_int])
    s("ref_moments", [_vp, _vp, _vp, C.c_int])
    L.ref_destroy.argtypes = [_vp]
    L.ref_destroy.restype = None


def _ck(rc, where):
    if rc != 0:
        raise RuntimeError(f"reference harness {where} failed with code {rc}")


def _p(a):
    return None if a is None else a.ctypes.data


class RefScene:
    """The reference's ObjectScene + Optimizer + Rays driven through its own entry points."""

    def __init__(self, W, H, D, sh_dim, band, step, planar, adaptive_lr=None, sparse_threshold=None):
        L = lib()
        self.W, self.H, self.D, self.sh_dim = W, H, D, sh_dim
        self.n_arrays = 1 + 3 * sh_dim
        planar = np.ascontiguousarray(planar, np.float32)
        h = _vp()
        if sparse_threshold is None:
            alr = None if adaptive_lr is None else np.ascontiguousarray(adaptive_lr, np.float32)
            _ck(L.ref_scene_create_dense(W, H, D, sh_dim, band, float(step), _p(planar), _p(alr), C.byref(h)),
                "scene_create_dense")
            self.in_cage_count = None
        else:
            cnt = C.c_uint32()
            _ck(L.ref_scene_create_sparse(W, H, D, sh_dim, band, float(step), _p(planar),
                                          float(sparse_threshold), C.byref(h), C.byref(cnt)),
                "scene_create_sparse")
            self.in_cage_count = int(cnt.value)
        self.h = h
        self.n_act = int(L.ref_n_active(h))
        self.n_rays = 0

    def occupancy(self):
        W, H, D = self.W, self.H, self.D
        occ = np.zeros((W - 1) * (H - 1) * (D - 1), np.uint8)
        cage = np.zeros(W * H * D, np.uint8)
        idx = np.zeros(W * H * D, np.uint32)
        _ck(lib().ref_download_occupancy(self.h, _p(occ), _p(cage), _p(idx)), "download_occupancy")
        return occ, cage, idx

    def set_offsets(self, ox, oy, oz):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (ox, oy, oz)]
        _ck(lib().ref_set_offsets(self.h, *[_p(a) for a in arrs], len(arrs[0])), "set_offsets")

    def sample_offsets(self, seed):
        """setSelfSampleOffset(stepSize / 2) after srand(seed): (x, y, z) float64 arrays."""
        n = int(lib().ref_max_sample_point(self.h))
        out = np.zeros(3 * n, np.float64)
        got = C.c_int()
        _ck(lib().ref_sample_offsets(self.h, int(seed), _p(out), C.byref(got)), "sample_offsets")
        return out[:n].copy(), out[n:2 * n].copy(), out[2 * n:].copy()

    def optimizer_init(self, hierarchy=False):
        _ck(lib().ref_optimizer_init(self.h, 1 if hierarchy else 0), "optimizer_init")

    def rays_create(self, white_bg, ox, oy, oz, dx, dy, dz, near, far, mask, r, g, b):
        fs = [np.ascontiguousarray(a, np.float32) for a in (ox, oy, oz, dx, dy, dz, near, far)]
        bs = [np.ascontiguousarray(a, np.uint8) for a in (mask, r, g, b)]
        n = fs[0].size
        _ck(lib().ref_rays_create(self.h, n, 1 if white_bg else 0, *[_p(a) for a in fs + bs]), "rays_create")
        self.n_rays = n

    def rays_init(self, cams, img_w, img_h, images, pix_lists, white_bg):
        """cams: list of dicts (alpha, principle, c2w, centre); images: list of (r,g,b,mask) planes."""
        n = len(cams)
        alpha = np.ascontiguousarray([c["alpha"] for c in cams], np.float64)
        principle = np.ascontiguousarray([c["principle"] for c in cams], np.float64)
        c2w = np.ascontiguousarray([np.asarray(c["c2w"]).reshape(16) for c in cams], np.float64)
        centre = np.ascontiguousarray([np.asarray(c["centre"]).reshape(4) for c in cams], np.float64)
        planes = np.ascontiguousarray(
            np.stack([np.stack([np.asarray(p, np.uint8).reshape(-1) for p in im]) for im in images]), np.uint8)
        pix = np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32) for p in pix_lists]), np.int32)
        npix = np.ascontiguousarray([len(p) for p in pix_lists], np.int32)
        _ck(lib().ref_rays_init(self.h, n, _p(alpha), _p(principle), _p(c2w), _p(centre), img_w, img_h,
                                _p(planes), _p(pix), _p(npix), 1 if white_bg else 0), "rays_init")
        self.n_rays = int(lib().ref_rays_count(self.h))

    def rays_download(self):
        n = self.n_rays
        names = ("ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b",
                 "acc_density", "acc_weights", "acc_r", "acc_g", "acc_b")
        out = {k: np.zeros(n, np.uint8 if k in ("mask", "r", "g", "b") else np.float32) for k in names}
        _ck(lib().ref_rays_download(self.h, *[_p(out[k]) for k in names]), "rays_download")
        return out

    def upsample(self, threshold, low_band_only=False, target_sh=None):
        """objectScene::initSelfByUpsample into a dense target of doubled dimensions."""
        target_sh = self.sh_dim if target_sh is None else int(target_sh)
        sh = 1 if low_band_only else target_sh
        out = np.zeros((1 + 3 * sh, 8 * self.W * self.H * self.D), np.float32)
        _ck(lib().ref_upsample(self.h, float(threshold), 1 if low_band_only else 0, target_sh, _p(out)), "upsample")
        return out

    def render_image(self, cam, width, height, white_bg=True):
        """RenderUtils::renderImage of one camera -> rgb [3, w*h], rgb8 [3, w*h], depth, mask."""
        alpha = np.ascontiguousarray(cam["alpha"], np.float64)
        principle = np.ascontiguousarray(cam["principle"], np.float64)
        c2w = np.ascontiguousarray(cam["c2w"], np.float64).reshape(16)
        centre = np.ascontiguousarray(cam["centre"], np.float64).reshape(4)
        n = int(width) * int(height)
        out = {"rgb": np.zeros((3, n), np.float32), "rgb8": np.zeros((3, n), np.uint8),
               "depth": np.zeros(n, np.float32), "mask": np.zeros(n, np.uint8)}
        _ck(lib().ref_render_image(self.h, _p(alpha), _p(principle), _p(c2w), _p(centre), int(width), int(height),
                                   1 if white_bg else 0, _p(out["rgb"]), _p(out["rgb8"]), _p(out["depth"]),
                                   _p(out["mask"])), "render_image")
        return out

    def render_forward(self, start, length):
        _ck(lib().ref_render_forward(self.h, int(start), int(length)), "render_forward")
        _ck(lib().ref_device_sync(), "sync")

    def render_backward(self, start, length, mask_coef, huber):
        losses = np.zeros(length, np.float64)
        _ck(lib().ref_render_backward(self.h, int(start), int(length), float(mask_coef), float(huber),
                                      _p(losses)), "render_backward")
        return losses

    def tv(self, lam_d, lam_sh, type_=0, nbrs=6, optimize_step=0):
        _ck(lib().ref_tv(self.h, float(lam_d), float(lam_sh), int(type_), int(nbrs), int(optimize_step)), "tv")

    def adam(self, lr, sh_lr, timestep):
        _ck(lib().ref_adam(self.h, float(lr), float(sh_lr), int(timestep)), "adam")

    def train_step(self, start, length, mask_coef, huber, lam_d, lam_sh, tv_type, nbrs, do_tv, lr, sh_lr,
                   timestep, losses_buf=None):
        losses = np.zeros(length, np.float64) if losses_buf is None else losses_buf
        mse = C.c_double()
        _ck(lib().ref_train_step(self.h, int(start), int(length), float(mask_coef), float(huber), float(lam_d),
                                 float(lam_sh), int(tv_type), int(nbrs), 1 if do_tv else 0, float(lr),
                                 float(sh_lr), int(timestep), _p(losses), C.byref(mse)), "train_step")
        return mse.value

    def bbox_silhouette(self, projections, images, img_w, img_h, radius=0, get_scale=False):
        """RenderUtils::bbox_silhouette: carving with every camera, then the box; returns
        (bbox tuple, scale ratio)."""
        P = np.ascontiguousarray(np.stack([np.asarray(p, np.float64).reshape(12) for p in projections]))
        planes = np.ascontiguousarray(np.stack([np.stack([np.asarray(q, np.uint8).reshape(-1) for q in img])
                                                for img in images]))
        box = np.zeros(6, np.int32)
        sr = C.c_double()
        _ck(lib().ref_bbox_silhouette(self.h, len(projections), _p(P), _p(planes), int(img_w), int(img_h),
                                      int(radius), 1 if get_scale else 0, _p(box), C.byref(sr)),
            "bbox_silhouette")
        return tuple(int(x) for x in box), sr.value

    def save_text(self, directory, band, density_only=False, hierarchy_mode=False):
        _ck(lib().ref_save_text(self.h, str(directory).encode(), 1 if density_only else 0, int(band),
                                1 if hierarchy_mode else 0), "save_text")

    def adaptive_lr(self):
        out = np.zeros(self.W * self.H * self.D, np.float32)
        _ck(lib().ref_adaptive_lr(self.h, _p(out)), "adaptive_lr")
        return out

    def params(self):
        out = np.zeros((self.n_arrays, self.n_act), np.float32)
        _ck(lib().ref_params(self.h, _p(out), 0), "params")
        return out

    def grads(self):
        out = np.zeros((self.n_arrays, self.n_act), np.float32)
        _ck(lib().ref_grads(self.h, _p(out), 0), "grads")
        return out

    def set_grads(self, planar):
        a = np.ascontiguousarray(planar, np.float32)
        _ck(lib().ref_grads(self.h, _p(a), 1), "set_grads")

    def moments(self):
        m = np.zeros((self.n_arrays, self.n_act), np.float32)
        v = np.zeros((self.n_arrays, self.n_act), np.float32)
        _ck(lib().ref_moments(self.h, _p(m), _p(v), 0), "moments")
        return m, v

    def set_moments(self, m, v):
        a = np.ascontiguousarray(m, np.float32)
        b = np.ascontiguousarray(v, np.float32)
        _ck(lib().ref_moments(self.h, _p(a), _p(b), 1), "set_moments")

    def sync(self):
        _ck(lib().ref_device_sync(), "sync")

    def close(self):
        if getattr(self, "h", None):
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rand_values(seed, n=3):
    """What the host's rand() returns after srand(seed) (the reference draws its jitter seeds so)."""
    out = np.zeros(n, np.uint32)
    lib().ref_rand_values(int(seed), _p(out), int(n))
    return out


def load_text(directory, W, H, D, step, sh_dim, target_sh):
    """objectScene::initFromFile of a dense checkpoint: planar parameters [1 + 3 target_sh][W*H*D]."""
    out = np.zeros((1 + 3 * target_sh, W * H * D), np.float32)
    _ck(lib().ref_load_text(str(directory).encode(), W, H, D, float(step), int(sh_dim), int(target_sh), _p(out)),
        "load_text")
    return out


def image_load_text(prefix, w, h):
    """Image::initSelfFromFile with mask: (r, g, b, mask) planes, bbox, masksIndex."""
    planes = np.zeros((4, w * h), np.uint8)
    box = np.zeros(4, np.int32)
    idx = np.zeros(w * h, np.int32)
    n = C.c_int()
    _ck(lib().ref_image_load_text(str(prefix).encode(), int(w), int(h), _p(planes), _p(box), _p(idx), C.byref(n)),
        "image_load_text")
    return tuple(planes), tuple(int(x) for x in box), idx[:n.value].copy()
