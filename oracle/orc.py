"""ctypes wrapper of liboracle.so (the CPU restatement of the reference's hot path).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  Array layouts follow the
reference: planar parameters [n_arrays][n_active], SoA rays.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

ORACLE_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"
if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: run `make -C {ORACLE_DIR} oracle`")
_lib = C.CDLL(str(LIB_PATH))

_vp = C.c_void_p

CONTRACT_RAYDIR = 1
CONTRACT_NORM_P0 = 2
CONTRACT_NORM_P1 = 4
CONTRACT_POS = 8
CONTRACT_ACCD = 16
CONTRACT_DEFAULT = CONTRACT_RAYDIR | CONTRACT_NORM_P0 | CONTRACT_POS


class _Scene(C.Structure):
    _fields_ = [
        ("W", C.c_int), ("H", C.c_int), ("D", C.c_int), ("sh_dim", C.c_int), ("band", C.c_int),
        ("hierarchy", C.c_int), ("optimize_step", C.c_int), ("step", C.c_float), ("sparse", C.c_int),
        ("n_act", C.c_int64), ("params", _vp), ("occ", _vp), ("index_offsets", _vp),
        ("in_cage", _vp), ("adaptive_lr", _vp), ("off_x", _vp), ("off_y", _vp), ("off_z", _vp),
        ("n_off", C.c_int),
    ]


class _Rays(C.Structure):
    _fields_ = [("n", C.c_int64), ("white_bg", C.c_int)] + [
        (f, _vp) for f in ("ox", "oy", "oz", "dx", "dy", "dz", "near_t", "far_t", "mask", "r", "g", "b",
                           "acc_den", "acc_w", "acc_r", "acc_g", "acc_b")
    ]


def _fn(name, args, res=None):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res
    return f


_fn("orc_set_contract_mode", [C.c_uint])
_fn("orc_get_contract_mode", [], C.c_uint)
_fn("orc_set_threads", [C.c_int])
_fn("orc_get_threads", [], C.c_int)
_fn("orc_density_activation", [C.c_float], C.c_float)
_fn("orc_density_derivation", [C.c_float], C.c_float)
_fn("orc_sigmoid", [C.c_float], C.c_float)
_fn("orc_sigmoid_derivative", [C.c_float], C.c_float)
_fn("orc_rays_from_camera", [_vp] * 5 + [C.c_int] + [_vp] * 4 + [C.c_int, _vp, C.c_int, C.POINTER(_Rays), C.c_int64])
_fn("orc_render_forward", [C.POINTER(_Scene), C.POINTER(_Rays), _vp, C.c_int, C.c_int, _vp])
_fn("orc_render_backward", [C.POINTER(_Scene), C.POINTER(_Rays), _vp, C.c_int, C.c_int, C.c_double,
                            C.c_float, _vp, _vp, _vp])
_fn("orc_tv_grad", [C.POINTER(_Scene), _vp, C.c_double, C.c_double, C.c_int, C.c_int])
_fn("orc_adam", [C.POINTER(_Scene), _vp, _vp, _vp, C.c_double, C.c_double, C.c_int])
_fn("orc_occupancy", [_vp, C.c_int, C.c_int, C.c_int, C.c_float, _vp, _vp, _vp, C.POINTER(C.c_int64)],
    C.c_uint32)
_fn("orc_compact", [_vp, C.c_int, C.c_int64, _vp, _vp, C.c_int64])
_fn("orc_mse", [_vp, C.c_int], C.c_double)
_fn("orc_composite_kat", [_vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp])
_fn("orc_render_image", [C.POINTER(_Scene)] + [_vp] * 5 + [C.c_int] * 3 + [_vp] * 4)
_fn("orc_upsample", [C.POINTER(_Scene), C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp])
_fn("orc_carve_silhouette", [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int])
_fn("orc_bbox", [_vp, C.c_int, C.c_int, C.c_int, _vp], C.c_double)
class _Bricks(C.Structure):
    _fields_ = [("bits", _vp), ("bx", C.c_int), ("by", C.c_int), ("bz", C.c_int), ("t_stop", C.c_double),
                ("cells", _vp)]


_fn("orc64_forward_backward", [C.POINTER(_Scene), C.POINTER(_Rays), C.POINTER(_Bricks), C.c_int, C.c_int, C.c_double,
                               C.c_double, _vp, _vp, _vp, _vp])
_fn("orc64_tv6", [C.POINTER(_Scene), _vp, _vp, C.c_double, C.c_double])
_fn("orc64_adam", [C.POINTER(_Scene), _vp, _vp, _vp, _vp, C.c_double, C.c_double, C.c_int])


def set_contract_mode(mode: int):
    _lib.orc_set_contract_mode(mode)


def set_threads(n: int):
    _lib.orc_set_threads(int(n))


def threads() -> int:
    return int(_lib.orc_get_threads())


def _p(a):
    return None if a is None else a.ctypes.data


class Scene:
    """Oracle view of a grid: planar float32 params [n_arrays][n_act] (owned, updated in place)."""

    def __init__(self, W, H, D, sh_dim, params, step=0.5, band=None, hierarchy=False, sparse=False,
                 occ=None, index_offsets=None, in_cage=None, adaptive_lr=None, offsets=None,
                 optimize_step=0):
        self.W, self.H, self.D, self.sh_dim = int(W), int(H), int(D), int(sh_dim)
        self.sparse = bool(sparse)
        self.band = int(round(sh_dim ** 0.5)) - 1 if band is None else int(band)
        self.params = np.ascontiguousarray(params, np.float32).reshape(1 + 3 * self.sh_dim, -1).copy()
        self.n_act = self.params.shape[1]
        self.occ = None if occ is None else np.ascontiguousarray(occ, np.uint8)
        self.index_offsets = None if index_offsets is None else np.ascontiguousarray(index_offsets, np.uint32)
        self.in_cage = None if in_cage is None else np.ascontiguousarray(in_cage, np.uint8)
        self.adaptive_lr = None if adaptive_lr is None else np.ascontiguousarray(adaptive_lr, np.float32)
        if offsets is not None:
            self.offsets = [np.ascontiguousarray(o, np.float64) for o in offsets]
        else:
            self.offsets = None
        s = _Scene()
        s.W, s.H, s.D, s.sh_dim, s.band = self.W, self.H, self.D, self.sh_dim, self.band
        s.hierarchy = 1 if hierarchy else 0
        s.optimize_step = int(optimize_step)
        s.step = float(step)
        s.sparse = 1 if sparse else 0
        s.n_act = self.n_act
        s.params = _p(self.params)
        s.occ = _p(self.occ)
        s.index_offsets = _p(self.index_offsets)
        s.in_cage = _p(self.in_cage)
        s.adaptive_lr = _p(self.adaptive_lr)
        if self.offsets:
            s.off_x, s.off_y, s.off_z = (_p(o) for o in self.offsets)
            s.n_off = len(self.offsets[0])
        self.c = s


class RaySet:
    """SoA ray table (host numpy arrays)."""

    FLOATS = ("ox", "oy", "oz", "dx", "dy", "dz", "near_t", "far_t", "acc_den", "acc_w", "acc_r", "acc_g",
              "acc_b")
    BYTES = ("mask", "r", "g", "b")

    def __init__(self, n, white_bg=True, **fields):
        self.n = int(n)
        self.white_bg = bool(white_bg)
        self.a = {}
        for f in self.FLOATS:
            self.a[f] = np.zeros(self.n, np.float32)
        for f in self.BYTES:
            self.a[f] = np.zeros(self.n, np.uint8)
        alias = {"near": "near_t", "far": "far_t"}
        for k, v in fields.items():
            k = alias.get(k, k)
            self.a[k][:] = np.asarray(v).reshape(-1)
        r = _Rays()
        r.n = self.n
        r.white_bg = 1 if white_bg else 0
        for f in self.FLOATS + self.BYTES:
            setattr(r, f, self.a[f].ctypes.data)
        self.c = r

    def __getitem__(self, k):
        return self.a[k]


def rays_from_camera(cam, bbox, img_w, red, green, blue, mask, white_bg, pix, out: RaySet, out_start: int):
    alpha = np.ascontiguousarray(cam["alpha"], np.float64)
    principle = np.ascontiguousarray(cam["principle"], np.float64)
    c2w = np.ascontiguousarray(cam["c2w"], np.float64).reshape(16)
    centre = np.ascontiguousarray(cam["centre"], np.float64).reshape(4)
    bb = np.ascontiguousarray(bbox, np.int32)
    red, green, blue = (np.ascontiguousarray(x, np.uint8).reshape(-1) for x in (red, green, blue))
    mask = None if mask is None else np.ascontiguousarray(mask, np.uint8).reshape(-1)
    pix = np.ascontiguousarray(pix, np.int32)
    _lib.orc_rays_from_camera(_p(alpha), _p(principle), _p(c2w), _p(centre), _p(bb), int(img_w), _p(red),
                              _p(green), _p(blue), _p(mask), 1 if white_bg else 0, _p(pix), pix.size,
                              C.byref(out.c), int(out_start))


def render_image(scene: Scene, cam, bbox, width, height, white_bg=True):
    """Held-out view (RenderUtils::renderImage, RenderUtils.cu:1720-1810) -> dict of
    rgb float32 [3, w*h], rgb8 uint8 [3, w*h], depth float32 [w*h], mask uint8 [w*h]."""
    alpha = np.ascontiguousarray(cam["alpha"], np.float64)
    principle = np.ascontiguousarray(cam["principle"], np.float64)
    c2w = np.ascontiguousarray(cam["c2w"], np.float64).reshape(16)
    centre = np.ascontiguousarray(cam["centre"], np.float64).reshape(4)
    bb = np.ascontiguousarray(bbox, np.int32)
    n = int(width) * int(height)
    out = {"rgb": np.zeros((3, n), np.float32), "rgb8": np.zeros((3, n), np.uint8),
           "depth": np.zeros(n, np.float32), "mask": np.zeros(n, np.uint8)}
    _lib.orc_render_image(C.byref(scene.c), _p(alpha), _p(principle), _p(c2w), _p(centre), _p(bb), int(width),
                          int(height), 1 if white_bg else 0, _p(out["rgb"]), _p(out["rgb8"]), _p(out["depth"]),
                          _p(out["mask"]))
    return out


def brick_map(occ, W, H, D):
    """One byte per 8x8x8-cell brick: 1 when any of its cells is occupied."""
    c = np.asarray(occ, np.uint8).reshape(D - 1, H - 1, W - 1)
    bz, by, bx = (-(-(D - 1) // 8), -(-(H - 1) // 8), -(-(W - 1) // 8))
    pad = np.zeros((bz * 8, by * 8, bx * 8), np.uint8)
    pad[:D - 1, :H - 1, :W - 1] = c
    b = pad.reshape(bz, 8, by, 8, bx, 8).max(axis=(1, 3, 5))
    return np.ascontiguousarray(b.reshape(-1), np.uint8), (bx, by, bz)


# transmittance below which the FP32 march of the mixed forms ends a ray (its default)
MIXED_T_STOP = 1.0e-4
# density at or below which a dense grid's cell is empty for the FP32 march (all 8 corners):
# the optimizer's density clamp, where trained empty space sits
EMPTY_DENSITY = np.float32(0.0)


def dense_open_cells(density, W, H, D):
    """One byte per cell of a dense grid: 1 unless all eight corner densities are at or below
    EMPTY_DENSITY (the FP32 march's dense empty-cell map)."""
    d = np.asarray(density, np.float32).reshape(D, H, W) > EMPTY_DENSITY
    o = (d[:-1, :-1, :-1] | d[:-1, :-1, 1:] | d[:-1, 1:, :-1] | d[:-1, 1:, 1:] | d[1:, :-1, :-1] | d[1:, :-1, 1:]
         | d[1:, 1:, :-1] | d[1:, 1:, 1:])
    return np.ascontiguousarray(o.reshape(-1), np.uint8)


def fp64_step(scene: Scene, rays: RaySet, mask_coef, huber, lam_d=None, lam_sh=None, lr=None, sh_lr=None,
              timestep=1, start=0, length=None, skip_empty=False, t_stop=0.0):
    """The FP64 host oracle of one training batch: forward+backward over rays[start:start+length]
    (skip_empty: the mixed forms' jumps over empty cells and bricks of a sparse grid; t_stop: their
    end of a ray once its transmittance falls below t_stop), then (when lr is given) TV type 0 / 6
    neighbours (when lam_d is given) and Adam from zero moments.  Returns pred [len, 3], accw,
    losses, grad [n_arrays, n_act] (before TV/Adam) and the post-step parameters (float64) or
    None."""
    length = rays.n - start if length is None else length
    na = 1 + 3 * scene.sh_dim
    pred = np.zeros((length, 3), np.float64)
    accw = np.zeros(length, np.float64)
    losses = np.zeros(length, np.float64)
    grad = np.zeros((na, scene.n_act), np.float64)
    bk = None
    if skip_empty and scene.sparse:
        bits, (bx, by, bz) = brick_map(scene.occ, scene.W, scene.H, scene.D)
        bk = _Bricks(bits.ctypes.data, bx, by, bz, float(t_stop), None)
    elif skip_empty:
        cells = dense_open_cells(scene.params[0], scene.W, scene.H, scene.D)
        bits, (bx, by, bz) = brick_map(cells, scene.W, scene.H, scene.D)
        bk = _Bricks(bits.ctypes.data, bx, by, bz, float(t_stop), cells.ctypes.data)
    elif t_stop > 0:
        bk = _Bricks(None, 0, 0, 0, float(t_stop), None)
    _lib.orc64_forward_backward(C.byref(scene.c), C.byref(rays.c), C.byref(bk) if bk is not None else None,
                                int(start), int(length), float(mask_coef), float(huber), _p(pred), _p(accw),
                                _p(losses), _p(grad))
    post = None
    if lr is not None:
        params = np.ascontiguousarray(scene.params, np.float64)
        g = grad.copy()
        if lam_d is not None:
            _lib.orc64_tv6(C.byref(scene.c), _p(params), _p(g), float(lam_d), float(lam_sh))
        m = np.zeros_like(params)
        v = np.zeros_like(params)
        _lib.orc64_adam(C.byref(scene.c), _p(params), _p(g), _p(m), _p(v), float(lr), float(sh_lr), int(timestep))
        post = params
    return pred, accw, losses, grad, post


def upsample(scene: Scene, dW, dH, dD, threshold, low_band_only=False, dst_sh=None):
    """upsampleScene of the scene into a dense dW x dH x dD target: planar float32 params."""
    dst_sh = (1 if low_band_only else scene.sh_dim) if dst_sh is None else int(dst_sh)
    out = np.zeros((1 + 3 * dst_sh, dW * dH * dD), np.float32)
    _lib.orc_upsample(C.byref(scene.c), int(dW), int(dH), int(dD), int(dst_sh), float(threshold),
                      1 if low_band_only else 0, _p(out))
    return out


def render_forward(scene: Scene, rays: RaySet, sample_index=None, start=0, length=None):
    length = rays.n - start if length is None else length
    counts = np.zeros(length, np.int32)
    si = None if sample_index is None else np.ascontiguousarray(sample_index, np.int32)
    _lib.orc_render_forward(C.byref(scene.c), C.byref(rays.c), _p(si), int(start), int(length), _p(counts))
    return counts


def render_backward(scene: Scene, rays: RaySet, mask_coef, huber, sample_index=None, start=0, length=None):
    length = rays.n - start if length is None else length
    counts = np.zeros(length, np.int32)
    losses = np.zeros(length, np.float64)
    grad = np.zeros(scene.params.shape, np.float64)
    si = None if sample_index is None else np.ascontiguousarray(sample_index, np.int32)
    _lib.orc_render_backward(C.byref(scene.c), C.byref(rays.c), _p(si), int(start), int(length),
                             float(mask_coef), float(huber), _p(losses), _p(grad), _p(counts))
    return losses, grad, counts


def tv_grad(scene: Scene, grad, lam_d, lam_sh, type_=0, nbrs=6):
    """grad: float32 planar array updated in place."""
    assert grad.dtype == np.float32 and grad.flags.c_contiguous
    _lib.orc_tv_grad(C.byref(scene.c), _p(grad), float(lam_d), float(lam_sh), int(type_), int(nbrs))


def adam(scene: Scene, grad, m, v, lr, sh_lr, timestep):
    for a in (grad, m, v):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    _lib.orc_adam(C.byref(scene.c), _p(grad), _p(m), _p(v), float(lr), float(sh_lr), int(timestep))


def occupancy(density, W, H, D, threshold):
    d = np.ascontiguousarray(density, np.float32).reshape(-1)
    occ = np.zeros((W - 1) * (H - 1) * (D - 1), np.uint8)
    cage = np.zeros(W * H * D, np.uint8)
    idx = np.zeros(W * H * D, np.uint32)
    dropped = C.c_int64(0)
    cnt = _lib.orc_occupancy(_p(d), W, H, D, float(threshold), _p(occ), _p(cage), _p(idx), C.byref(dropped))
    return occ, cage, idx, int(cnt), int(dropped.value)


def compact(dense_planar, in_cage, n_compact):
    dense = np.ascontiguousarray(dense_planar, np.float32)
    out = np.zeros((dense.shape[0], n_compact), np.float32)
    cage = np.ascontiguousarray(in_cage, np.uint8)
    _lib.orc_compact(_p(dense), dense.shape[0], dense.shape[1], _p(cage), _p(out), int(n_compact))
    return out


def mse(losses):
    l = np.ascontiguousarray(losses, np.float64)
    return float(_lib.orc_mse(_p(l), l.size))


def composite_kat(opacity, colour, gt):
    op = np.ascontiguousarray(opacity, np.float64)
    col = np.ascontiguousarray(colour, np.float64).reshape(3, -1)
    g = np.ascontiguousarray(gt, np.float64)
    n = op.size
    rr = np.zeros(3)
    w = np.zeros(n)
    og = np.zeros(n)
    cg = np.zeros((3, n))
    _lib.orc_composite_kat(_p(op), _p(col), n, _p(g), _p(rr), _p(w), _p(og), _p(cg))
    return rr, w, og, cg


def activations(x):
    """Vectorised R4 activations (for small arrays)."""
    x = np.asarray(x, np.float32).reshape(-1)
    f = [_lib.orc_density_activation, _lib.orc_density_derivation, _lib.orc_sigmoid, _lib.orc_sigmoid_derivative]
    return [np.array([fn(float(v)) for v in x], np.float32) for fn in f]


def carve_silhouette(density, lr, W, H, D, projection, image, img_w, img_h, radius=0):
    """silhouetteCarving of one camera, in place on float32 density / lr arrays [W*H*D]."""
    assert density.dtype == np.float32 and lr.dtype == np.float32
    assert density.flags.c_contiguous and lr.flags.c_contiguous
    P = np.ascontiguousarray(projection, np.float64).reshape(12)
    planes = [None if p is None else np.ascontiguousarray(p, np.uint8).reshape(-1) for p in image]
    _lib.orc_carve_silhouette(_p(density), _p(lr), int(W), int(H), int(D), _p(P), int(img_w), int(img_h),
                              _p(planes[0]), _p(planes[1]), _p(planes[2]),
                              None if planes[3] is None else _p(planes[3]), int(radius))


def bbox(lr, W, H, D):
    """(bbox tuple, scale ratio) of the vertices with lr > 1e-6."""
    out = np.zeros(6, np.int32)
    sr = _lib.orc_bbox(_p(np.ascontiguousarray(lr, np.float32)), int(W), int(H), int(D), _p(out))
    return tuple(int(x) for x in out), float(sr)


_fn("orc_sobol_offsets", [_vp, _vp, C.c_int, C.c_uint64, C.c_double, _vp])

_CURAND_SCRAMBLED_DIRECTION_VECTORS_64_JOEKUO6 = 104  # curandDirectionVectorSet_t (curand.h)
_sobol_tables = None


def sobol_tables(n_states):
    """cuRAND's scrambled 64-bit JOEKUO6 direction numbers [n_states][64] and the first n_states
    32-bit words of its 64-bit scramble constants (how randGPU copies them), read through the
    host API at run time (curandGetDirectionVectors64 / curandGetScrambleConstants64)."""
    global _sobol_tables
    if _sobol_tables is None:
        import ctypes.util
        import os

        names = [os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64", "libcurand.so"),
                 ctypes.util.find_library("curand") or "libcurand.so"]
        lib = None
        for nm in names:
            try:
                lib = C.CDLL(nm)
                break
            except OSError:
                continue
        if lib is None:
            raise ImportError("libcurand is needed for the jitter oracle's direction numbers")
        dirs, scr = C.c_void_p(), C.c_void_p()
        if lib.curandGetDirectionVectors64(C.byref(dirs), _CURAND_SCRAMBLED_DIRECTION_VECTORS_64_JOEKUO6) != 0 or \
                lib.curandGetScrambleConstants64(C.byref(scr)) != 0:
            raise RuntimeError("cuRAND tables unavailable")
        _sobol_tables = (lib, dirs.value, scr.value)
    _, dp, sp = _sobol_tables
    d = np.ctypeslib.as_array(C.cast(dp, C.POINTER(C.c_uint64)), shape=(n_states * 64,)).copy()
    s = np.ctypeslib.as_array(C.cast(sp, C.POINTER(C.c_uint32)), shape=(n_states,)).copy()
    return d.reshape(n_states, 64), s


def max_sample_point(W, H, D, step):
    """objectScene::maxSamplePoint (SceneUtils.cu:96)."""
    return int(np.sqrt(float(W * W + H * H + D * D)) / np.float64(np.float32(step)) + 1.5)


def sobol_offsets(length, first, radius, out=None):
    """randGPU(dest, length, radius, 1) (Utils.cu:1002-1044): float64[length]; entries beyond
    the reference's launch grid keep `out`'s values (zero by default)."""
    n_states = min(length, 20000)
    d, s = sobol_tables(n_states)
    res = np.zeros(length, np.float64) if out is None else np.ascontiguousarray(out, np.float64).copy()
    _lib.orc_sobol_offsets(d.ctypes.data, s.ctypes.data, int(length), int(first),
                           float(np.float64(np.float32(radius))), res.ctypes.data)
    return res
