"""Host-side mirror of the reference's training-path interface over libcpx.so.

The reference exposes its hot path as C++ static methods on structs passed by
value (SparseVolumeRadianceField/RenderUtils.cuh:7-85, Optimizer.cuh:5-38,
SceneUtils.cuh:4-98, Rays.cuh:8-57).  This module keeps those names and
argument meanings -- ``ObjectScene``, ``Rays``, ``RenderUtils.renderRays``,
``RenderUtils.renderRays_withGradients_RGB``, ``RenderUtils.addVarianceLoss``,
``Optimizer.updateRGBScene`` -- and calls the C ABI of include/cpx.h.  Where the
reference exits the process on a CUDA error (checkGPUStatus, Utils.cu:700-717)
these raise ``CpxError`` carrying the status code.

Device buffers that the reference takes as raw device pointers (the sample
index table and the per-ray losses) are passed as CUDA tensors or integer
device addresses.  There is no CPU fallback: importing this module fails
loudly when the compiled library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
# CPX_LIBRARY selects another build of the same ABI (e.g. a profiling variant)
LIB_PATH = pathlib.Path(os.environ.get("CPX_LIBRARY", PKG_DIR / "lib" / "libcpx.so"))

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` (or __graft_entry__.build())"
    )
_lib = C.CDLL(str(LIB_PATH))

STATUS = {
    0: "CPX_OK",
    1: "CPX_ERR_INVALID_ARGUMENT",
    2: "CPX_ERR_OUT_OF_MEMORY",
    3: "CPX_ERR_CUDA",
    4: "CPX_ERR_ITERATION_CAP",
    5: "CPX_ERR_NAN",
    6: "CPX_ERR_NOT_READY",
    7: "CPX_ERR_UNSUPPORTED",
}

# Exported symbols of include/cpx.h (checked by the CPU test suite).
EXPORTED = [
    "cpx_status_string", "cpx_last_error", "cpx_version", "cpx_grid_create", "cpx_grid_destroy",
    "cpx_grid_info", "cpx_grid_upload_params", "cpx_grid_upload_params_device", "cpx_grid_download_params", "cpx_grid_upload_grads",
    "cpx_grid_download_grads", "cpx_grid_upload_moments", "cpx_grid_download_moments",
    "cpx_grid_set_adaptive_lr", "cpx_grid_set_sample_offsets", "cpx_grid_fill_sample_offsets",
    "cpx_grid_download_sample_offsets",
    "cpx_grid_set_optimize_step",
    "cpx_occupancy_build", "cpx_grid_download_occupancy", "cpx_grid_make_sparse", "cpx_rays_create", "cpx_rays_destroy",
    "cpx_rays_upload", "cpx_rays_upload_packed", "cpx_rays_download", "cpx_rays_init_camera",
    "cpx_render_forward", "cpx_render_backward", "cpx_render_forward_backward", "cpx_tv_grad",
    "cpx_adam_step", "cpx_tv_adam_step", "cpx_train_step", "cpx_train_step_ahead", "cpx_grid_check",
    "cpx_last_sample_counts", "cpx_kernel_launches", "cpx_render_forward_backward_noalloc",
    "cpx_render_image", "cpx_image_mse", "cpx_grid_touched_count", "cpx_grid_download_cell_map",
    "cpx_proposal_param_count", "cpx_proposal_create", "cpx_proposal_destroy", "cpx_proposal_params",
    "cpx_proposal_infer", "cpx_proposal_gradient", "cpx_proposal_train", "cpx_proposal_stats",
    "cpx_render_forward_backward_guided", "cpx_train_step_proposal", "cpx_render_forward_guided",
    "cpx_grid_set_options", "cpx_grid_upsample",
    "cpx_batch_create", "cpx_batch_destroy", "cpx_batch_step", "cpx_batch_mse", "cpx_batch_check",
    "cpx_batch_info", "cpx_batch_set_tuning", "cpx_batch_get_tuning", "cpx_batch_autotune",
    "cpx_carve_silhouette", "cpx_grid_bbox",
    "cpx_ray_source_create", "cpx_ray_source_destroy", "cpx_ray_source_count", "cpx_ray_source_shuffle",
    "cpx_ray_source_keys", "cpx_ray_source_generate", "cpx_ray_source_check",
    "cpx_grid_save_text", "cpx_grid_load_text", "cpx_grid_load_text_sparse", "cpx_config_read", "cpx_image_load_text", "cpx_image_mask_pixels",
]


class CpxError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        self.name = STATUS.get(status, str(status))
        msg = _lib.cpx_last_error().decode(errors="replace")
        super().__init__(f"{where}: {self.name}: {msg}")


class GridDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("depth", C.c_int),
        ("sh_dim", C.c_int), ("optimizing_band", C.c_int), ("hierarchy_strategy", C.c_int),
        ("step_size", C.c_float), ("bbox", C.c_int * 6), ("precision", C.c_int), ("sr_seed", C.c_uint32),
    ]


# storage forms (cpx_precision)
PRECISIONS = {"fp32": 0, "bf16": 1, "fp16": 2, "fp16full": 3}


class Camera(C.Structure):
    """Device fields of the reference's Camera that getBound reads (CameraUtils.cuh:16-26)."""
    _fields_ = [
        ("alpha", C.c_double * 2), ("principle", C.c_double * 2),
        ("c2w", C.c_double * 16), ("centre", C.c_double * 4),
    ]

    @classmethod
    def make(cls, alpha, principle, c2w, centre):
        cam = cls()
        cam.alpha[:] = [float(a) for a in alpha]
        cam.principle[:] = [float(p) for p in principle]
        cam.c2w[:] = [float(v) for v in np.asarray(c2w, dtype=np.float64).reshape(16)]
        cam.centre[:] = [float(v) for v in np.asarray(centre, dtype=np.float64).reshape(4)]
        return cam


class StepArgs(C.Structure):
    _fields_ = [
        ("mask_coef", C.c_double), ("huber_delta", C.c_float), ("do_tv", C.c_int),
        ("tv_type", C.c_int), ("tv_neighbours", C.c_int), ("lam_density", C.c_double),
        ("lam_sh", C.c_double), ("lr", C.c_double), ("sh_lr", C.c_double), ("timestep", C.c_int),
    ]


_vp = C.c_void_p
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _sig(name, args, res=C.c_int):
    fn = getattr(_lib, name)
    fn.argtypes = args
    fn.restype = res
    return fn


_lib.cpx_last_error.restype = C.c_char_p
_lib.cpx_status_string.restype = C.c_char_p
_lib.cpx_status_string.argtypes = [C.c_int]
_sig("cpx_version", [])
_sig("cpx_kernel_launches", [], C.c_int64)
_sig("cpx_grid_create", [C.POINTER(GridDesc), C.POINTER(_vp)])
_sig("cpx_grid_destroy", [_vp])
_sig("cpx_grid_info", [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int)])
for _n in ("upload_params", "download_params", "upload_grads", "download_grads"):
    _sig(f"cpx_grid_{_n}", [_vp, _f32p, C.c_int64])
_sig("cpx_grid_upload_params_device", [_vp, _vp, C.c_int64])
_sig("cpx_grid_upload_moments", [_vp, _f32p, _f32p, C.c_int64])
_sig("cpx_grid_download_moments", [_vp, _f32p, _f32p, C.c_int64])
_sig("cpx_grid_set_adaptive_lr", [_vp, _f32p, C.c_int64])
_sig("cpx_grid_set_sample_offsets", [_vp, _vp, _vp, _vp, C.c_int])
_sig("cpx_grid_fill_sample_offsets", [_vp, C.c_float, _vp, _vp])
_sig("cpx_grid_download_sample_offsets", [_vp, _vp, _vp, _vp, C.c_int])
_sig("cpx_grid_set_optimize_step", [_vp, C.c_int])
_sig("cpx_occupancy_build", [_vp, C.c_float, _vp, _vp, _vp, C.POINTER(C.c_uint32)])
_sig("cpx_grid_make_sparse", [_vp])
_sig("cpx_grid_check", [_vp])
_sig("cpx_rays_create", [C.c_int64, C.c_int, C.POINTER(_vp)])
_sig("cpx_rays_destroy", [_vp])
_sig("cpx_rays_upload", [_vp, C.c_int64, C.c_int64] + [_vp] * 12 + [_vp])
_sig("cpx_rays_upload_packed", [_vp, C.c_int64, C.c_int64, _vp, _vp])
_sig("cpx_rays_download", [_vp, C.c_int64, C.c_int64] + [_vp] * 17)
_sig("cpx_rays_init_camera", [_vp, _vp, C.POINTER(Camera), C.c_int, C.c_int, _u8p, _u8p, _u8p,
                              _vp, _i32p, C.c_int64, C.c_int64])
_sig("cpx_render_forward", [_vp, _vp, _vp, C.c_int, C.c_int, _vp])
_sig("cpx_render_backward", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_double, C.c_float, _vp])
_sig("cpx_render_forward_backward", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_double, C.c_float, _vp])
_sig("cpx_tv_grad", [_vp, C.c_double, C.c_double, C.c_int, C.c_int, _vp])
_sig("cpx_adam_step", [_vp, C.c_double, C.c_double, C.c_int, _vp])
_sig("cpx_tv_adam_step", [_vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _vp])
_sig("cpx_train_step", [_vp, _vp, _vp, C.c_int, C.c_int, C.POINTER(StepArgs), _vp,
                        C.POINTER(C.c_double), _vp])
_sig("cpx_train_step_ahead", [_vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp, C.c_int, C.c_int, C.POINTER(StepArgs), _vp,
                              C.POINTER(C.c_double), _vp])
_sig("cpx_last_sample_counts", [_vp, _i32p, C.c_int])
_sig("cpx_render_image", [_vp, C.POINTER(Camera), C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp])
_sig("cpx_image_mse", [_vp, _vp, C.c_int64, C.POINTER(C.c_double), _vp])
_sig("cpx_grid_touched_count", [_vp, C.POINTER(C.c_int64)])
_sig("cpx_grid_download_cell_map", [_vp, _vp, C.c_int64])


class ProposalDesc(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("confidence", C.c_float), ("label_weight", C.c_float),
                ("learning_rate", C.c_float)]


class ProposalSchedule(C.Structure):
    _fields_ = [("warmup", C.c_int), ("train_every", C.c_int), ("train_steps", C.c_int),
                ("rays_per_step", C.c_int)]


_sig("cpx_proposal_param_count", [])
_sig("cpx_proposal_create", [C.POINTER(ProposalDesc), C.POINTER(_vp)])
_sig("cpx_proposal_destroy", [_vp])
_sig("cpx_proposal_params", [_vp, _f32p, C.c_int])
_sig("cpx_proposal_infer", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp])
_sig("cpx_proposal_gradient", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _f32p, C.POINTER(C.c_double)])
_sig("cpx_proposal_train", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.POINTER(C.c_double),
                            _vp])
_sig("cpx_proposal_stats", [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int)])
_sig("cpx_render_forward_backward_guided", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_double, C.c_float, _vp, _vp,
                                            _vp])
_sig("cpx_render_forward_guided", [_vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp])
_sig("cpx_grid_set_options", [_vp, C.c_int])
_sig("cpx_grid_upsample", [_vp, _vp, C.c_float, C.c_int, _vp])
OPT_NO_EMPTY_SKIP = 1  # the FP32 march steps through empty cells one step at a time
OPT_FP32_MARCH = 2     # an FP32-storage grid marches like the mixed forms
OPT_NO_EARLY_STOP = 4  # the FP32 march runs every ray to its far bound (no transmittance stop)
OPT_FUSED_MARCH = 8  # placement and shading overlapped in one launch instead of two launches
OPT_PLANE_SWEEP = 16  # the FP32 dense sweep walking z with a tile's plane on chip instead of a block per row
OPT_SPLIT_SWEEP = 32  # the untouched vertices' sweep beside the shading, the touched ones after it
OPT_SPARSE_ADAM = 64  # mixed forms: the sweep updates the touched vertices only, in place
_sig("cpx_train_step_proposal", [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.POINTER(StepArgs), C.POINTER(ProposalSchedule),
                                 C.c_int, _vp, C.POINTER(C.c_double), _vp])


class BatchScene(C.Structure):
    _fields_ = [("grid", _vp), ("rays", _vp), ("rays_per_batch", C.c_int)]


class BatchTuning(C.Structure):
    _fields_ = [("place_block", C.c_int), ("shade_warps", C.c_int), ("grab", C.c_int), ("samples_per_step", C.c_int)]


_sig("cpx_ray_source_create", [C.c_void_p, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int,
                              C.POINTER(_vp)])
_sig("cpx_ray_source_destroy", [_vp])
_sig("cpx_ray_source_count", [_vp, C.POINTER(C.c_int64)])
_sig("cpx_ray_source_shuffle", [_vp, C.c_uint64, C.c_int])
_sig("cpx_ray_source_keys", [_vp, C.POINTER(C.c_uint32), C.POINTER(C.c_int)])
_sig("cpx_ray_source_generate", [_vp, _vp, C.c_int64, C.c_int, _vp, _vp])
_sig("cpx_ray_source_check", [_vp])
_sig("cpx_grid_save_text", [_vp, C.c_char_p, C.c_int, C.c_int, C.c_int])
_sig("cpx_grid_load_text", [_vp, C.c_char_p, C.c_int])
_sig("cpx_grid_load_text_sparse", [_vp, C.c_char_p, C.c_int])
_sig("cpx_grid_download_occupancy", [_vp, _vp, _vp, _vp, C.POINTER(C.c_uint32)])
_sig("cpx_image_load_text", [C.c_char_p, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_int)])
_sig("cpx_image_mask_pixels", [C.POINTER(C.c_int), C.c_int, _vp, C.POINTER(C.c_int64)])
_sig("cpx_carve_silhouette", [_vp, C.POINTER(C.c_double), C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp])
_sig("cpx_grid_bbox", [_vp, C.POINTER(C.c_int), C.POINTER(C.c_double)])
_sig("cpx_batch_create", [C.POINTER(BatchScene), C.c_int, C.POINTER(StepArgs), C.POINTER(_vp)])
_sig("cpx_batch_destroy", [_vp])
_sig("cpx_batch_step", [_vp, C.c_int, _vp])
_sig("cpx_batch_mse", [_vp, C.POINTER(C.c_double), _vp])
_sig("cpx_batch_check", [_vp])
_sig("cpx_batch_info", [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)])
_sig("cpx_batch_set_tuning", [_vp, C.POINTER(BatchTuning)])
_sig("cpx_batch_get_tuning", [_vp, C.POINTER(BatchTuning)])
_sig("cpx_batch_autotune", [_vp, C.c_int, C.POINTER(BatchTuning), _vp])


def _check(rc: int, where: str):
    if rc != 0:
        raise CpxError(rc, where)


def _ptr(x) -> int | None:
    """Device address of a CUDA tensor / integer, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        return x.data_ptr()
    raise TypeError(f"cannot take a device address of {type(x)}")


def _stream(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def kernel_launches() -> int:
    return int(_lib.cpx_kernel_launches())


def version() -> int:
    return int(_lib.cpx_version())


class ObjectScene:
    """Grid + optimizer state (objectScene, SceneUtils.cuh:4-98, and optimizer, Optimizer.cuh)."""

    def __init__(self, width, height, depth, sh_dim=9, optimizing_band=None, step_size=0.5,
                 hierarchy_strategy=False, bbox=None, precision="fp32", sr_seed=0):
        """precision: "fp32" (the reference's form) or the mixed forms "bf16" / "fp16" /
        "fp16full" (16-bit SH and moments -- bfloat16 moments in "bf16" and "fp16", half moments
        in "fp16full" -- FP32 density, gradients and march, stochastic rounding)."""
        if optimizing_band is None:
            optimizing_band = int(round(sh_dim ** 0.5)) - 1
        if bbox is None:  # initSelf: bbox spans the grid (SceneUtils.cu:107-112)
            bbox = (0, width - 1, 0, height - 1, 0, depth - 1)
        d = GridDesc()
        d.width, d.height, d.depth = int(width), int(height), int(depth)
        d.sh_dim = int(sh_dim)
        d.optimizing_band = int(optimizing_band)
        d.hierarchy_strategy = 1 if hierarchy_strategy else 0
        d.step_size = float(step_size)
        d.bbox[:] = [int(b) for b in bbox]
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        d.precision = PRECISIONS[precision]
        d.sr_seed = int(sr_seed) & 0xFFFFFFFF
        self.precision = precision
        self.desc = d
        self.width, self.height, self.depth = d.width, d.height, d.depth
        self.sh_dim = d.sh_dim
        self.optimizing_band = d.optimizing_band
        self.step_size = float(step_size)
        self.bbox = tuple(bbox)
        h = _vp()
        _check(_lib.cpx_grid_create(C.byref(d), C.byref(h)), "cpx_grid_create")
        self._h = h

    # -- bookkeeping
    @property
    def handle(self):
        return self._h

    def info(self):
        n = C.c_int64()
        a = C.c_int()
        s = C.c_int()
        _check(_lib.cpx_grid_info(self._h, C.byref(n), C.byref(a), C.byref(s)), "cpx_grid_info")
        return n.value, a.value, bool(s.value)

    @property
    def actual_grid_nums(self) -> int:
        return self.info()[0]

    @property
    def n_arrays(self) -> int:
        return 1 + 3 * self.sh_dim

    @property
    def sparse(self) -> bool:
        return self.info()[2]

    def close(self):
        if getattr(self, "_h", None):
            _lib.cpx_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameter blocks (planar [n_arrays][n_active], reference layout)
    def _planar(self, a):
        n = self.actual_grid_nums
        a = np.ascontiguousarray(a, dtype=np.float32)
        if a.size != self.n_arrays * n:
            raise ValueError(f"expected {self.n_arrays}x{n} floats, got shape {a.shape}")
        return a.reshape(self.n_arrays, n), n

    def upload_params(self, planar):
        a, n = self._planar(planar)
        _check(_lib.cpx_grid_upload_params(self._h, a, n), "cpx_grid_upload_params")

    def upload_params_device(self, planar_dev):
        """planar_dev: CUDA float32 tensor [n_arrays, n_active] (or [n_arrays*n_active])."""
        n = self.actual_grid_nums
        if planar_dev.numel() != self.n_arrays * n or not planar_dev.is_contiguous():
            raise ValueError("expected a contiguous CUDA tensor of n_arrays x n_active floats")
        _check(_lib.cpx_grid_upload_params_device(self._h, _ptr(planar_dev), n), "cpx_grid_upload_params_device")

    def download_params(self):
        n = self.actual_grid_nums
        out = np.empty((self.n_arrays, n), np.float32)
        _check(_lib.cpx_grid_download_params(self._h, out, n), "cpx_grid_download_params")
        return out

    def upload_grads(self, planar):
        a, n = self._planar(planar)
        _check(_lib.cpx_grid_upload_grads(self._h, a, n), "cpx_grid_upload_grads")

    def download_grads(self):
        n = self.actual_grid_nums
        out = np.empty((self.n_arrays, n), np.float32)
        _check(_lib.cpx_grid_download_grads(self._h, out, n), "cpx_grid_download_grads")
        return out

    def upload_moments(self, m, v):
        a, n = self._planar(m)
        b, _ = self._planar(v)
        _check(_lib.cpx_grid_upload_moments(self._h, a, b, n), "cpx_grid_upload_moments")

    def download_moments(self):
        n = self.actual_grid_nums
        m = np.empty((self.n_arrays, n), np.float32)
        v = np.empty((self.n_arrays, n), np.float32)
        _check(_lib.cpx_grid_download_moments(self._h, m, v, n), "cpx_grid_download_moments")
        return m, v

    def set_adaptive_lr(self, lr_mult):
        a = np.ascontiguousarray(lr_mult, dtype=np.float32).reshape(-1)
        _check(_lib.cpx_grid_set_adaptive_lr(self._h, a, a.size), "cpx_grid_set_adaptive_lr")

    def set_sample_offsets(self, ox, oy, oz):
        if ox is None or len(ox) == 0:
            _check(_lib.cpx_grid_set_sample_offsets(self._h, None, None, None, 0), "offsets")
            return
        arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (ox, oy, oz)]
        self._offsets_keep = arrs
        _check(_lib.cpx_grid_set_sample_offsets(self._h, *[a.ctypes.data for a in arrs], len(arrs[0])),
               "cpx_grid_set_sample_offsets")

    def fill_sample_offsets(self, radius: float, seeds, stream=None):
        """setSelfSampleOffset(radius) (SceneUtils.cu:792-798): the reference's scrambled-Sobol
        jitter offsets, from the three host rand() values its randGPU calls would draw."""
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        if sd.size != 3:
            raise ValueError("three seeds, one per axis")
        _check(_lib.cpx_grid_fill_sample_offsets(self._h, C.c_float(radius), sd.ctypes.data, _stream(stream)),
               "cpx_grid_fill_sample_offsets")

    def sample_offsets(self, n: int):
        """The first n jitter offsets per axis: (x, y, z) float64 arrays."""
        out = [np.zeros(n, np.float64) for _ in range(3)]
        _check(_lib.cpx_grid_download_sample_offsets(self._h, *[a.ctypes.data for a in out], int(n)),
               "cpx_grid_download_sample_offsets")
        return tuple(out)

    def set_optimize_step(self, step: int):
        _check(_lib.cpx_grid_set_optimize_step(self._h, int(step)), "cpx_grid_set_optimize_step")

    # -- occupancy (pruneSelf + getCagedNums, SceneUtils.cu:883, 1081)
    def prune_self(self, threshold: float, download: bool = True):
        """objectScene::pruneSelf + getCagedNums on the device.  Returns (occupancy, in_cage,
        index_offsets, in-cage count); with download=False only the count (the tables stay on
        the device)."""
        cnt = C.c_uint32()
        if not download:
            _check(_lib.cpx_occupancy_build(self._h, float(threshold), None, None, None, C.byref(cnt)),
                   "cpx_occupancy_build")
            return None, None, None, int(cnt.value)
        W, H, D = self.width, self.height, self.depth
        occ = np.empty((W - 1) * (H - 1) * (D - 1), np.uint8)
        cage = np.empty(W * H * D, np.uint8)
        idx = np.empty(W * H * D, np.uint32)
        _check(_lib.cpx_occupancy_build(self._h, float(threshold), occ.ctypes.data, cage.ctypes.data,
                                        idx.ctypes.data, C.byref(cnt)), "cpx_occupancy_build")
        return occ, cage, idx, int(cnt.value)

    def occupancy_tables(self):
        """The grid's current (occupancy, in_cage, index_offsets) tables."""
        W, H, D = self.width, self.height, self.depth
        occ = np.empty((W - 1) * (H - 1) * (D - 1), np.uint8)
        cage = np.empty(W * H * D, np.uint8)
        idx = np.empty(W * H * D, np.uint32)
        cnt = C.c_uint32()
        _check(_lib.cpx_grid_download_occupancy(self._h, occ.ctypes.data, cage.ctypes.data, idx.ctypes.data,
                                                C.byref(cnt)), "cpx_grid_download_occupancy")
        return occ, cage, idx

    def init_by_upsample(self, src: "ObjectScene", threshold: float, low_band_only: bool = False, stream=None):
        """upsampleScene of src into this (normally fresh) grid (SceneUtils.cu:419-485)."""
        _check(_lib.cpx_grid_upsample(src.handle, self._h, float(threshold), 1 if low_band_only else 0,
                                      _stream(stream)), "cpx_grid_upsample")

    def set_options(self, options: int):
        """March and sweep options (OPT_NO_EMPTY_SKIP, OPT_FP32_MARCH, OPT_NO_EARLY_STOP, OPT_FUSED_MARCH,
        OPT_PLANE_SWEEP, OPT_SPLIT_SWEEP, OPT_SPARSE_ADAM)."""
        _check(_lib.cpx_grid_set_options(self._h, int(options)), "cpx_grid_set_options")

    def touched_count(self) -> int:
        """Vertices whose gradient records the next optimizer sweep will read."""
        t = C.c_int64()
        _check(_lib.cpx_grid_touched_count(self._h, C.byref(t)), "cpx_grid_touched_count")
        return int(t.value)

    def cell_map(self) -> np.ndarray:
        """The march's dense empty-space map, one uint8 per cell (1 = open) in x-fastest order."""
        cells = (self.width - 1) * (self.height - 1) * (self.depth - 1)
        words = np.zeros((cells + 31) // 32, np.uint32)
        _check(_lib.cpx_grid_download_cell_map(self._h, words.ctypes.data, words.size), "cpx_grid_download_cell_map")
        return np.unpackbits(words.view(np.uint8), bitorder="little")[:cells]

    def make_sparse(self):
        _check(_lib.cpx_grid_make_sparse(self._h), "cpx_grid_make_sparse")

    def check(self):
        _check(_lib.cpx_grid_check(self._h), "cpx_grid_check")

    def last_sample_counts(self, n: int):
        out = np.empty(n, np.int32)
        _check(_lib.cpx_last_sample_counts(self._h, out, n), "cpx_last_sample_counts")
        return out


RAY_INPUTS = ("ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b")
RAY_OUTPUTS = ("acc_density", "acc_weights", "acc_r", "acc_g", "acc_b")
_FLOAT_FIELDS = set(RAY_INPUTS[:8]) | set(RAY_OUTPUTS)


class Rays:
    """Training-ray table (_rays, Rays.cuh:8-57)."""

    def __init__(self, total_rays: int, white_bg: bool = True):
        h = _vp()
        _check(_lib.cpx_rays_create(int(total_rays), 1 if white_bg else 0, C.byref(h)), "cpx_rays_create")
        self._h = h
        self.total_rays = int(total_rays)
        self.white_bg = bool(white_bg)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            _lib.cpx_rays_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, offset: int = 0, stream=None, **fields):
        count = None
        keep = []
        ptrs = []
        for name in RAY_INPUTS:
            if name in fields and fields[name] is not None:
                dt = np.float32 if name in _FLOAT_FIELDS else np.uint8
                a = np.ascontiguousarray(fields[name], dtype=dt).reshape(-1)
                count = a.size if count is None else count
                if a.size != count:
                    raise ValueError("ray fields differ in length")
                keep.append(a)
                ptrs.append(a.ctypes.data)
            else:
                ptrs.append(None)
        if count is None:
            return
        _check(_lib.cpx_rays_upload(self._h, int(offset), count, *ptrs, _stream(stream)), "cpx_rays_upload")

    def upload_packed(self, packed, offset: int = 0, stream=None):
        """packed: uint32 [count, 9] host array (pinned torch tensor or numpy)."""
        if hasattr(packed, "data_ptr"):
            count = packed.shape[0]
            ptr = packed.data_ptr()
        else:
            packed = np.ascontiguousarray(packed, dtype=np.uint32)
            count = packed.shape[0]
            ptr = packed.ctypes.data
        _check(_lib.cpx_rays_upload_packed(self._h, int(offset), int(count), ptr, _stream(stream)),
               "cpx_rays_upload_packed")

    def download(self, offset: int = 0, count: int | None = None, fields=None):
        if count is None:
            count = self.total_rays - offset
        names = list(RAY_INPUTS) + list(RAY_OUTPUTS)
        fields = names if fields is None else list(fields)
        out = {}
        ptrs = []
        for name in names:
            if name in fields:
                a = np.empty(count, np.float32 if name in _FLOAT_FIELDS else np.uint8)
                out[name] = a
                ptrs.append(a.ctypes.data)
            else:
                ptrs.append(None)
        _check(_lib.cpx_rays_download(self._h, int(offset), int(count), *ptrs), "cpx_rays_download")
        return out

    def initial_self(self, scene: ObjectScene, cameras, images, pixel_lists, img_w: int, img_h: int):
        """_rays::initialSelf (Rays.cu:187-240): cameras[i] with images[i] = (r, g, b, mask)
        planes of img_h*img_w bytes and pixel_lists[i] (row*img_w + col); rays of camera i
        follow those of camera i-1."""
        off = 0
        for cam, img, pix in zip(cameras, images, pixel_lists):
            r, g, b, m = (None if p is None else np.ascontiguousarray(p, np.uint8).reshape(-1) for p in img)
            pix = np.ascontiguousarray(pix, np.int32).reshape(-1)
            _check(_lib.cpx_rays_init_camera(self._h, scene.handle, C.byref(cam), int(img_w), int(img_h),
                                             r, g, b, None if m is None else m.ctypes.data, pix,
                                             pix.size, off), "cpx_rays_init_camera")
            off += pix.size
        return off


class RaySource:
    """Training samples (camera, pixel) whose rays are generated per batch on the device (no
    ray table); a drop-in for _rays::initialSelf + the training shuffle (Rays.cu:187-287)."""

    def __init__(self, cameras, images, img_w: int, img_h: int, pixel_lists=None, white_bg: bool = True):
        n = int(img_w) * int(img_h)
        cams = (Camera * len(cameras))(*cameras)
        planes = []
        for q in range(4):
            if q == 3 and any(img[3] is None for img in images):
                planes.append(None)
                continue
            planes.append(np.ascontiguousarray(np.stack([np.asarray(img[q], np.uint8).reshape(n) for img in images])))
        pix = npx = None
        if pixel_lists is not None:
            pix = np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32).reshape(-1) for p in pixel_lists]))
            npx = np.ascontiguousarray([len(p) for p in pixel_lists], np.int64)
        h = _vp()
        _check(_lib.cpx_ray_source_create(C.cast(cams, C.c_void_p), len(cameras), int(img_w), int(img_h),
                                          planes[0].ctypes.data, planes[1].ctypes.data, planes[2].ctypes.data,
                                          None if planes[3] is None else planes[3].ctypes.data,
                                          None if pix is None else pix.ctypes.data,
                                          None if npx is None else npx.ctypes.data, 1 if white_bg else 0,
                                          C.byref(h)), "cpx_ray_source_create")
        self._h = h
        self.white_bg = bool(white_bg)

    @property
    def handle(self):
        return self._h

    def __len__(self):
        n = C.c_int64()
        _check(_lib.cpx_ray_source_count(self._h, C.byref(n)), "cpx_ray_source_count")
        return int(n.value)

    def shuffle(self, seed: int, shuffled: bool = True):
        _check(_lib.cpx_ray_source_shuffle(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, 1 if shuffled else 0),
               "cpx_ray_source_shuffle")

    def keys(self):
        k = (C.c_uint32 * 4)()
        hb = C.c_int()
        _check(_lib.cpx_ray_source_keys(self._h, k, C.byref(hb)), "cpx_ray_source_keys")
        return [int(x) for x in k], int(hb.value)

    def generate(self, scene: ObjectScene, start: int, length: int, batch: Rays, stream=None):
        _check(_lib.cpx_ray_source_generate(self._h, scene.handle, int(start), int(length), batch.handle,
                                            _stream(stream)), "cpx_ray_source_generate")

    def check(self):
        _check(_lib.cpx_ray_source_check(self._h), "cpx_ray_source_check")

    def close(self):
        if getattr(self, "_h", None):
            _lib.cpx_ray_source_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _len(rays: Rays, start: int, length):
    return rays.total_rays - start if length is None else int(length)


class RenderUtils:
    """Per-batch march entry points (RenderUtils.cuh:7-85)."""

    @staticmethod
    def bbox_silhouette(projections, images, scene: "ObjectScene", img_w: int, img_h: int, radius: int = 0,
                        isGettingScaleRatio: bool = False, skipIndex=()):
        """RenderUtils::bbox_silhouette (RenderUtils.cu:323-478): carve with every camera not in
        skipIndex, then the bounding box (set as the grid's ray box); returns the scale ratio
        (0.0 unless isGettingScaleRatio)."""
        skip = set(int(i) for i in skipIndex)
        for i, (P, img) in enumerate(zip(projections, images)):
            if i not in skip:
                carve_silhouette(scene, P, img, img_w, img_h, radius)
        _, sr = grid_bbox(scene, isGettingScaleRatio)
        return sr if isGettingScaleRatio else 0.0

    @staticmethod
    def renderRays(rays: Rays, scene: ObjectScene, sampleIndex=None, startSampleIndex: int = 0,
                   len: int | None = None, stream=None):
        n = _len(rays, startSampleIndex, len)
        _check(_lib.cpx_render_forward(scene.handle, rays.handle, _ptr(sampleIndex),
                                       int(startSampleIndex), n, _stream(stream)), "renderRays")

    @staticmethod
    def renderRays_withGradients_RGB(scene: ObjectScene, rays: Rays, losses, sampleIndex=None,
                                     startSampleIndex: int = 0, len: int | None = None,
                                     maskRayLossCoefficient: float = 5.e-5, huberDelta: float = 0.01,
                                     stream=None):
        n = _len(rays, startSampleIndex, len)
        _check(_lib.cpx_render_backward(scene.handle, rays.handle, _ptr(losses), _ptr(sampleIndex),
                                        int(startSampleIndex), n, float(maskRayLossCoefficient),
                                        float(huberDelta), _stream(stream)),
               "renderRays_withGradients_RGB")

    @staticmethod
    def renderRays_forwardBackward(scene: ObjectScene, rays: Rays, losses, sampleIndex=None,
                                   startSampleIndex: int = 0, len: int | None = None,
                                   maskRayLossCoefficient: float = 5.e-5, huberDelta: float = 0.01,
                                   stream=None):
        n = _len(rays, startSampleIndex, len)
        _check(_lib.cpx_render_forward_backward(scene.handle, rays.handle, _ptr(losses), _ptr(sampleIndex),
                                                int(startSampleIndex), n, float(maskRayLossCoefficient),
                                                float(huberDelta), _stream(stream)),
               "renderRays_forwardBackward")

    @staticmethod
    def renderImage(scene: ObjectScene, camera: Camera, width: int, height: int, whiteBG: bool = True,
                    outputs=("rgb", "rgb8", "depth", "mask"), stream=None) -> dict:
        """Held-out view render (RenderUtils::renderImage, RenderUtils.cu:1802).  Returns CUDA
        tensors: rgb float32 [3, h*w], rgb8 uint8 [3, h*w], depth float32 [h*w], mask uint8
        [h*w] (those named in `outputs`).  Pixel p is at row p // width and column
        p % height, as the reference indexes it."""
        import torch

        n = int(width) * int(height)
        dev = torch.device("cuda", torch.cuda.current_device())
        shapes = {"rgb": ((3, n), torch.float32), "rgb8": ((3, n), torch.uint8),
                  "depth": ((n,), torch.float32), "mask": ((n,), torch.uint8)}
        out = {k: torch.empty(shapes[k][0], dtype=shapes[k][1], device=dev) for k in outputs}
        _check(_lib.cpx_render_image(scene.handle, C.byref(camera), int(width), int(height), int(bool(whiteBG)),
                                     _ptr(out.get("rgb")), _ptr(out.get("rgb8")), _ptr(out.get("depth")),
                                     _ptr(out.get("mask")), _stream(stream)), "renderImage")
        return out

    @staticmethod
    def addVarianceLoss(scene: ObjectScene, varianceCoefficient: float = 0.001,
                        shCoefficient: float = 0.001, varianceType: int = 0,
                        neighboorNums: int = 6, stream=None):
        _check(_lib.cpx_tv_grad(scene.handle, float(varianceCoefficient), float(shCoefficient),
                                int(varianceType), int(neighboorNums), _stream(stream)), "addVarianceLoss")


def _plane(p, n):
    if p is None:
        return None
    a = np.ascontiguousarray(p, np.uint8).reshape(-1)
    if a.size != n:
        raise ValueError(f"image plane of {a.size} bytes, expected {n}")
    return a


def carve_silhouette(scene: "ObjectScene", projection, image, img_w: int, img_h: int, radius: int = 0, stream=None):
    """silhouetteCarving (RenderUtils.cu:181-254) of one camera: projection is the camera's
    3x4 world-to-pixel matrix, image = (r, g, b, mask) planes of img_h*img_w bytes."""
    P = np.ascontiguousarray(projection, np.float64).reshape(12)
    n = int(img_w) * int(img_h)
    r, g, b, m = (_plane(p, n) for p in image)
    _check(_lib.cpx_carve_silhouette(scene.handle, P.ctypes.data_as(C.POINTER(C.c_double)), int(img_w), int(img_h),
                                     r.ctypes.data, g.ctypes.data, b.ctypes.data,
                                     None if m is None else m.ctypes.data, int(radius), _stream(stream)),
           "cpx_carve_silhouette")


def save_text(scene: "ObjectScene", directory: str, band: int, density_only: bool = False,
              hierarchy_mode: bool = False):
    """objectScene::saveSelf (SceneUtils.cu:1246-1300): the reference's text checkpoint."""
    _check(_lib.cpx_grid_save_text(scene.handle, str(directory).encode(), int(band), 1 if density_only else 0,
                                   1 if hierarchy_mode else 0), "cpx_grid_save_text")


def load_text(scene: "ObjectScene", directory: str, file_sh_dim: int):
    """objectScene::initFromFile (SceneUtils.cu:703-790), dense."""
    _check(_lib.cpx_grid_load_text(scene.handle, str(directory).encode(), int(file_sh_dim)), "cpx_grid_load_text")


def load_text_sparse(scene: "ObjectScene", directory: str, file_sh_dim: int):
    """objectScene::initFromFile (SceneUtils.cu:703-790), sparse with occupancy, into a fresh dense
    grid of the checkpoint's dimensions (which becomes sparse)."""
    _check(_lib.cpx_grid_load_text_sparse(scene.handle, str(directory).encode(), int(file_sh_dim)),
           "cpx_grid_load_text_sparse")


CONFIG_MAX_SKIPS = 256


class Config(C.Structure):
    """cpx_config: the reference's positional config.txt (readConfig, Utils.cu:765-932)."""
    _fields_ = [(n, C.c_int) for n in ("width", "height", "depth", "render_width", "render_height", "graylized",
                                       "sh_band", "hierarchy_band_strategy", "shs_for_target_resolution_only",
                                       "hierarchy", "minimum_hierarchy", "to_sparse_hierarchy", "silhouette_bound",
                                       "silhouette_initial", "silhouette_radius", "mask_area_only",
                                       "initial_from_file")] + [
        ("initial_file_dir_base", C.c_char * 512), ("available_sh_bands", C.c_int), ("render_only", C.c_int),
        ("views_directory", C.c_char * 512), ("camera_pose_file", C.c_char * 512),
        ("validation_pose_file", C.c_char * 512), ("novel_view_pose_file", C.c_char * 512),
        ("camera_distance", C.c_double)] + [(n, C.c_int) for n in (
            "view_count", "validation_count", "test_count", "train_process_view_index", "white_bg", "test_skip",
            "repeat_layers", "random_seed")] + [
        ("learning_rate", C.c_double), ("sh_learning_rate", C.c_double), ("density_optimizer", C.c_int),
        ("color_channel_optimizer", C.c_int), ("momentum", C.c_double), ("epochs", C.c_int),
        ("validation_interval", C.c_int), ("batch_size", C.c_int), ("fix_batch_size", C.c_int),
        ("base_dir", C.c_char * 512), ("save_intervals", C.c_int), ("half_lr_intervals", C.c_int),
        ("lowest_lr", C.c_double), ("prune_epoch", C.c_int), ("prune_threshold", C.c_float), ("skips", C.c_int),
        ("skip_index", C.c_int * CONFIG_MAX_SKIPS), ("step_size", C.c_float), ("solid_strategy", C.c_int),
        ("initial_density", C.c_float), ("initial_color", C.c_float), ("variance_loss_interval", C.c_int),
        ("variance_coefficient", C.c_double), ("sh_coefficient", C.c_double),
        ("mask_ray_coefficient", C.c_double), ("variance_type", C.c_int), ("neighbour_nums", C.c_int),
        ("diffuse_ratio", C.c_double), ("export_model", C.c_int), ("shuffle_rays", C.c_int),
        ("just_model", C.c_int), ("huber_delta", C.c_float)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, bytes):
                v = v.decode()
            elif name == "skip_index":
                v = [int(x) for x in v[:self.skips]]
            out[name] = v
        return out


_sig("cpx_config_read", [C.c_char_p, C.POINTER(Config)])


def read_config(path) -> dict:
    """readConfig (Utils.cu:765-932) without its side effects: the fields of config.txt."""
    c = Config()
    _check(_lib.cpx_config_read(str(path).encode(), C.byref(c)), "cpx_config_read")
    return c.as_dict()


def load_image_text(prefix: str, width: int, height: int, gray_only: bool = False, use_mask: bool = True):
    """Image::initSelfFromFile (ImageUtils.cu:84-128): planes (r, g, b, mask) or (gray, mask),
    the mask bounds, and the mask-area pixel list (processMasksInfo) when use_mask."""
    n = int(width) * int(height)
    planes = [np.zeros(n, np.uint8) for _ in range(5)]
    box = (C.c_int * 4)()
    _check(_lib.cpx_image_load_text(str(prefix).encode(), int(width), int(height), 1 if gray_only else 0,
                                    planes[0].ctypes.data, planes[1].ctypes.data, planes[2].ctypes.data,
                                    planes[3].ctypes.data, planes[4].ctypes.data, box), "cpx_image_load_text")
    pix = None
    if use_mask:
        cnt = C.c_int64()
        _check(_lib.cpx_image_mask_pixels(box, int(width), None, C.byref(cnt)), "cpx_image_mask_pixels")
        pix = np.zeros(cnt.value, np.int32)
        _check(_lib.cpx_image_mask_pixels(box, int(width), pix.ctypes.data, C.byref(cnt)), "cpx_image_mask_pixels")
    img = (planes[3], planes[4]) if gray_only else (planes[0], planes[1], planes[2], planes[4])
    return img, tuple(box[:]), pix


def grid_bbox(scene: "ObjectScene", scale_ratio: bool = False):
    """Bounding box of the uncarved vertices (getBoundingBoxZ + bbox_silhouette's reduction);
    it becomes the grid's ray box.  Returns (bbox tuple, scale ratio or None)."""
    box = (C.c_int * 6)()
    sr = C.c_double(0.0)
    _check(_lib.cpx_grid_bbox(scene.handle, box, C.byref(sr) if scale_ratio else None), "cpx_grid_bbox")
    scene.bbox = tuple(box[:])
    return tuple(box[:]), (sr.value if scale_ratio else None)


class Optimizer:
    """Adam step (Optimizer::updateRGBScene, Optimizer.cu:451-479)."""

    @staticmethod
    def updateRGBScene(scene: ObjectScene, learningRate: float, shLearningRate: float, timeStep: int,
                       stream=None):
        _check(_lib.cpx_adam_step(scene.handle, float(learningRate), float(shLearningRate), int(timeStep),
                                  _stream(stream)), "updateRGBScene")

    @staticmethod
    def varianceAndUpdate(scene: ObjectScene, varianceCoefficient: float, shCoefficient: float,
                          learningRate: float, shLearningRate: float, timeStep: int, stream=None):
        """TV type 0 / 6 neighbours fused with the Adam sweep."""
        _check(_lib.cpx_tv_adam_step(scene.handle, float(varianceCoefficient), float(shCoefficient),
                                     float(learningRate), float(shLearningRate), int(timeStep),
                                     _stream(stream)), "varianceAndUpdate")


def train_step(scene: ObjectScene, rays: Rays, losses, *, start: int = 0, length: int | None = None,
               sample_index=None, mask_coef: float = 1.0, huber_delta: float = 0.1, do_tv: bool = True,
               tv_type: int = 0, tv_neighbours: int = 6, lam_density: float = 1e-5,
               lam_sh: float = 1e-6, lr: float = 0.3, sh_lr: float = 1.0, timestep: int = 1,
               want_mse: bool = True, stream=None):
    """One batch of the reference's training loop (Render.cu:407-500); returns the batch MSE."""
    a = StepArgs()
    a.mask_coef = float(mask_coef)
    a.huber_delta = float(huber_delta)
    a.do_tv = 1 if do_tv else 0
    a.tv_type = int(tv_type)
    a.tv_neighbours = int(tv_neighbours)
    a.lam_density = float(lam_density)
    a.lam_sh = float(lam_sh)
    a.lr = float(lr)
    a.sh_lr = float(sh_lr)
    a.timestep = int(timestep)
    n = _len(rays, start, length)
    mse = C.c_double(0.0)
    _check(_lib.cpx_train_step(scene.handle, rays.handle, _ptr(sample_index), int(start), n, C.byref(a),
                               _ptr(losses), C.byref(mse) if want_mse else None, _stream(stream)),
           "train_step")
    return mse.value if want_mse else None


def train_step_ahead(scene: ObjectScene, rays: Rays, losses, *, start: int = 0, length: int | None = None,
                     sample_index=None, next_rays: Rays | None = None, next_start: int = 0, next_length: int = 0,
                     next_sample_index=None, mask_coef: float = 1.0, huber_delta: float = 0.1, do_tv: bool = True,
                     tv_type: int = 0, tv_neighbours: int = 6, lam_density: float = 1e-5, lam_sh: float = 1e-6,
                     lr: float = 0.3, sh_lr: float = 1.0, timestep: int = 1, want_mse: bool = True, stream=None):
    """train_step that also places the next batch's samples while the optimizer sweep runs (the
    next call with that batch shades it at once); returns the batch MSE."""
    a = StepArgs()
    a.mask_coef = float(mask_coef)
    a.huber_delta = float(huber_delta)
    a.do_tv = 1 if do_tv else 0
    a.tv_type = int(tv_type)
    a.tv_neighbours = int(tv_neighbours)
    a.lam_density = float(lam_density)
    a.lam_sh = float(lam_sh)
    a.lr = float(lr)
    a.sh_lr = float(sh_lr)
    a.timestep = int(timestep)
    n = _len(rays, start, length)
    mse = C.c_double(0.0)
    _check(_lib.cpx_train_step_ahead(scene.handle, rays.handle, _ptr(sample_index), int(start), n,
                                     None if next_rays is None else next_rays.handle, _ptr(next_sample_index),
                                     int(next_start), int(next_length), C.byref(a), _ptr(losses),
                                     C.byref(mse) if want_mse else None, _stream(stream)),
           "train_step_ahead")
    return mse.value if want_mse else None


def lr_decay(lr: float, batch_count: int, epoch: int) -> float:
    """Per-batch learning-rate decay of the reference (Render.cu:499-500)."""
    return lr / (2.0 ** (1.0 / batch_count / (epoch + 1.0)))


class Proposal:
    """Learned sample-interval proposal (no reference counterpart): 32 segments per ray,
    MLP 48 -> 64 -> 64 -> 64 -> 1 with BF16 tensor-core inference and FP32 training."""

    SEGMENTS = 32

    def __init__(self, seed=0, confidence=0.9, label_weight=1e-3, learning_rate=1e-3):
        d = ProposalDesc()
        d.seed, d.confidence, d.label_weight, d.learning_rate = int(seed), float(confidence), float(label_weight), \
            float(learning_rate)
        self.desc = d
        h = _vp()
        _check(_lib.cpx_proposal_create(C.byref(d), C.byref(h)), "cpx_proposal_create")
        self._h = h
        self.n_params = int(_lib.cpx_proposal_param_count())

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            _lib.cpx_proposal_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.empty(self.n_params, np.float32)
        _check(_lib.cpx_proposal_params(self._h, out, 0), "cpx_proposal_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32).copy()
        _check(_lib.cpx_proposal_params(self._h, p, 1), "cpx_proposal_params")

    def infer(self, scene, rays, start=0, length=None, sample_index=None, tensor_cores=True, stream=None):
        """(logits [len, 32], masks [len] uint32 as int32) CUDA tensors."""
        import torch

        n = _len(rays, start, length)
        dev = torch.device("cuda", torch.cuda.current_device())
        logits = torch.empty((n, self.SEGMENTS), dtype=torch.float32, device=dev)
        masks = torch.empty(n, dtype=torch.int32, device=dev)
        _check(_lib.cpx_proposal_infer(self._h, scene.handle, rays.handle, _ptr(sample_index), int(start), n,
                                       _ptr(logits), _ptr(masks), 1 if tensor_cores else 0, _stream(stream)),
               "cpx_proposal_infer")
        return logits, masks

    def masks_into(self, scene, rays, masks, start=0, length=None, sample_index=None, stream=None):
        """Segment masks of a batch into a preallocated int32 CUDA tensor (no logits)."""
        n = _len(rays, start, length)
        _check(_lib.cpx_proposal_infer(self._h, scene.handle, rays.handle, _ptr(sample_index), int(start), n, None,
                                       _ptr(masks), 1, _stream(stream)), "cpx_proposal_infer")

    def gradient(self, scene, rays, seg_weights, start=0, length=None, sample_index=None):
        n = _len(rays, start, length)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        _check(_lib.cpx_proposal_gradient(self._h, scene.handle, rays.handle, _ptr(sample_index), int(start), n,
                                          _ptr(seg_weights), g, C.byref(loss)), "cpx_proposal_gradient")
        return g, loss.value

    def train(self, scene, rays, seg_weights, steps, rays_per_step=0, start=0, length=None, sample_index=None,
              stream=None, want_loss=True):
        """Adam steps on the labels of seg_weights; returns the mean loss (synchronises) or None."""
        n = _len(rays, start, length)
        loss = C.c_double()
        _check(_lib.cpx_proposal_train(self._h, scene.handle, rays.handle, _ptr(sample_index), int(start), n,
                                       _ptr(seg_weights), int(steps), int(rays_per_step),
                                       C.byref(loss) if want_loss else None, _stream(stream)), "cpx_proposal_train")
        return loss.value if want_loss else None

    def stats(self):
        r, c, f = C.c_int(), C.c_int64(), C.c_int()
        _check(_lib.cpx_proposal_stats(self._h, C.byref(r), C.byref(c), C.byref(f)), "cpx_proposal_stats")
        return {"rounds": r.value, "skipped_segments": c.value, "error_flags": f.value}


def render_guided(scene: ObjectScene, rays: Rays, losses, start=0, length=None, sample_index=None, mask_coef=1.0,
                  huber_delta=0.1, masks=None, seg_weights=None, stream=None):
    """The mixed-form march guided by per-ray segment masks and/or recording segment weights."""
    n = _len(rays, start, length)
    _check(_lib.cpx_render_forward_backward_guided(scene.handle, rays.handle, _ptr(losses), _ptr(sample_index),
                                                   int(start), n, float(mask_coef), float(huber_delta),
                                                   _ptr(masks), _ptr(seg_weights), _stream(stream)),
           "cpx_render_forward_backward_guided")


def render_forward_guided(scene: ObjectScene, rays: Rays, start=0, length=None, sample_index=None, masks=None,
                          stream=None):
    """Forward of the mixed forms' march (guided by segment masks when given)."""
    n = _len(rays, start, length)
    _check(_lib.cpx_render_forward_guided(scene.handle, rays.handle, _ptr(sample_index), int(start), n, _ptr(masks),
                                          _stream(stream)), "cpx_render_forward_guided")


def train_step_proposal(scene: ObjectScene, rays: Rays, proposal: Proposal, losses, iteration: int, *, start=0,
                        length=None, sample_index=None, mask_coef=1.0, huber_delta=0.1, do_tv=True,
                        lam_density=1e-5, lam_sh=1e-6, lr=0.3, sh_lr=1.0, timestep=1, warmup=0, train_every=50,
                        train_steps=16, rays_per_step=1024, want_mse=True, stream=None):
    """One batch of the mixed form with the learned proposal; returns the batch MSE."""
    a = StepArgs()
    a.mask_coef, a.huber_delta, a.do_tv, a.tv_type, a.tv_neighbours = float(mask_coef), float(huber_delta), \
        1 if do_tv else 0, 0, 6
    a.lam_density, a.lam_sh, a.lr, a.sh_lr, a.timestep = float(lam_density), float(lam_sh), float(lr), \
        float(sh_lr), int(timestep)
    sch = ProposalSchedule()
    sch.warmup, sch.train_every, sch.train_steps, sch.rays_per_step = int(warmup), int(train_every), \
        int(train_steps), int(rays_per_step)
    n = _len(rays, start, length)
    mse = C.c_double(0.0)
    _check(_lib.cpx_train_step_proposal(scene.handle, rays.handle, proposal.handle, _ptr(sample_index), int(start), n,
                                        C.byref(a), C.byref(sch), int(iteration), _ptr(losses),
                                        C.byref(mse) if want_mse else None, _stream(stream)),
           "cpx_train_step_proposal")
    return mse.value if want_mse else None


def step_args(*, mask_coef: float = 1.0, huber_delta: float = 0.1, do_tv: bool = True, tv_type: int = 0,
              tv_neighbours: int = 6, lam_density: float = 1e-5, lam_sh: float = 1e-6, lr: float = 0.3,
              sh_lr: float = 1.0, timestep: int = 1) -> StepArgs:
    a = StepArgs()
    a.mask_coef, a.huber_delta, a.do_tv = float(mask_coef), float(huber_delta), 1 if do_tv else 0
    a.tv_type, a.tv_neighbours = int(tv_type), int(tv_neighbours)
    a.lam_density, a.lam_sh, a.lr, a.sh_lr, a.timestep = float(lam_density), float(lam_sh), float(lr), \
        float(sh_lr), int(timestep)
    return a


class Batch:
    """Batched multi-scene training (no reference counterpart): every scene of the batch
    steps together, one placement and one shading launch over all their rays, then each
    scene's TV + Adam sweep.  Iteration i of a scene trains on rays
    [(i % pool) * len, (i + 1) * len) of its ray table with Adam timestep i + 1, exactly as
    train_step(start=(i % pool) * len, timestep=i + 1) on that scene alone."""

    def __init__(self, scenes, **step_kw):
        """scenes: (ObjectScene, Rays, rays_per_batch) triples; step_kw as train_step's."""
        self.scenes = list(scenes)
        arr = (BatchScene * len(self.scenes))()
        for i, (sc, r, n) in enumerate(self.scenes):
            arr[i].grid, arr[i].rays, arr[i].rays_per_batch = sc.handle, r.handle, int(n)
        self.args = step_args(**step_kw)
        h = _vp()
        _check(_lib.cpx_batch_create(arr, len(self.scenes), C.byref(self.args), C.byref(h)), "cpx_batch_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            _lib.cpx_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, graphs: bool = True, stream=None):
        _check(_lib.cpx_batch_step(self._h, 1 if graphs else 0, _stream(stream)), "cpx_batch_step")

    def mse(self, stream=None) -> np.ndarray:
        out = (C.c_double * len(self.scenes))()
        _check(_lib.cpx_batch_mse(self._h, out, _stream(stream)), "cpx_batch_mse")
        return np.array(out[:], np.float64)

    def check(self):
        _check(_lib.cpx_batch_check(self._h), "cpx_batch_check")

    def info(self) -> dict:
        it, tot, lps = C.c_int(0), C.c_int(0), C.c_int(0)
        _check(_lib.cpx_batch_info(self._h, C.byref(it), C.byref(tot), C.byref(lps)), "cpx_batch_info")
        return {"iteration": it.value, "total_rays": tot.value, "launches_per_step": lps.value}

    @property
    def tuning(self) -> dict:
        t = BatchTuning()
        _check(_lib.cpx_batch_get_tuning(self._h, C.byref(t)), "cpx_batch_get_tuning")
        return {"place_block": t.place_block, "shade_warps": t.shade_warps, "grab": t.grab,
                "samples_per_step": t.samples_per_step}

    def set_tuning(self, place_block: int, shade_warps: int, grab: int, samples_per_step: int = 1):
        t = BatchTuning()
        t.place_block, t.shade_warps, t.grab = int(place_block), int(shade_warps), int(grab)
        t.samples_per_step = int(samples_per_step)
        _check(_lib.cpx_batch_set_tuning(self._h, C.byref(t)), "cpx_batch_set_tuning")

    def autotune(self, steps_per_trial: int = 3, stream=None) -> dict:
        t = BatchTuning()
        _check(_lib.cpx_batch_autotune(self._h, int(steps_per_trial), C.byref(t), _stream(stream)),
               "cpx_batch_autotune")
        return {"place_block": t.place_block, "shade_warps": t.shade_warps, "grab": t.grab,
                "samples_per_step": t.samples_per_step}


def image_mse(a, b, stream=None) -> float:
    """Mean squared difference of two float32 CUDA tensors of equal size (double sums)."""
    if (a.numel() != b.numel() or str(a.dtype) != "torch.float32" or str(b.dtype) != "torch.float32"
            or not a.is_contiguous() or not b.is_contiguous()):
        raise ValueError("image_mse wants two contiguous tensors of the same size and dtype")
    out = C.c_double(0.0)
    _check(_lib.cpx_image_mse(_ptr(a), _ptr(b), int(a.numel()), C.byref(out), _stream(stream)), "image_mse")
    return out.value


def image_psnr(a, b, stream=None) -> float:
    """PSNR of two images in [0, 1]: 10 log10(1 / mse)."""
    return float(10.0 * np.log10(1.0 / image_mse(a, b, stream)))


def psnr_from_mse(mse: float) -> float:
    """PSNR on the 255^2 scale of the per-ray loss (Render.cu:465)."""
    return 10.0 * np.log10(65025.0 / mse)
