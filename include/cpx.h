/*
 * cpx.h -- C ABI of the B200-native Clear-plenoxels training hot path.
 *
 * A drop-in for the reference's per-batch entry points (citations are
 * file:line in the reference project, SVRF = SparseVolumeRadianceField/):
 *
 *   cpx_render_forward           RenderUtils::renderRays                     SVRF/RenderUtils.cuh:37, .cu:1961
 *   cpx_render_backward          RenderUtils::renderRays_withGradients_RGB   SVRF/RenderUtils.cuh:51, .cu:2258
 *   cpx_tv_grad                  RenderUtils::addVarianceLoss                SVRF/RenderUtils.cuh:76, .cu:2815
 *   cpx_adam_step                Optimizer::updateRGBScene                   SVRF/Optimizer.cuh:35, .cu:451
 *   cpx_grid_create/upload       objectScene::initSelf, optimizer::initialSelf/initialAll
 *                                                                            SVRF/SceneUtils.cu:60, Optimizer.cu:81,163
 *   cpx_occupancy_build          objectScene::pruneSelf + getCagedNums       SVRF/SceneUtils.cu:883, 1081
 *   cpx_grid_make_sparse         sparse compaction of initSelfByUpsample     SVRF/SceneUtils.cu:520-600
 *   cpx_rays_init_camera         _rays::initialSelf / initialRays            SVRF/Rays.cu:187, 77
 *
 * Conventions.  Every call returns a cpx_status instead of exiting the
 * process.  Work is enqueued on the caller's stream (a cudaStream_t passed as
 * void*, NULL = legacy default stream) with no implicit device synchronisation;
 * only the host upload/download calls block.  Grid and ray buffers are owned
 * by the library behind opaque handles; host arrays are copied.  Arrays named
 * *_dev are device pointers, exactly where the reference takes device
 * pointers (sample index table, per-ray losses).  A handle is used by one host
 * thread at a time.
 *
 * Parameter order follows the reference's totalVariableGPUPtrs table
 * (SVRF/SceneUtils.cu:148-166): array 0 is density, arrays 1+c*sh_dim+i are
 * SH coefficient i of colour channel c (R, G, B).  Host parameter blocks are
 * planar float [n_arrays][n_active], the layout the reference keeps on device.
 */
#ifndef CPX_H
#define CPX_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cpx_status {
    CPX_OK = 0,
    CPX_ERR_INVALID_ARGUMENT = 1,
    CPX_ERR_OUT_OF_MEMORY = 2,
    CPX_ERR_CUDA = 3,
    CPX_ERR_ITERATION_CAP = 4, /* a ray's march exceeded its provable sample bound */
    CPX_ERR_NAN = 5,           /* reserved: NaN detected where a caller asked for a check */
    CPX_ERR_NOT_READY = 6,     /* e.g. sparse call before cpx_occupancy_build */
    CPX_ERR_UNSUPPORTED = 7
} cpx_status;

typedef void* cpx_stream; /* cudaStream_t */
typedef struct cpx_grid cpx_grid;
typedef struct cpx_rays cpx_rays;

typedef struct cpx_grid_desc {
    int width, height, depth; /* vertices per axis (sceneWidth/Height/Depth) */
    int sh_dim;               /* SH coefficients per channel: 1, 4 or 9 */
    int optimizing_band;      /* ObjectScene::optimizingBand; forward uses (band+1)^2 <= sh_dim */
    int hierarchy_strategy;   /* Optimizer::hierarchyStrategy (band-restricted grads/updates) */
    float step_size;          /* ObjectScene::stepSize, > 0 */
    int bbox[6];              /* ray AABB in voxel space: wmin,wmax,hmin,hmax,dmin,dmax */
    int precision;            /* cpx_precision: storage and march form (no reference
                                 counterpart beyond CPX_PRECISION_FP32, its own form) */
    uint32_t sr_seed;         /* seed of the stochastic rounding of the 16-bit forms */
} cpx_grid_desc;

/* Storage forms.  FP32 is the reference's (every parameter and moment in float, the march
 * in the reference's FP64/FP32 mix, bit-compatible with it).  The mixed forms store the SH
 * coefficients in bfloat16 (BF16) or half (FP16 and FP16_FULL) and both Adam moments in
 * bfloat16 (BF16, FP16) or half (FP16_FULL: the first moment as m * 2^8, the second through
 * its root, sqrt(v) * 2^8, since v spans more decades than half holds; stores saturate at
 * 255.9), keep density, gradients and all accumulation in FP32, march in FP32, and write the
 * optimizer results back with stochastic rounding.  They support TV type 0 with 6 neighbours,
 * fused into the optimizer sweep (cpx_tv_adam_step / cpx_train_step), or no TV. */
typedef enum cpx_precision {
    CPX_PRECISION_FP32 = 0,
    CPX_PRECISION_BF16 = 1,
    CPX_PRECISION_FP16 = 2,
    CPX_PRECISION_FP16_FULL = 3
} cpx_precision;

/* Pinhole camera as the reference's getBound reads it (SVRF/CameraUtils.cuh:16-26):
 * focal lengths, principal point, camera-to-world 4x4 (row-major) and centre. */
typedef struct cpx_camera {
    double alpha[2];
    double principle[2];
    double c2w[16];
    double centre[4];
} cpx_camera;

/* ------------------------------------------------------------------ status */
const char* cpx_status_string(cpx_status s);
/* Text of the last error raised on the calling thread ("" if none). */
const char* cpx_last_error(void);
/* Library version as major*10000 + minor*100 + patch. */
int cpx_version(void);

/* ------------------------------------------------------------------ configuration */
/* The reference's positional config.txt (readConfig, SVRF/Utils.cu:765-932; Configuration,
 * SVRF/Utils.cuh): every key in the reference's order, one per line ("SceneSize:512 512 512").
 * Flags are 0/1 as the reference's bools hold them; strings are at most 511 bytes. */
#define CPX_CONFIG_MAX_SKIPS 256
typedef struct cpx_config {
    int width, height, depth;                 /* SceneSize */
    int render_width, render_height;          /* RenderSize */
    int graylized;                            /* Graylized */
    int sh_band;                              /* SphericalHarmonicsBand */
    int hierarchy_band_strategy;              /* HierarchyBandStrategy */
    int shs_for_target_resolution_only;       /* SHsForTargetResolutionOnly */
    int hierarchy, minimum_hierarchy;         /* Hierarchy, MinimumHierarchy */
    int to_sparse_hierarchy;                  /* ToSparseHierarchy */
    int silhouette_bound, silhouette_initial; /* SilhouetteBound, SilhouetteInitial */
    int silhouette_radius;                    /* SilhouetteRadius */
    int mask_area_only;                       /* MaskAreaOnly */
    int initial_from_file;                    /* InitialFromFile */
    char initial_file_dir_base[512];          /* InitialFileDirBase */
    int available_sh_bands;                   /* AvailableSHBands */
    int render_only;                          /* RenderOnly */
    char views_directory[512];                /* ViewDirectory */
    char camera_pose_file[512];               /* CameraPoseFile */
    char validation_pose_file[512];           /* ValidationPoseFile */
    char novel_view_pose_file[512];           /* NovelViewPoseFile */
    double camera_distance;                   /* CameraDistance */
    int view_count, validation_count;         /* ViewCount, ValidationCount */
    int test_count;                           /* TestCount */
    int train_process_view_index;             /* TrainProcessViewIndex */
    int white_bg;                             /* WhiteBG */
    int test_skip, repeat_layers;             /* TestSkip, RepeatLayers */
    int random_seed;                          /* RandomSeed */
    double learning_rate, sh_learning_rate;   /* LearningRate, SHLearningRate */
    int density_optimizer;                    /* DensityOptimizer */
    int color_channel_optimizer;              /* ColorChannelOptimizer */
    double momentum;                          /* Momentum */
    int epochs, validation_interval;          /* Epochs, ValidationInterval */
    int batch_size, fix_batch_size;           /* BatchSize, FixBatchSize */
    char base_dir[512];                       /* BaseDir */
    int save_intervals, half_lr_intervals;    /* SaveIntervals, HalfLR */
    double lowest_lr;                         /* LowestLR */
    int prune_epoch;                          /* PruneEpoch */
    float prune_threshold;                    /* PruneThreshold */
    int skips;                                /* Skips */
    int skip_index[CPX_CONFIG_MAX_SKIPS];     /* SkipIndex (the first `skips`) */
    float step_size;                          /* StepSize */
    int solid_strategy;                       /* SolidStrategy */
    float initial_density, initial_color;     /* InitialDensity, InitialColor */
    int variance_loss_interval;               /* VarianceLossInterval */
    double variance_coefficient;              /* VarianceCoefficient (TV lambda, density) */
    double sh_coefficient;                    /* ColorDisparityCoefficient (TV lambda, SH) */
    double mask_ray_coefficient;              /* MaskRayCoefficient */
    int variance_type, neighbour_nums;        /* VarianceType, NeighboorNumsForTVLoss */
    double diffuse_ratio;                     /* DiffuseRatio */
    int export_model, shuffle_rays;           /* ExportModel, ShuffleRays */
    int just_model;                           /* JustModel */
    float huber_delta;                        /* HuberDelta */
} cpx_config;
/* Parses `path` as readConfig does, without its side effects (no directories created, no
 * files copied, rand() not seeded).  CPX_ERR_INVALID_ARGUMENT names the first line that is
 * missing or out of order (where the reference reads on with fields unset). */
cpx_status cpx_config_read(const char* path, cpx_config* out);

/* ------------------------------------------------------------------ grid */
/* Dense grid, every parameter zero, Adam moments zero, adaptive LR one, no jitter.
 * Replaces objectScene::initSelf(solid) + optimizer::initialSelf/initialAll. */
cpx_status cpx_grid_create(const cpx_grid_desc* desc, cpx_grid** out);
cpx_status cpx_grid_destroy(cpx_grid* g);
/* n_active: W*H*D (dense) or the in-cage count (sparse); n_arrays = 1 + 3*sh_dim. */
cpx_status cpx_grid_info(const cpx_grid* g, int64_t* n_active, int* n_arrays, int* sparse);

/* Planar [n_arrays][n_active] host copies of parameters, gradients and moments. */
cpx_status cpx_grid_upload_params(cpx_grid* g, const float* planar, int64_t n_active);
cpx_status cpx_grid_download_params(const cpx_grid* g, float* planar, int64_t n_active);
/* Same as cpx_grid_upload_params from a planar block already in device memory. */
cpx_status cpx_grid_upload_params_device(cpx_grid* g, const float* planar_dev, int64_t n_active);
cpx_status cpx_grid_upload_grads(cpx_grid* g, const float* planar, int64_t n_active);
cpx_status cpx_grid_download_grads(const cpx_grid* g, float* planar, int64_t n_active);
cpx_status cpx_grid_upload_moments(cpx_grid* g, const float* m, const float* v, int64_t n_active);
cpx_status cpx_grid_download_moments(const cpx_grid* g, float* m, float* v, int64_t n_active);
/* Density LR multiplier (ObjectScene::adaptiveLRDevice), [W*H*D]; dense Adam only. */
cpx_status cpx_grid_set_adaptive_lr(cpx_grid* g, const float* lr_mult, int64_t n_dense);
/* Per-sample jitter offsets (ObjectScene::offset{X,Y,Z}Device, filled by setSelfSampleOffset,
 * SVRF/SceneUtils.cu:792); entries past n read as zero.  n = 0 clears them. */
cpx_status cpx_grid_set_sample_offsets(cpx_grid* g, const double* ox, const double* oy,
                                       const double* oz, int n);
/* objectScene::setSelfSampleOffset(radius) (SVRF/SceneUtils.cu:792-798, randGPU at
 * SVRF/Utils.cu:1002-1044): fills the grid's three offset arrays (maxSamplePoint =
 * (int)(sqrt(W^2+H^2+D^2)/step + 1.5) entries, zero when first created) with
 * N(0,1)/4 * radius from cuRAND's scrambled Sobol64 generator, exactly as the reference
 * does.  seeds[3] are the three host rand() values the reference's three randGPU calls
 * would draw (each axis's generator starts at point state + seed).  The reference calls it
 * before every batch with radius = stepSize/2 when SolidStrategy is 0.  Asynchronous on
 * `stream` after the first call (which fetches cuRAND's direction numbers). */
cpx_status cpx_grid_fill_sample_offsets(cpx_grid* g, float radius, const uint32_t* seeds, cpx_stream stream);
/* Host copy of the first n jitter offsets per axis (n at most the grid's offset count).
 * Synchronous.  No reference counterpart beyond reading offset{X,Y,Z}Device. */
cpx_status cpx_grid_download_sample_offsets(const cpx_grid* g, double* ox, double* oy, double* oz, int n);
/* ObjectScene::optimizeStep (hierarchy level); gates SH in the type-1 TV term. */
cpx_status cpx_grid_set_optimize_step(cpx_grid* g, int optimize_step);

/* ------------------------------------------------------------------ occupancy */
/* From the dense density: occupancy per cell ((W-1)(H-1)(D-1) bytes), in-cage flag per
 * vertex and the in-cage prefix index (0 when not in cage), exactly as pruneScene
 * (SVRF/SceneUtils.cu:831) and getCagedNums (SVRF/SceneUtils.cu:1081).  Optional host
 * outputs may be NULL.  The grid stays dense until cpx_grid_make_sparse. */
cpx_status cpx_occupancy_build(cpx_grid* g, float threshold, uint8_t* occupancy_out,
                               uint8_t* in_cage_out, uint32_t* index_offsets_out,
                               uint32_t* in_cage_count_out);
/* Host copies of the grid's current occupancy tables (those of the last cpx_occupancy_build,
 * or of a loaded sparse checkpoint); any output may be NULL.  CPX_ERR_NOT_READY without
 * tables.  Synchronous.  (The reference keeps them as occupancyHost / inCageInfoHost /
 * indexOffsetsHost, SVRF/SceneUtils.cuh:4-98.) */
cpx_status cpx_grid_download_occupancy(const cpx_grid* g, uint8_t* occupancy_out, uint8_t* in_cage_out,
                                       uint32_t* index_offsets_out, uint32_t* in_cage_count_out);
/* Switch to the sparse layout of the last cpx_occupancy_build: parameters compacted in
 * z-y-x order of the in-cage flags, optimizer state reset to zero. */
cpx_status cpx_grid_make_sparse(cpx_grid* g);

/* ------------------------------------------------------------------ rays */
cpx_status cpx_rays_create(int64_t n_rays, int white_bg, cpx_rays** out);
cpx_status cpx_rays_destroy(cpx_rays* r);
/* Rays [offset, offset+count) from host SoA arrays (the 12 input fields of _rays). */
cpx_status cpx_rays_upload(cpx_rays* r, int64_t offset, int64_t count, const float* ox,
                           const float* oy, const float* oz, const float* dx, const float* dy,
                           const float* dz, const float* near_t, const float* far_t,
                           const uint8_t* gt_mask, const uint8_t* gt_r, const uint8_t* gt_g,
                           const uint8_t* gt_b, cpx_stream stream);
/* Rays [offset, offset+count) from one packed host array of 9 32-bit words per ray:
 * ox, oy, oz, dx, dy, dz, near, far (float) and the ground truth r, g, b, mask bytes
 * packed little-endian into the ninth word.  One host-to-device copy per call. */
cpx_status cpx_rays_upload_packed(cpx_rays* r, int64_t offset, int64_t count,
                                  const uint32_t* packed, cpx_stream stream);
/* Download any subset of the 17 fields (NULL skips a field). */
cpx_status cpx_rays_download(const cpx_rays* r, int64_t offset, int64_t count, float* ox,
                             float* oy, float* oz, float* dx, float* dy, float* dz,
                             float* near_t, float* far_t, uint8_t* gt_mask, uint8_t* gt_r,
                             uint8_t* gt_g, uint8_t* gt_b, float* acc_density,
                             float* acc_weights, float* acc_r, float* acc_g, float* acc_b);
/* Rays of one camera for the listed pixels (row*img_w+col), written at [offset, offset+n_pix):
 * getBound + initialRays (SVRF/Rays.cu:22-144) on the device.  Image planes are host
 * arrays of img_w*img_h bytes; gt_mask may be NULL (treated as 255). */
cpx_status cpx_rays_init_camera(cpx_rays* r, const cpx_grid* g, const cpx_camera* cam,
                                int img_w, int img_h, const uint8_t* red, const uint8_t* green,
                                const uint8_t* blue, const uint8_t* gt_mask,
                                const int32_t* pixel_index, int64_t n_pix, int64_t offset);

/* Ray source (no ray table): the training samples (camera, pixel) of n_cams cameras whose
 * images stay on the device; each batch's rays are generated on the device, bit for bit the
 * rays cpx_rays_init_camera makes (getBound + initialRays, SVRF/Rays.cu:22-144), replacing
 * _rays::initialSelf's table of every ray and the host shuffle (ShuffleRank + shuffleTo,
 * SVRF/Utils.cu:488, Rays.cu:242).  Planes are host arrays [n_cams][img_w*img_h] (gt_mask may
 * be NULL: 255); pixel_index concatenates each camera's pixel list (n_pix[c] entries; NULL:
 * every pixel of every camera).  Sample i of an epoch is permute(i): the identity, or after
 * cpx_ray_source_shuffle(seed, 1) a keyed bijection of [0, n) (4-round Feistel network with
 * cycle walking; the keys come from seed through SplitMix64). */
typedef struct cpx_ray_source cpx_ray_source;
cpx_status cpx_ray_source_create(const cpx_camera* cams, int n_cams, int img_w, int img_h, const uint8_t* red,
                                 const uint8_t* green, const uint8_t* blue, const uint8_t* gt_mask,
                                 const int32_t* pixel_index, const int64_t* n_pix, int white_bg,
                                 cpx_ray_source** out);
cpx_status cpx_ray_source_destroy(cpx_ray_source* s);
cpx_status cpx_ray_source_count(const cpx_ray_source* s, int64_t* n);
/* New epoch order: shuffled = 0 restores the identity. */
cpx_status cpx_ray_source_shuffle(cpx_ray_source* s, uint64_t seed, int shuffled);
/* The permutation's round keys [4] and half width (for checking it on the host). */
cpx_status cpx_ray_source_keys(const cpx_ray_source* s, uint32_t* keys, int* half_bits);
/* Rays of samples permute(start .. start+len) into batch[0 .. len), with the grid's ray box. */
cpx_status cpx_ray_source_generate(cpx_ray_source* s, const cpx_grid* g, int64_t start, int len, cpx_rays* batch,
                                   cpx_stream stream);
/* Synchronise and report a shuffle whose cycle walk ran out of steps (none expected). */
cpx_status cpx_ray_source_check(cpx_ray_source* s);

/* ------------------------------------------------------------------ per-batch path */
/* Batch = rays sample_index_dev[start .. start+len) (identity when NULL).
 * Forward march: accumulated density, weight and RGB (+white background) per ray. */
cpx_status cpx_render_forward(cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev,
                              int start, int len, cpx_stream stream);
/* Backward: per-ray loss into losses_dev[0..len) and gradients accumulated into the grid. */
cpx_status cpx_render_backward(cpx_grid* g, cpx_rays* r, double* losses_dev,
                               const int32_t* sample_index_dev, int start, int len,
                               double mask_coef, float huber_delta, cpx_stream stream);
/* Forward and backward of one batch in one pass over the samples (same results as the
 * two calls above in sequence). */
cpx_status cpx_render_forward_backward(cpx_grid* g, cpx_rays* r, double* losses_dev,
                                       const int32_t* sample_index_dev, int start, int len,
                                       double mask_coef, float huber_delta, cpx_stream stream);
/* The same forward+backward as cpx_render_forward_backward without allocating device
 * memory.  No counterpart in the reference: it is for callers that cannot allocate while
 * they run -- a host whose own pool allocator owns the device memory, or a loop that may
 * not allocate once it has started.  Its sample scratch is one fixed array (about 48 MiB)
 * that the library holds on every device that loads it until the process exits; a batch
 * may use at most 16384 rays and 1048576 sample slots (rays times the grid's per-ray sample
 * bound), larger batches return CPX_ERR_INVALID_ARGUMENT.  The first call on a device looks
 * up the array's device address; make that first call before any stream capture.  Every
 * call on a device shares the array and overwrites it, so calls that overlap on the GPU
 * race.  The call synchronises its stream: it reads its device-side check flags back and
 * returns once the batch has run, with their status; cpx_last_sample_counts does not see its
 * counts.  The array's address is looked up once per device and kept for the life of the
 * process, so the library is not for use across a cudaDeviceReset. */
cpx_status cpx_render_forward_backward_noalloc(cpx_grid* g, cpx_rays* r, double* losses_dev,
                                               const int32_t* sample_index_dev, int start,
                                               int len, double mask_coef, float huber_delta,
                                               cpx_stream stream);
/* Held-out view render (RenderUtils::renderImage, SVRF/RenderUtils.cu:1801; the RGB branch of
 * renderImageGPU, RenderUtils.cu:1720).  One ray per pixel of a width x height image through
 * `cam`, in double as the reference sets it up (getBound), pixel p at row p / width and
 * column p % height as the reference indexes it.  Outputs are device buffers, any may be
 * NULL: rgb_dev float [3][w*h] (Image.red/green/blueFloatDevice, white background added
 * when white_bg), rgb8_dev u8 [3][w*h] (red/green/blueDevice, composited on white),
 * depth_dev float [w*h] (disparityDevice, the expected t), mask_dev u8 [w*h] (opacity x 255).
 * Does not synchronise. */
cpx_status cpx_render_image(cpx_grid* g, const cpx_camera* cam, int width, int height,
                            int white_bg, float* rgb_dev, uint8_t* rgb8_dev, float* depth_dev,
                            uint8_t* mask_dev, cpx_stream stream);
/* No reference counterpart (the reference's Render::travelScene, SVRF/Render.cu:947, only
 * saves its renders): mean of squared differences of two device float arrays of n elements,
 * summed in double on the device, for held-out PSNR; synchronises. */
cpx_status cpx_image_mse(const float* a_dev, const float* b_dev, int64_t n, double* mse_out,
                         cpx_stream stream);
/* Coarse-to-fine refinement (upsampleScene, SVRF/SceneUtils.cu:419-485, as
 * objectScene::initSelfByUpsample runs it, SceneUtils.cu:487-657): every vertex of dst takes
 * the trilinear interpolation of src at (col*srcW/dstW, row*srcH/dstH, depth*srcD/dstD);
 * densities below threshold become 0.  low_band_only interpolates and writes only the first
 * SH coefficient per channel (the reference's lowBoundOnly; otherwise dst->sh_dim must equal
 * src->sh_dim).  A sparse src gives zeros in its unoccupied cells; a sparse dst (occupancy built,
 * compacted) receives its in-cage vertices.  The reference's sparse target is reached by
 * upsampling into a dense dst, then cpx_occupancy_build and cpx_grid_make_sparse.  FP32 form;
 * dst is normally a fresh grid. */
cpx_status cpx_grid_upsample(const cpx_grid* src, cpx_grid* dst, float threshold, int low_band_only,
                             cpx_stream stream);

/* Silhouette carving, one camera (silhouetteCarving, SVRF/RenderUtils.cu:181-254, as
 * RenderUtils::bbox_silhouette runs it per training image): every vertex (x, y, z) of the dense
 * grid projects its point (x + 0.5, y + 0.5, z) through `projection` (the camera's 3x4
 * row-major world-to-pixel matrix, Camera::projectionMatHost) and, when no pixel within
 * `radius` of the truncated image position has a nonzero mask or colour byte, gets density 0
 * and density-LR multiplier 0.  Image planes are host arrays of img_w*img_h bytes (mask may be
 * NULL: all zero).  Dense grids.  Synchronous. */
cpx_status cpx_carve_silhouette(cpx_grid* g, const double* projection, int img_w, int img_h,
                                const uint8_t* red, const uint8_t* green, const uint8_t* blue,
                                const uint8_t* mask, int radius, cpx_stream stream);
/* Bounding box of the vertices whose density-LR multiplier exceeds 1e-6 (getBoundingBoxZ and
 * the reduction of bbox_silhouette, SVRF/RenderUtils.cu:256-286, 372-464): bbox_out[6] =
 * wmin, wmax, hmin, hmax, dmin, dmax, which also becomes the grid's ray box (as the reference
 * sets scene->bbox_*).  scale_ratio_out (may be NULL): getMaxRadius's largest distance of such
 * a vertex from the grid centre, / width * 2 (bbox_silhouette's return value).  Dense grids.
 * Synchronous. */
cpx_status cpx_grid_bbox(cpx_grid* g, int* bbox_out, double* scale_ratio_out);

/* ------------------------------------------------------------------ text formats */
/* objectScene::saveSelf (SVRF/SceneUtils.cu:1246-1300) into the existing directory `dir`:
 * occupancy.txt, opacity_band<band>.txt and <red|green|blue>_<k>.txt for the first (band+1)^2
 * coefficients (from band^2 with hierarchy_mode), or the sparse files; rows of "%.6lf " values
 * as the reference writes them (saveFloaters2File, SVRF/Utils.cu:648).  Synchronous. */
cpx_status cpx_grid_save_text(const cpx_grid* g, const char* dir, int band, int density_only, int hierarchy_mode);
/* objectScene::initFromFile (SVRF/SceneUtils.cu:703-790), dense: the density and the first
 * file_sh_dim SH coefficients per channel from `dir` into a dense grid of at least that many
 * (the rest zero); values parsed as the reference's fscanf("%f ").  Synchronous. */
cpx_status cpx_grid_load_text(cpx_grid* g, const char* dir, int file_sh_dim);
/* objectScene::initFromFile (SVRF/SceneUtils.cu:703-790), sparse with occupancy: a sparse
 * checkpoint of cpx_grid_save_text or the reference's saveSelf into a fresh dense grid of its
 * dimensions, which becomes sparse.  The in-cage count comes from
 * sparse_inCageInfo_band<b>.txt, where the reference's saveSelf writes it (over the in-cage
 * flags, SVRF/SceneUtils.cu:1280-1283); the flags are rebuilt from occupancy.txt by the rule
 * pruneScene made them with, and must give sparse_indexOffset.txt and the count exactly
 * (else CPX_ERR_INVALID_ARGUMENT: an inconsistent checkpoint).  Compact density and the first
 * file_sh_dim SH coefficients per channel come from the *_sparse.txt files.  (The reference's
 * loader reads its in-cage flags from the file that then holds only the count, so every flag
 * it loads is the count's low byte; the flags here are the saved grid's.)  Synchronous. */
cpx_status cpx_grid_load_text_sparse(cpx_grid* g, const char* dir, int file_sh_dim);
/* Image::initSelfFromFile (SVRF/ImageUtils.cu:84-128): <prefix>_mask.txt and
 * <prefix>_{red,green,blue}.txt (or <prefix>.txt when gray_only) into host planes of
 * width*height bytes; bbox[4] = the rows and columns bounding the nonzero mask pixels
 * (row min, row max, col min, col max; readMask, SVRF/Utils.cu:508). */
cpx_status cpx_image_load_text(const char* prefix, int width, int height, int gray_only, uint8_t* red, uint8_t* green,
                               uint8_t* blue, uint8_t* gray, uint8_t* mask, int* bbox);
/* processMasksInfo's masksIndex (SVRF/ImageUtils.cu:130-146): the pixels of the bbox rectangle,
 * row by row -- the mask-area rays' pixel list.  index_out NULL: only the count. */
cpx_status cpx_image_mask_pixels(const int* bbox, int width, int32_t* index_out, int64_t* n_out);

/* March options (no reference counterpart; for studying the mixed forms):
 * CPX_OPT_NO_EMPTY_SKIP  the FP32 march steps through every empty cell of a sparse grid as
 *                        the reference does, instead of jumping over empty cells and bricks;
 * CPX_OPT_FP32_MARCH     an FP32-storage grid marches like the mixed forms (FP32 arithmetic,
 *                        empty-space jumps, early stop) instead of the reference's FP64/FP32
 *                        sequence;
 * CPX_OPT_NO_EARLY_STOP  the FP32 march runs every ray to its far bound, instead of ending it
 *                        once its transmittance is below 1e-4 (what the rest of the ray could
 *                        add to its colour and weight);
 * CPX_OPT_FUSED_MARCH    the march runs as one launch that shades rays while others are
 *                        still being placed, instead of two launches (placement of every ray,
 *                        then shading).  Results are the same; slower on the B200 (placement's
 *                        dependent chains lose issue slots to the shading warps beside them);
 *                        for comparison;
 * CPX_OPT_PLANE_SWEEP    the FP32 form's fused TV + Adam sweep of a dense grid (SH band 2)
 *                        walks z with the x-y plane of a tile on chip instead of running a
 *                        block per row of vertices that reads neighbours from L1/L2.  Results
 *                        are the same bit for bit; slower on the B200 (one z-step of loads in
 *                        flight per SM); for comparison;
 * CPX_OPT_SPLIT_SWEEP    cpx_train_step on a dense FP32 grid of SH band 2 with the fused TV:
 *                        once the batch is placed, the vertices its samples cannot reach (the
 *                        corners of no sample's cell, marked from the placed samples) are swept
 *                        on a second stream while the batch is shaded, and the rest after the
 *                        shading.  Results are those of the single sweep bit for bit.  Slower on
 *                        the B200 (6.1 against 4.5 ms a step at 256^3: the shading's gathers
 *                        and atomics wait behind the sweep's DRAM traffic); for comparison;
 * CPX_OPT_SPARSE_ADAM    mixed forms only (no reference counterpart): the optimizer sweep
 *                        updates only the vertices the batch touched -- a vertex whose gradient
 *                        is zero keeps its parameters and moments, as sparse Adam skips zero
 *                        gradients -- in place, so it neither reads nor writes the others; the
 *                        TV term applies at the updated vertices, from neighbour values that
 *                        may already be this step's.  The grid then trains differently from the
 *                        reference's dense Adam; bench.py --quality measures by how much. */
#define CPX_OPT_NO_EMPTY_SKIP 1
#define CPX_OPT_FP32_MARCH 2
#define CPX_OPT_NO_EARLY_STOP 4
#define CPX_OPT_FUSED_MARCH 8
#define CPX_OPT_PLANE_SWEEP 16
#define CPX_OPT_SPLIT_SWEEP 32
#define CPX_OPT_SPARSE_ADAM 64
cpx_status cpx_grid_set_options(cpx_grid* g, int options);

/* TV ("variance") gradient: type 0 with 3/6/26 neighbours, type 1 voxel disparity,
 * type 2 both. */
cpx_status cpx_tv_grad(cpx_grid* g, double lam_density, double lam_sh, int type,
                       int neighbours, cpx_stream stream);
/* Adam over every active vertex (beta 0.9/0.999, eps 1e-6), density clamped at 0,
 * gradients zeroed. */
cpx_status cpx_adam_step(cpx_grid* g, double lr, double sh_lr, int timestep, cpx_stream stream);
/* TV type 0 (6 neighbours) fused into the Adam sweep: each vertex record is read once.
 * Same results as cpx_tv_grad(type 0, 6) followed by cpx_adam_step. */
cpx_status cpx_tv_adam_step(cpx_grid* g, double lam_density, double lam_sh, double lr,
                            double sh_lr, int timestep, cpx_stream stream);

/* One training batch as the reference's loop runs it (SVRF/Render.cu:407-500):
 * forward+backward, TV (when do_tv; fused into Adam for type 0 / 6 neighbours),
 * Adam at `timestep`.  losses_dev receives the per-ray losses; when mse_out is
 * non-NULL the losses are reduced on the device to the batch MSE (Utils.cu:311) and
 * copied to *mse_out (this synchronises the stream). */
typedef struct cpx_step_args {
    double mask_coef;
    float huber_delta;
    int do_tv;
    int tv_type;
    int tv_neighbours;
    double lam_density;
    double lam_sh;
    double lr;
    double sh_lr;
    int timestep;
} cpx_step_args;
cpx_status cpx_train_step(cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev, int start,
                          int len, const cpx_step_args* args, double* losses_dev,
                          double* mse_out, cpx_stream stream);
/* cpx_train_step (the reference's batch, SVRF/Render.cu:407-500) that also places the NEXT
 * batch's samples while this batch's optimizer sweep runs: after this batch's march, the
 * densities the sweep will write are worked out first (bit-identical to the sweep's), and a
 * second stream places next_r's rays [next_start, next_start + next_len) on them beside the
 * sweep.  The next call with that batch then only shades it.  Results are those of
 * cpx_train_step bit for bit in every placed sample.  A comparison form: on the B200 at 256^3
 * with 8192-ray batches it is slower than cpx_train_step (7.7 against 4.7 ms a step) -- working
 * out the densities ahead reads a sector of every parameter, gradient and moment record and
 * costs more than the placement it hides, and placement beside the bandwidth-bound sweep waits
 * behind the sweep's traffic.  The placement done in advance
 * is used only if nothing it read has changed: any call that changes the grid's densities,
 * jitter offsets, occupancy or march options, or the next batch's ray fields, makes the next
 * call place the batch itself.  It applies to dense FP32 grids of SH band 2 with TV type 0/6 (or
 * none) in the reference's march; elsewhere (or with next_r NULL) the call is cpx_train_step.
 * The next batch's sample index and ray buffers must stay valid until the next call.  No
 * reference counterpart beyond the batch it replaces. */
cpx_status cpx_train_step_ahead(cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev, int start, int len,
                                cpx_rays* next_r, const int32_t* next_sample_index_dev, int next_start,
                                int next_len, const cpx_step_args* args, double* losses_dev, double* mse_out,
                                cpx_stream stream);

/* Synchronise the grid's work and report (then clear) the sticky device-side errors of
 * earlier asynchronous calls: CPX_ERR_ITERATION_CAP when a ray's march exceeded its
 * sample bound, CPX_ERR_INVALID_ARGUMENT when a sample index was out of range,
 * CPX_ERR_NOT_READY when a shading warp gave up one of its bounded waits (a ray's placement in
 * the fused march, or a vertex record copy) and stopped. */
cpx_status cpx_grid_check(cpx_grid* g);
/* No reference counterpart (a diagnostic): the number of vertices marked in the touched map
 * the next optimizer sweep will read.  The backward marks every vertex it scatters gradients
 * into and a sweep reads and clears gradient records only there; after
 * cpx_grid_upload_grads or a standalone cpx_tv_grad every vertex counts.  Synchronous. */
cpx_status cpx_grid_touched_count(cpx_grid* g, int64_t* count);
/* No reference counterpart (a diagnostic): the dense empty-space map the mixed forms' march
 * (and the FP32 march under CPX_OPT_FP32_MARCH) jumps by -- one bit per cell, set unless all
 * eight corner densities are at or below 0; cell (x, y, z) of the (W-1) x (H-1) x (D-1) cells
 * is bit c % 32 of word c / 32, c = (z (H-1) + y) (W-1) + x.  The map follows every density
 * change (upload, sweep, carving).  n_words must be at least ceil(cells / 32).
 * CPX_ERR_UNSUPPORTED for a grid whose march keeps no such map (sparse, the FP32 form's
 * march, CPX_OPT_NO_EMPTY_SKIP); CPX_ERR_NOT_READY before the first density upload.
 * Synchronous. */
cpx_status cpx_grid_download_cell_map(cpx_grid* g, uint32_t* words, int64_t n_words);

/* Per-ray sample counts of the last forward/backward batch (device int32[len], or a
 * host copy) -- the march's sample sequence, for bit-exact checks. */
cpx_status cpx_last_sample_counts(const cpx_grid* g, int32_t* counts_host, int len);

/* Number of kernels this library launched since load (for launch accounting). */
int64_t cpx_kernel_launches(void);

/* ---- Learned sample-interval proposal (no reference counterpart) ----
 * A small MLP (48 -> 64 -> 64 -> 64 -> 1, ReLU; BF16 tensor-core inference, FP32 training)
 * predicts for each of 32 equal segments of a ray's [near, far] whether it holds visible
 * density.  Input per segment: the midpoint in box coordinates with its 4-octave sin/cos
 * encoding, the ray direction and the ray origin.  Label: the samples of a full march inside
 * the segment carry total weight above label_weight (empty and occluded segments are 0).
 * The march skips the segments predicted empty with confidence (sigmoid(logit) <= 1 -
 * confidence) and marches the others in full: a ray whose predictions are all uncertain
 * runs the plain full march. */
typedef struct cpx_proposal cpx_proposal;
typedef struct cpx_proposal_desc {
    uint32_t seed;         /* parameter initialisation */
    float confidence;      /* a segment is skipped when sigmoid(logit) <= 1 - confidence (0.9) */
    float label_weight;    /* segment label threshold on the summed sample weights (1e-3) */
    float learning_rate;   /* Adam (1e-3) */
} cpx_proposal_desc;

int cpx_proposal_param_count(void);
cpx_status cpx_proposal_create(const cpx_proposal_desc* desc, cpx_proposal** out);
cpx_status cpx_proposal_destroy(cpx_proposal* p);
/* FP32 parameters [cpx_proposal_param_count()] (W1 [64][48], b1, W2 [64][64], b2, W3, b3,
 * w4 [64], b4) to (upload = 0) or from (upload = 1) host memory. */
cpx_status cpx_proposal_params(cpx_proposal* p, float* host, int upload);
/* Logits [len][32] and/or per-ray segment masks [len] (all ones = full march) of a batch;
 * tensor_cores = 0 runs the FP32 CUDA-core forward instead (for checking). */
cpx_status cpx_proposal_infer(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev,
                              int start, int len, float* logits_dev, uint32_t* masks_dev, int tensor_cores,
                              cpx_stream stream);
/* Gradient of the mean binary cross-entropy over the batch's 32*len points against the
 * labels of seg_weights_dev [len][32], to host memory, without an update.  Synchronous. */
cpx_status cpx_proposal_gradient(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev,
                                 int start, int len, const float* seg_weights_dev, float* grad_host,
                                 double* loss_out);
/* `steps` Adam steps over consecutive slices of rays_per_step rays of the batch. */
cpx_status cpx_proposal_train(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev,
                              int start, int len, const float* seg_weights_dev, int steps, int rays_per_step,
                              double* loss_out, cpx_stream stream);
/* Completed training rounds, segments predicted empty (and skipped) so far, and the device
 * error flags (4: a tensor-core wait ran out).  Synchronous. */
cpx_status cpx_proposal_stats(cpx_proposal* p, int* rounds, int64_t* skipped_segments, int* error_flags);
/* The march of cpx_render_forward_backward with segment weights [len][32] recorded
 * (seg_weights_dev, the proposal's labels) when non-NULL, or guided by per-ray segment masks
 * [len] (masks_dev, from cpx_proposal_infer) when non-NULL.  The mixed-precision forms
 * only (FP32 march).  With neither it equals cpx_render_forward_backward. */
cpx_status cpx_render_forward_backward_guided(cpx_grid* g, cpx_rays* r, double* losses_dev,
                                              const int32_t* sample_index_dev, int start, int len,
                                              double mask_coef, float huber_delta,
                                              const uint32_t* masks_dev, float* seg_weights_dev,
                                              cpx_stream stream);
/* The forward alone of cpx_render_forward_backward_guided (masks_dev may be NULL: the mixed
 * forms' full march). */
cpx_status cpx_render_forward_guided(cpx_grid* g, cpx_rays* r, const int32_t* sample_index_dev, int start, int len,
                                     const uint32_t* masks_dev, cpx_stream stream);
/* One training batch of the mixed form with the proposal: every train_every-th iteration
 * (and every iteration before warmup) runs the full march, records labels and then trains
 * the proposal (train_steps Adam steps of rays_per_step rays); the other iterations infer
 * the masks and run the guided march; then TV + Adam as cpx_train_step. */
typedef struct cpx_proposal_schedule {
    int warmup;          /* iterations of full march before the proposal is used */
    int train_every;     /* label + training period (50) */
    int train_steps;     /* Adam steps per training round */
    int rays_per_step;   /* rays per Adam step */
} cpx_proposal_schedule;
cpx_status cpx_train_step_proposal(cpx_grid* g, cpx_rays* r, cpx_proposal* p, const int32_t* sample_index_dev,
                                   int start, int len, const cpx_step_args* args,
                                   const cpx_proposal_schedule* schedule, int iteration, double* losses_dev,
                                   double* mse_out, cpx_stream stream);

/* ---- Batched multi-scene training (no reference counterpart: the reference trains one
 * scene per process, Experiment.cu).  A batch holds scenes of any grid size and any batch
 * length -- one precision form, SH band 2 -- and steps all of them together: one placement
 * and one shading launch over every scene's rays (persistent kernels taking rays from a
 * work counter), then each scene's TV + Adam sweep.  Iteration i of scene s reads rays
 * [(i % pool) * len_s, (i + 1) * len_s) of its ray table, pool = floor(n_rays / len_s), and
 * steps Adam with timestep i + 1: one batched step equals cpx_train_step on every scene with
 * start = (i % pool) * len_s and no sample index (shuffle the ray table once, on upload).
 * The iteration counter lives on the device, so a whole step can replay as a CUDA graph. */
typedef struct cpx_batch cpx_batch;
typedef struct cpx_batch_scene {
    cpx_grid* grid;
    cpx_rays* rays;
    int rays_per_batch;
} cpx_batch_scene;
/* Launch shapes of the batched march: threads per placement block (32..512, a multiple of
 * 32), warps per shading block (2, 4 or 8), rays a shading warp takes per work-counter
 * access (1..8), and samples a shading lane takes per chunk (1, 2 or 4; a chunk of
 * 32 * samples_per_step samples shares one vertex table, so its corners are gathered and its
 * gradients scattered once; shade_warps * samples_per_step <= 8, the tables' shared memory). */
typedef struct cpx_batch_tuning {
    int place_block;
    int shade_warps;
    int grab;
    int samples_per_step;
} cpx_batch_tuning;
/* args->timestep is the first iteration's timestep; losses of every step stay on the device
 * ([sum of rays_per_batch], scene after scene). */
cpx_status cpx_batch_create(const cpx_batch_scene* scenes, int n_scenes, const cpx_step_args* args,
                            cpx_batch** out);
cpx_status cpx_batch_destroy(cpx_batch* b);
/* One training iteration of every scene.  use_graphs: replay a captured CUDA graph of the
 * whole iteration (captured on first use, one per parity of the grids' ping-pong buffers,
 * and re-captured when a grid changed outside the batch). */
cpx_status cpx_batch_step(cpx_batch* b, int use_graphs, cpx_stream stream);
/* Per-scene batch MSE of the last step (getMSEError of each scene's losses) into
 * mse_host[n_scenes].  Synchronous. */
cpx_status cpx_batch_mse(cpx_batch* b, double* mse_host, cpx_stream stream);
/* Synchronise and report the sticky device errors of the batch's marches, as cpx_grid_check. */
cpx_status cpx_batch_check(cpx_batch* b);
/* The iteration the next step runs (timestep - 1) and the per-step ray and launch totals. */
cpx_status cpx_batch_info(const cpx_batch* b, int* iteration, int* total_rays, int* launches_per_step);
cpx_status cpx_batch_set_tuning(cpx_batch* b, const cpx_batch_tuning* t);
cpx_status cpx_batch_get_tuning(const cpx_batch* b, cpx_batch_tuning* t);
/* Coordinate-descent search of the launch shapes (placement blocks of 64/128/256/512 threads,
 * shading blocks of 2/4/8 warps, 1/2/4/8 rays per access, 1/2/4 samples per lane and chunk,
 * where the tables fit): every candidate runs steps_per_trial real
 * training iterations (they advance training like cpx_batch_step), timed with CUDA events;
 * the fastest shapes are kept and written to best (may be NULL). */
cpx_status cpx_batch_autotune(cpx_batch* b, int steps_per_trial, cpx_batch_tuning* best, cpx_stream stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* CPX_H */
