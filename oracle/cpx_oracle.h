/*
 * cpx_oracle.h -- CPU restatement of the Clear-plenoxels training hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product path (libcpx.so) is compared against, and the timed CPU baseline
 * of bench.py.  Nothing in the product links, loads or calls it.
 *
 * Every function follows the reference line by line (file:line citations are
 * relative to the reference project root; SVRF = SparseVolumeRadianceField).
 * Types follow the reference exactly: where the reference computes in double
 * and stores float, so does the oracle, and the multiply-add pairs that nvcc
 * contracts into one fused operation are written as fma() (see the
 * ORC_CONTRACT_* switches, pinned against the reference's own kernels run on
 * a B200).  Transcendentals come from the host libm, so results that pass
 * through exp/log/pow agree with the GPU to a few ulp, not bit for bit;
 * everything built from +,-,*,/,sqrt alone (ray/AABB hits, occupancy and
 * index lists) is bit-exact.
 */
#ifndef CPX_ORACLE_H
#define CPX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scene: the fields of ObjectScene (SVRF/SceneUtils.cuh:4-98) the path reads. */
typedef struct orc_scene {
    int W, H, D;              /* vertices per axis (sceneWidth/Height/Depth) */
    int sh_dim;               /* SH coefficients per channel in storage */
    int band;                 /* optimizingBand: forward uses (band+1)^2 coefficients */
    int hierarchy;            /* Optimizer::hierarchyStrategy */
    int optimize_step;        /* ObjectScene::optimizeStep (TV type 1 colour gate) */
    float step;               /* stepSize */
    int sparse;
    int64_t n_act;            /* actualGridNums: length of every parameter array */
    float* params;            /* planar [(1 + 3*sh_dim)][n_act]: k=0 density, 1+c*sh_dim+i SH */
    const uint8_t* occ;       /* [(W-1)(H-1)(D-1)] occupancy bytes (sparse) */
    const uint32_t* index_offsets; /* [W*H*D] vertex -> compact index (sparse) */
    const uint8_t* in_cage;   /* [W*H*D] (sparse) */
    const float* adaptive_lr; /* [n_act] density LR multiplier (dense Adam); NULL = 1 */
    const double* off_x;      /* per-sample jitter offsets [n_off]; NULL or beyond n_off = 0 */
    const double* off_y;
    const double* off_z;
    int n_off;
} orc_scene;

/* Rays: the SoA of _rays (SVRF/Rays.cuh:8-57), RGB only. */
typedef struct orc_rays {
    int64_t n;
    int white_bg;
    float *ox, *oy, *oz, *dx, *dy, *dz, *near_t, *far_t;
    uint8_t *mask, *r, *g, *b;
    float *acc_den, *acc_w, *acc_r, *acc_g, *acc_b;
} orc_rays;

/* Contraction switches (which mul+add pairs nvcc fuses); default ORC_CONTRACT_DEFAULT. */
#define ORC_CONTRACT_RAYDIR      1u  /* secondPoint += c2w*x as one fma (Rays.cu:40) */
#define ORC_CONTRACT_NORM_P0     2u  /* normalize: fma(p2,p2, fma(p0,p0, p1*p1)) */
#define ORC_CONTRACT_NORM_P1     4u  /* normalize: fma(p2,p2, fma(p1,p1, p0*p0)) */
#define ORC_CONTRACT_POS         8u  /* o + t*d as one fma (RenderUtils.cu:1676) */
#define ORC_CONTRACT_ACCD       16u  /* accD += sigma*step with the float product fused */
#define ORC_CONTRACT_DEFAULT (ORC_CONTRACT_RAYDIR | ORC_CONTRACT_NORM_P0 | ORC_CONTRACT_POS)

void orc_set_contract_mode(unsigned mode);
unsigned orc_get_contract_mode(void);
void orc_set_threads(int n);
int orc_get_threads(void);

/* R4 activations (RenderUtils.cu:480-515). */
float orc_density_activation(float x);
float orc_density_derivation(float x);
float orc_sigmoid(float x);
float orc_sigmoid_derivative(float x);

/* R5: unnormalised SH basis on the float direction (RenderUtils.cu:1646-1670). */
void orc_sh_basis(const float dir[3], float shs[25]);

/* R1: rays of one camera (Rays.cu:22-144).  pix_index lists the pixels (row*w+col);
 * rays are written at out->*[out_start + i].  Camera fields are the device copies
 * getBound reads: alpha[2], principle[2], c2w[16] (row-major), centre[4]. */
void orc_rays_from_camera(const double* alpha, const double* principle,
                          const double* c2w, const double* centre,
                          const int* bbox /* wmin,wmax,hmin,hmax,dmin,dmax */,
                          int img_w, const uint8_t* red, const uint8_t* green,
                          const uint8_t* blue, const uint8_t* mask, int white_bg,
                          const int* pix_index, int n_pix,
                          orc_rays* out, int64_t out_start);

/* R7: forward march of the rays sample_index[start .. start+len) (RenderUtils.cu:1582-1718,
 * 1919-1959).  counts[tid] (optional) receives the number of evaluated samples. */
void orc_render_forward(const orc_scene* s, orc_rays* r, const int* sample_index,
                        int start, int len, int* counts);

/* R8: backward (RenderUtils.cu:2051-2256, 1074-1364).  losses[tid] as the reference;
 * grad is planar [(1+3 sh_dim)][n_act] in double (each per-sample contribution is
 * rounded to float as the reference's atomicAdd operand, then summed in double). */
void orc_render_backward(const orc_scene* s, const orc_rays* r, const int* sample_index,
                         int start, int len, double mask_coef, float huber_delta,
                         double* losses, double* grad, int* counts);

/* R9: TV / voxel-disparity gradient added into the float grad (RenderUtils.cu:2442-2851). */
void orc_tv_grad(const orc_scene* s, float* grad, double lam_density, double lam_sh,
                 int type, int nbrs);

/* R10: Adam over every parameter slot, params updated in place, grad zeroed
 * (Optimizer.cu:359-415). */
void orc_adam(orc_scene* s, float* grad, float* m, float* v, double lr, double sh_lr,
              int timestep);

/* R3: occupancy bytes, in-cage flags and index offsets from a dense density
 * (SceneUtils.cu:800-881, 1081-1120).  Returns the in-cage count.  The x = W-1
 * face flag is written where the reference writes it (SceneUtils.cu:872); that
 * index is always inside the array, *dropped_writes (bounds check) stays 0. */
uint32_t orc_occupancy(const float* density, int W, int H, int D, float threshold,
                       uint8_t* occ, uint8_t* in_cage, uint32_t* index_offsets,
                       int64_t* dropped_writes);

/* Compaction of a dense planar parameter block into in-cage order (SceneUtils.cu:585-602). */
void orc_compact(const float* dense, int n_arrays, int64_t n_dense, const uint8_t* in_cage,
                 float* compact, int64_t n_compact);

/* R13: render one view (renderImageGPU + volumeRender_RGB, RenderUtils.cu:1720-1810,
 * 1443-1580, getBound in double at RenderUtils.cu:34-97).  Outputs (any may be NULL):
 * rgb float planes [3][w*h] (background added when white_bg), rgb8 planes [3][w*h],
 * depth (sum of w*t) [w*h], mask (acc*255) [w*h]. */
void orc_render_image(const orc_scene* s, const double* alpha, const double* principle,
                      const double* c2w, const double* centre, const int* bbox, int width,
                      int height, int white_bg, float* rgb, uint8_t* rgb8, float* depth,
                      uint8_t* mask);

/* Coarse-to-fine refinement: upsampleScene / upsample_trilinear (SceneUtils.cu:262-485).
 * src: the oracle scene (dense or sparse); dst: planar [1 + 3*dst_sh][dW*dH*dD] (dense target,
 * written for every vertex; entries beyond the written coefficients are left as they are). */
/* silhouetteCarving (SVRF/RenderUtils.cu:181-254) of one camera on a dense W x H x D grid:
 * density[v] and lr[v] become 0 where no pixel within `radius` of the vertex's projection has a
 * nonzero byte (mask may be NULL). */
void orc_carve_silhouette(float* density, float* lr, int W, int H, int D, const double* P, int img_w,
                          int img_h, const uint8_t* red, const uint8_t* green, const uint8_t* blue,
                          const uint8_t* mask, int radius);
/* getBoundingBoxZ + getMaxRadius + bbox_silhouette's reduction (SVRF/RenderUtils.cu:256-478):
 * bbox[6] = wmin, wmax, hmin, hmax, dmin, dmax of the vertices with lr > 1e-6; returns the
 * scale ratio (max radius / W * 2). */
double orc_bbox(const float* lr, int W, int H, int D, int* bbox);
void orc_upsample(const orc_scene* src, int dW, int dH, int dD, int dst_sh, float threshold,
                  int low_band_only, float* dst);

/* R11: batch MSE of the per-ray losses (Utils.cu:311-320). */
double orc_mse(const double* losses, int n);
/* randGPU's normal jitter offsets (SVRF/Utils.cu:1002-1044) from cuRAND's scrambled Sobol64
 * direction numbers dirs[n_states][64] and 32-bit scramble words, for len entries. */
void orc_sobol_offsets(const uint64_t* dirs, const uint32_t* scramble32, int len, uint64_t first, double radius,
                       double* out);

/* Compositing known-answer test: the arithmetic of testRender
 * (SVRF/VolumeFieldRender.cu:111-183), FP64. */
void orc_composite_kat(const double* opacity, const double* colour /*[3][n]*/, int n,
                       const double* gt /*[3]*/, double* render_res /*[3]*/,
                       double* weights /*[n]*/, double* opacity_grad /*[n]*/,
                       double* colour_grad /*[3][n]*/);

/* ---- FP64 host oracle of the training step (every quantity in double) ----
 * The same march, backward, TV (type 0, 6 neighbours) and Adam as the reference, with
 * every operation in double: the yardstick the FP32 and the mixed 16-bit forms are both
 * measured against.  pred [len][3] (background included), accw [len], losses [len],
 * grad planar [n_arrays][n_act] (accumulated into). */
typedef struct orc_bricks {
    const uint8_t* bits; /* one byte per 8x8x8-cell brick: any cell occupied (NULL: no jumps) */
    int bx, by, bz;
    double t_stop;       /* a ray ends once its transmittance is below this (0: never) */
    const uint8_t* cells; /* dense grid: one byte per cell, 0 when every corner density is at or
                             below the empty bound -- such cells are jumped like unoccupied ones
                             (NULL: none) */
} orc_bricks;
/* bricks non-NULL: the FP32 march of the mixed forms.  With bits, on a sparse grid it moves
 * through an empty cell (or through its whole brick when the brick is empty) in one jump of
 * whole steps, leaving the sample sequence of step-by-step stepping unchanged; with t_stop it
 * ends a ray after the sample that takes its transmittance below t_stop. */
void orc64_forward_backward(const orc_scene* s, const orc_rays* r, const orc_bricks* bricks, int start,
                            int len, double mask_coef, double huber, double* pred, double* accw,
                            double* losses, double* grad);
/* TV type 0 / 6 neighbours in double, added into grad (same gating as orc_tv_grad). */
void orc64_tv6(const orc_scene* s, const double* params, double* grad, double lam_d,
               double lam_sh);
/* Adam in double over planar params/moments (params updated in place, grad zeroed). */
void orc64_adam(const orc_scene* s, double* params, double* grad, double* m, double* v,
                double lr, double sh_lr, int timestep);

#ifdef __cplusplus
}
#endif
#endif
