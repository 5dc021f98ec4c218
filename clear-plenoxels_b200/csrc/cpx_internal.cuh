// cpx_internal.cuh -- handles, device views and shared helpers of libcpx.
//
// Data layout in HBM (plain FP32 form):
//   * parameters: array-of-records, one record of `rec` floats per active vertex
//     ([density, R0..R(s-1), G0.., B0..], padded to a multiple of 4 floats: 28 floats
//     = 112 B at SH band 2), so a trilinear corner is 7 aligned 16-byte loads and the
//     optimizer sweep streams whole records.  Two parameter buffers alternate (the
//     fused TV+Adam sweep reads one and writes the other, so TV sees pre-step values).
//   * gradients, Adam first and second moments: same record layout.
//   * density mirror: the density of every active vertex again as a packed float
//     array, read by the sample-placement march (4 B per corner instead of a record).
//   * sparse tables: occupancy as one bit per cell, index_offsets u32 per dense vertex
//     (the reference's compact-index table), compact->dense u32 per active vertex.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/cpx.h"
#include "lowp.cuh"

namespace cpx {

constexpr int kMaxShDim = 9;  // SH coefficients per channel supported by the kernels (band <= 2)

// Record of one evaluated sample, written by the placement march, read by the shading pass.
struct __align__(16) SampleRec {
    uint16_t bx, by, bz, pad;  // base vertex of the sample's cell (unsigned-truncated position)
    float fx, fy, fz;          // fractional position in the cell (computed in double)
    float raw;                 // interpolated raw density
    float w;                   // compositing weight T_i (1 - exp(-sigma step))
    float tn;                  // transmittance after the sample, exp(-sum sigma step)
};
static_assert(sizeof(SampleRec) == 32, "SampleRec must be 32 bytes");

// Per-kernel view of a grid (passed by value).
struct GridView {
    int W, H, D;
    int sh_dim, band, n_sh_fwd, hierarchy;
    int n_arrays, rec;  // rec = floats per record (multiple of 4)
    float step;
    int sparse;
    int64_t n_act;
    // FP32 form: parameter records [n_act][rec].  Mixed forms: the 16-bit SH records
    // [n_act][slots], read through sh16_records() by kernels instantiated for those forms
    // (the storage form is a template parameter of every kernel, so the view stays as small
    // as the FP32 kernels need).
    const float* __restrict__ params;
    const float* __restrict__ density;  // [n_act]
    float* grad;                        // [n_act][rec]
    const uint32_t* __restrict__ occ_bits;       // [(C + 31) / 32]
    const uint32_t* __restrict__ index_offsets;  // [W*H*D]
    const double* __restrict__ off_x;
    const double* __restrict__ off_y;
    const double* __restrict__ off_z;
    int n_off;
};

struct RaysView {
    const float* __restrict__ ox;
    const float* __restrict__ oy;
    const float* __restrict__ oz;
    const float* __restrict__ dx;
    const float* __restrict__ dy;
    const float* __restrict__ dz;
    const float* __restrict__ near_t;
    const float* __restrict__ far_t;
    const uint8_t* __restrict__ mask;
    const uint8_t* __restrict__ r;
    const uint8_t* __restrict__ g;
    const uint8_t* __restrict__ b;
    float* acc_den;
    float* acc_w;
    float* acc_r;
    float* acc_g;
    float* acc_b;
    int white_bg;
};

// Scratch of the two-stage march (sized for `cap_rays` rays of `maxs` samples).
struct MarchScratch {
    int maxs = 0;
    int cap_rays = 0;
    SampleRec* samples = nullptr;  // [cap_rays][maxs]
    float4* colours = nullptr;     // [cap_rays][maxs]: sigmoid colour of each sample
    int* counts = nullptr;         // [cap_rays]
    double* acc = nullptr;         // [cap_rays]: sum of weights (double, for the background)
    int* err = nullptr;            // [4] device error flags
    double* mse = nullptr;         // [1]
    int* queue = nullptr;          // [cap_rays + 4]: work counters and ready slots of the fused march
};

}  // namespace cpx

struct cpx_grid {
    int W, H, D;
    int sh_dim, band, hierarchy, optimize_step;
    int n_arrays, rec;
    float step;
    int bbox[6];
    int64_t n_dense, n_act;
    int sparse = 0;
    int prec = 0;          // storage form: kPrecFP32, kPrecBF16 or kPrecFP16 (the SH storage)
    int mom_h = 0;         // kPrecFP16 with both Adam moments in half (CPX_PRECISION_FP16_FULL)
    uint32_t sr_seed = 0;
    int slots = 0;         // 16-bit slots per record of the mixed forms
    float* params[2] = {nullptr, nullptr};  // FP32 form: parameter records, ping-pong
    int cur = 0;
    float* grad = nullptr;
    float* m = nullptr;    // FP32 form: Adam moment records
    float* v = nullptr;
    float* density = nullptr;  // FP32 form: density mirror; mixed forms: dens[cur]
    uint16_t* sh16[2] = {nullptr, nullptr};  // mixed forms: SH records, ping-pong
    uint16_t* m16 = nullptr;                  // mixed forms: bfloat16 moment records
    uint16_t* v16 = nullptr;
    float* dens[2] = {nullptr, nullptr};      // mixed forms: FP32 density, ping-pong
    // Touched-vertex bitmaps (1 bit per active vertex): the backward marks every vertex it
    // scatters gradients into, so the optimizer sweep reads and clears gradient records only
    // where they can be non-zero.  Two maps alternate: a sweep reads map `tcur` and clears the
    // other one for the next batch.  all_touched: gradients were written by another route
    // (upload, standalone TV), so the next sweep reads every record.
    uint32_t* touched[2] = {nullptr, nullptr};
    int tcur = 0;
    int all_touched = 0;
    float* adaptive_lr = nullptr;  // [n_dense]
    // occupancy (built by cpx_occupancy_build)
    int have_occupancy = 0;
    uint32_t in_cage_count = 0;
    uint8_t* occ_bytes = nullptr;       // [C]
    uint32_t* occ_bits = nullptr;       // [(C+31)/32]
    uint8_t* in_cage = nullptr;         // [n_dense]
    uint32_t* index_offsets = nullptr;  // [n_dense]
    uint32_t* compact_to_dense = nullptr;  // [n_act] when sparse
    // bricks of 8x8x8 cells, one bit each (set when any cell of the brick is occupied): the
    // FP32 march of the mixed forms crosses empty bricks in one jump
    // sparse grids: the density again at every dense vertex position, so the placement march
    // reads a corner with one load instead of an index_offsets lookup and a dependent load;
    // vertices outside the cage hold kMirrorEmpty and read compact vertex 0 as the reference does
    float* dense_mirror = nullptr;
    uint32_t* brick_bits = nullptr;
    int bricks[3] = {0, 0, 0};
    int options = 0;  // CPX_OPT_* march options
    // dense grids, FP32 march: one bit per cell, set unless all eight corner densities are at
    // or below kEmptyDensity, and the 8x8x8 brick map of those bits (refreshed whenever the
    // density changes); the march jumps over the cells and bricks they mark empty
    uint32_t* dense_cells = nullptr;
    uint32_t* dense_vbits = nullptr;   // vertex bits the cell map is built from (rows of ceil(W / 32) words)
    uint32_t* dense_bricks = nullptr;
    // jitter
    double* off[3] = {nullptr, nullptr, nullptr};
    int n_off = 0;
    // cuRAND's scrambled Sobol direction numbers (64 words per state) and 32-bit scramble
    // words of the jitter generator (jitter.cu), for sobol_n states
    unsigned long long* sobol_dirs = nullptr;
    uint32_t* sobol_scramble = nullptr;
    int sobol_n = 0;
    cpx::MarchScratch scratch;
    int last_len = 0;
    // The look-ahead step (cpx_train_step_ahead): a second sample scratch, the batch it holds
    // placed in advance, and the side stream that placed it.  `epoch` counts every change of
    // what placement reads (densities, jitter offsets, occupancy, march options); a placement
    // done in advance is used only while the epoch and its rays' epoch are unchanged.
    cpx::MarchScratch scratch2;
    uint64_t epoch = 0;
    struct {
        int valid = 0;
        const cpx_rays* r = nullptr;
        uint64_t rays_epoch = 0;
        const int32_t* sidx = nullptr;
        int start = 0, len = 0;
        uint64_t epoch = 0;
    } ahead;
    cudaStream_t aside = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

struct cpx_rays {
    int64_t n;
    int white_bg;
    void* block = nullptr;
    float *ox, *oy, *oz, *dx, *dy, *dz, *near_t, *far_t;
    uint8_t *mask, *r, *g, *b;
    float *acc_den, *acc_w, *acc_r, *acc_g, *acc_b;
    uint32_t* staging = nullptr;  // device copy of the last packed upload
    int64_t staging_cap = 0;
    uint64_t epoch = 0;  // counts every change of the ray fields (a placement done in advance checks it)
};

namespace cpx {

void set_error(const char* fmt, ...);
cpx_status cuda_status(cudaError_t e, const char* where);
void count_launch(int n = 1);

// Sparse TV neighbourhood of compact vertex v (RenderUtils.cu:2663-2763): its six neighbours'
// compact indices in the reference's order z-1, y-1, x-1, x+1, y+1, z+1, a bit per neighbour
// whose compact index is 0 (it reads as the vertex itself), and whether v gets the term at all.
// The reference gates sparse TV with inCageInfo[indexOffsets[v]] -- the dense flag array read
// at the compact index (RenderUtils.cu:2669) -- so vertex c gets its term only when dense
// vertex #c is in cage.
struct SparseTv {
    uint32_t nb[6];
    uint32_t flags;  // bits 0..5: neighbour k reads the vertex itself; bit 6: the term applies
};

__device__ __forceinline__ SparseTv sparse_tv(uint32_t v, const uint32_t* __restrict__ c2d,
                                              const uint8_t* __restrict__ in_cage,
                                              const uint32_t* __restrict__ index_offsets, int W, int H, int D)
{
    SparseTv t;
    t.flags = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) t.nb[k] = 0;
    const uint32_t WH = (uint32_t)W * H;
    const uint32_t dv = c2d[v];
    const uint32_t x = dv % W, y = (dv / W) % H, z = dv / WH;
    const bool on = x >= 1 && x + 2 <= (uint32_t)W && y >= 1 && y + 2 <= (uint32_t)H && z >= 1 &&
                    z + 2 <= (uint32_t)D && in_cage[v] != 0;
    if (!on) return t;
    const uint32_t nbd[6] = {dv - WH, dv - W, dv - 1, dv + 1, dv + W, dv + WH};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        t.nb[k] = index_offsets[nbd[k]];
        if (t.nb[k] == 0) t.flags |= 1u << k;
    }
    t.flags |= 1u << 6;
    return t;
}

// The SparseTv of vertex `from_lane`'s slot in a warp (every lane must call).
__device__ __forceinline__ SparseTv shfl_tv(const SparseTv& mine, int from_lane)
{
    SparseTv t;
#pragma unroll
    for (int k = 0; k < 6; k++) t.nb[k] = __shfl_sync(0xffffffffu, mine.nb[k], from_lane);
    t.flags = __shfl_sync(0xffffffffu, mine.flags, from_lane);
    return t;
}

// Touched-map bit of vertex v (a null map means every vertex).
__device__ __forceinline__ bool touched_bit(const uint32_t* __restrict__ map, uint32_t v)
{
    return map == nullptr || ((__ldg(map + (v >> 5)) >> (v & 31u)) & 1u);
}

__device__ __forceinline__ const uint16_t* sh16_records(const GridView& g)
{
    return reinterpret_cast<const uint16_t*>(g.params);
}

inline GridView grid_view(cpx_grid* g)
{
    GridView v;
    v.W = g->W;
    v.H = g->H;
    v.D = g->D;
    v.sh_dim = g->sh_dim;
    v.band = g->band;
    v.n_sh_fwd = (g->band + 1) * (g->band + 1);
    v.hierarchy = g->hierarchy;
    v.n_arrays = g->n_arrays;
    v.rec = g->rec;
    v.step = g->step;
    v.sparse = g->sparse;
    v.n_act = g->n_act;
    v.params = g->prec == kPrecFP32 ? g->params[g->cur] : reinterpret_cast<const float*>(g->sh16[g->cur]);
    v.density = g->density;
    v.grad = g->grad;
    v.occ_bits = g->occ_bits;
    v.index_offsets = g->index_offsets;
    v.off_x = g->off[0];
    v.off_y = g->off[1];
    v.off_z = g->off[2];
    v.n_off = g->n_off;
    return v;
}

inline RaysView rays_view(cpx_rays* r)
{
    RaysView v;
    v.ox = r->ox;
    v.oy = r->oy;
    v.oz = r->oz;
    v.dx = r->dx;
    v.dy = r->dy;
    v.dz = r->dz;
    v.near_t = r->near_t;
    v.far_t = r->far_t;
    v.mask = r->mask;
    v.r = r->r;
    v.g = r->g;
    v.b = r->b;
    v.acc_den = r->acc_den;
    v.acc_w = r->acc_w;
    v.acc_r = r->acc_r;
    v.acc_g = r->acc_g;
    v.acc_b = r->acc_b;
    v.white_bg = r->white_bg;
    return v;
}

enum MarchMode { kForward = 1, kBackward = 2, kForwardBackward = 3 };

// Segments per ray of the learned proposal (proposal.cu).
constexpr int kProposalSegments = 32;

// Marker of a dense-mirror entry outside the cage (a quiet NaN with a payload no arithmetic
// produces).
constexpr uint32_t kMirrorEmpty = 0x7FBADA55u;

// Rebuilds the dense density mirror of a sparse grid from its compact density (occupancy.cu).
cpx_status refresh_dense_mirror(cpx_grid* g, cudaStream_t st);
// Dense grids marched by the FP32 march with empty-space jumps: the cell and brick maps of
// the current density (allocated on first use).  refresh_dense_mirror calls it too.
bool dense_skip_on(const cpx_grid* g);
cpx_status refresh_dense_skip(cpx_grid* g, cudaStream_t st);

// ---- batched form (march.cu kernels, batch.cu host side)
constexpr int kMaxBatchScenes = 64;

// Brick occupancy and dense density mirror of a sparse grid, as the placement march reads them.
struct Skip {
    const uint32_t* __restrict__ bits = nullptr;
    int bx = 0, by = 0, bz = 0;
    // sparse grids: the dense density mirror (kMirrorEmpty outside the cage), so a corner's
    // density is one load; every march form reads it
    const float* __restrict__ dense = nullptr;
    // FP32 march: a ray stops once its transmittance falls below this (0: marches to far)
    float t_stop = 0.f;
    // FP32 march on a dense grid: the cell bits of cpx_grid::dense_cells (bits then holds
    // their brick map), or null
    const uint32_t* __restrict__ cells = nullptr;
};

// Density at or below which a dense grid's cell counts as empty for the FP32 march.  The
// optimizer clamps density at 0 (Optimizer.cu:384), so trained empty space sits exactly there;
// the softplus activation gives it softplus(-13) = 2.3e-6 per voxel of path, so a sample there
// carries a weight of at most 1.2e-6 (step 0.5).
constexpr float kEmptyDensity = 0.0f;

// Transmittance below which the FP32 march of the mixed forms ends a ray: what the samples
// after it could still add to the colour or the accumulated weight is below this bound.
constexpr float kStopTransmittance = 1.0e-4f;

// One scene of a batch: its views as of the batch's step parity (the parameter and touched
// buffers alternate every step).
struct BatchScene {
    GridView g;
    RaysView r;
    Skip skip;
    uint32_t* touched;
    int len;            // rays per batch
    int pool_batches;   // batches in the scene's ray table; iteration i uses batch i % pool_batches
    int maxs;           // sample slots per ray
    int ray_base;       // first ray of the scene among the iteration's rays
    int64_t n_rays;
    int64_t sample_base;  // first sample slot of the scene
};

struct BatchArgs {
    const BatchScene* scenes;
    int n_scenes, total_rays;
    SampleRec* samples;
    float4* colours;
    int* counts;
    double* acc;
    double* losses;
    int* err;
    int* queue;        // [2] work counters of the placement and shading launches, zeroed per step
    const int* iter;   // the batch's iteration counter (device)
    double mask_coef;
    float huber;
    int grab;          // rays a warp takes per work-counter access in shading
};

struct BatchTuning {
    int place_block = 64;  // threads per block of the placement launch
    int shade_warps = 4;   // warps per block of the shading launch
    int grab = 1;          // rays per warp per work-counter access in shading
    int spl = 1;           // samples a shading lane takes per chunk (shade_warps * spl <= 8)
};

cpx_status batch_launch_march(int prec, const BatchArgs& a, const BatchTuning& tn, cudaStream_t st);
BatchScene batch_scene_view(cpx_grid* g, cpx_rays* r, int len, int pool_batches, int ray_base, int64_t sample_base);

// Per-vertex state of the grid's storage form (api.cu).
cudaError_t alloc_state(cpx_grid* g, int64_t n);
void free_state(cpx_grid* g);

// Launch helpers implemented in the kernel files.
cpx_status march_launch(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                        int mode, double* losses, double mask_coef, float huber,
                        cudaStream_t s);
// The forward+backward march in stages (bit 0: placement, bit 1: shading) on scratch `which`
// (0: the grid's own, 1: the look-ahead step's second one).
cpx_status march_launch_stages(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len, double* losses,
                               double mask_coef, float huber, int which, int stages, cudaStream_t st);
// sweep.cu: the densities the next FP32 dense sweep will write (TV type 0/6 fused when
// fused_tv, else none), written to the density mirror ahead of the sweep, bit for bit.
// The touched map of the batch in the grid's scratch, from its placed samples (the corners of
// every sample's cell), ahead of the shading.
cpx_status mark_touched(cpx_grid* g, int len, cudaStream_t st);
// One pass of the FP32 dense fused sweep: 1 = the vertices the touched map leaves out, 2 = the
// touched ones (and the grid's buffer flips).  Together, the single sweep's results.
cpx_status sweep_adam_pass(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, int pass, cudaStream_t st);
cpx_status density_preview(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, cudaStream_t st);
cpx_status march_launch_with(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                             int mode, double* losses, double mask_coef, float huber,
                             const MarchScratch& s, cudaStream_t st);
int march_samples_per_ray(const cpx_grid* g);
cpx_status march_launch_guided(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                               double* losses, double mask_coef, float huber, const uint32_t* masks,
                               float* seg_w, cudaStream_t st, int mode = kForwardBackward);
// proposal.cu
cpx_status proposal_masks(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                          cudaStream_t st, uint32_t** masks_out);
float* proposal_label_buffer(cpx_proposal* p, int len);
cpx_status proposal_train(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                          const float* seg_w, int steps, int rays_per_step, bool adam, cudaStream_t st);
cpx_status sweep_adam(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr,
                      double sh_lr, int timestep, cudaStream_t s, const int* t_dev = nullptr);
// The batched form's FP32 sweeps in one launch (sweep.cu): grids that qualify (dense FP32, SH
// band 2, fused TV), a device table of sweep_table_bytes(n) filled from the host image that
// sweep_table_fill writes (it returns the launch's rows), then the launch, which flips
// the grids' buffers as sweep_adam does.
bool sweep_batchable(const cpx_grid* g, bool fused_tv);
size_t sweep_table_bytes(int n);
int sweep_table_fill(cpx_grid* const* grids, int n, double lam_d, double lam_sh, double lr, double sh_lr,
                     const int* t_dev, void* host_image);
cpx_status sweep_batched_launch(cpx_grid* const* grids, int n, const void* dev_table, int items, cudaStream_t st);
// Once per process, before any graph capture (grid creation of a mixed form calls it): the
// shared-memory opt-in of the mixed forms' pipelined dense sweep.
cpx_status lowp_prepare();
cpx_status sweep_adam_lowp(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, uint32_t tv_mask, uint32_t adam_mask, cudaStream_t st,
                           const int* t_dev = nullptr);
cpx_status tv_launch(cpx_grid* g, double lam_d, double lam_sh, int type, int nbrs,
                     cudaStream_t s);
cpx_status occupancy_launch(cpx_grid* g, float threshold);
// The occupancy tables from given cell bytes (device, one per cell) instead of the density.
cpx_status occupancy_build(cpx_grid* g, float threshold, const uint8_t* occ_in_dev);
cpx_status make_sparse_launch(cpx_grid* g);
cpx_status rays_camera_launch(cpx_rays* r, const cpx_grid* g, const cpx_camera* cam,
                              int img_w, int64_t plane_bytes, const uint8_t* planes_dev,
                              const int32_t* pix_dev, int64_t n_pix, int64_t offset,
                              int has_mask, cudaStream_t s);
cpx_status mse_launch(const double* losses, int len, double* out, cudaStream_t s);



}  // namespace cpx
