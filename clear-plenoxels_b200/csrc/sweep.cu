// sweep.cu -- TV gradient and Adam over the grid (HBM-bound sweeps).
//
// The reference runs the TV term (RenderUtils.cu:2577-2813, a thread per (x,y)
// column walking z over 28 planar arrays) and then Adam (Optimizer.cu:359-415,
// a thread per vertex over the same 28 arrays) as two passes.  Here the
// default pair -- TV type 0 with 6 neighbours, then Adam -- is one pass: a
// thread owns one 16-byte slot (4 parameters) of one vertex record, reads the
// slot from the current parameter buffer, its 6 neighbours' slots (L1/L2
// resident: the sweep walks z-y-x rows in order, so rows y+-1 and planes z+-1
// are recent), the gradient and both moments, and writes the updated slot to
// the other parameter buffer.  Per vertex that is the algorithmic minimum:
// params r+w, grad r + zero-w, m r+w, v r+w (+4 B density mirror write).
//
// TV and Adam arithmetic is FP32 (the reference mixes double into the TV
// division and the Adam update; the FP32 results differ from it by a few ulp).
// The fused sweep takes its square roots from the hardware approximation
// (sqrt.approx.ftz, about an ulp); the standalone TV kernels keep sqrtf and the
// division by the neighbour count as the reference writes them.
#include "cpx_internal.cuh"

namespace cpx {

struct SweepArgs {
    int W, H, D;
    uint32_t n_act;
    const float4* __restrict__ p_in;
    float4* p_out;
    float4* grad;
    float4* m;
    float4* v;
    float* density_out;
    float* dense_mirror;  // sparse grids: density at dense positions (or null)
    const float* __restrict__ adaptive_lr;
    const uint32_t* __restrict__ index_offsets;
    const uint32_t* __restrict__ compact_to_dense;
    const uint8_t* __restrict__ in_cage;  // dense in-cage flags (sparse TV gate, see k_sweep)
    const uint32_t* __restrict__ touched;  // vertices whose gradients may be non-zero; null = all
    uint32_t* clear;                       // the other touched map, cleared for the next batch
    uint32_t tv_mask;    // bit e: parameter e of a record gets the TV term (RenderUtils.cu:2743-2746)
    uint32_t adam_mask;  // bit e: parameter e is updated by Adam (Optimizer.cu:380-413)
    float lam_d, lam_sh;
    float lr, sh_lr;
    int timestep;
    const int* t_dev;  // when set, the timestep is *t_dev + 1 (a replayed CUDA graph)
    int pass;          // 0: every vertex; 1: untouched vertices only; 2: touched vertices only
    int full_masks;    // every element of a record takes TV and Adam (no padding, no hierarchy)
};

__device__ __forceinline__ float f4get(const float4& v, int c)
{
    return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}
__device__ __forceinline__ void f4set(float4& v, int c, float x)
{
    if (c == 0) v.x = x;
    else if (c == 1) v.y = x;
    else if (c == 2) v.z = x;
    else v.w = x;
}

// Hardware square root (about an ulp), a denormal argument flushed to zero: a TV sum or an Adam
// second moment below 1.2e-38 changes no FP32 result the sweep writes.
__device__ __forceinline__ float sqrt_ftz(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The six-neighbour TV term for one parameter (RenderUtils.cu:2672-2757); neighbours in
// the reference's order z-1, y-1, x-1, x+1, y+1, z+1.
__device__ __forceinline__ float tv6(float self, const float* nb, float lam)
{
    float sum = 0.f, disp = 0.f;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        const float d = self - nb[j];
        sum += d * d;
        disp = (j == 0) ? d : disp + d;
    }
    // sqrt(sum) / 6 (RenderUtils.cu:2708) by the hardware square root and a multiply: the IEEE
    // square root and division take a dozen instructions each with their special-case checks,
    // in a sweep that issues about 450 instructions per slot; the result differs by an ulp or two
    const float sd = sqrt_ftz(sum) * (1.f / 6.f);
    return __fdividef(lam * disp, sd + 1.e-6f);
}

// The arithmetic of one 16-byte slot: optional TV term from the six neighbour slots nbv (the
// reference's order z-1, y-1, x-1, x+1, y+1, z+1), then Adam.  g, m, vv are updated in place
// (g to zero where Adam ran); returns the new parameters.  FULL: every element takes TV and
// Adam (SweepArgs::full_masks), so the per-element mask tests drop out.
template <bool TV, bool FULL = false>
__device__ __forceinline__ float4 slot_update(const SweepArgs& a, int j, bool tv_on, const float4& p,
                                              const float4* nbv, float4& g, float4& m, float4& vv, float inv_bc1,
                                              float inv_bc2, float lr_density)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1.e-6f;
    if (TV && tv_on) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int e = 4 * j + c;
            if (!FULL && !((a.tv_mask >> e) & 1u)) continue;
            float nb[6];
#pragma unroll
            for (int k = 0; k < 6; k++) nb[k] = f4get(nbv[k], c);
            f4set(g, c, f4get(g, c) + tv6(f4get(p, c), nb, e == 0 ? a.lam_d : a.lam_sh));
        }
    }
    float4 pn = p;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int e = 4 * j + c;
        if (!FULL && !((a.adam_mask >> e) & 1u)) continue;
        const float gc = f4get(g, c);
        const float mc = fmaf(1.f - beta1, gc, beta1 * f4get(m, c));
        const float vc = fmaf((1.f - beta2) * gc, gc, beta2 * f4get(vv, c));
        f4set(m, c, mc);
        f4set(vv, c, vc);
        const float lr = e == 0 ? lr_density : a.sh_lr;
        float np = f4get(p, c) - __fdividef(lr * (mc * inv_bc1), sqrt_ftz(vc * inv_bc2) + eps);
        if (e == 0) np = np < 0.f ? 0.f : np;  // density clamp (Optimizer.cu:384)
        f4set(pn, c, np);
        f4set(g, c, 0.f);
    }
    return pn;
}

// One 16-byte slot: optional TV term from six neighbour slots, then Adam; writes the slot.
// touched_bit is shared with the mixed-form sweep (cpx_internal.cuh).
template <bool TV>
__device__ __forceinline__ void sweep_slot(const SweepArgs& a, uint32_t sl, uint32_t v, int j,
                                           bool tv_on, const uint32_t* nb_slot, const bool* nb_self,
                                           float inv_bc1, float inv_bc2, float lr_density)
{
    // untouched vertices have zero gradients: their records are neither read nor written
    const bool tch = touched_bit(a.touched, v);
    if (a.clear && a.pass != 2 && j == 0 && (v & 31u) == 0) a.clear[v >> 5] = 0u;
    if ((a.pass == 1 && tch) || (a.pass == 2 && !tch)) return;  // the other pass's vertex
    const float4 p = a.p_in[sl];
    float4 g = tch ? a.grad[sl] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 m = a.m[sl];
    float4 vv = a.v[sl];
    float4 nbv[6];
    if (TV && tv_on) {
#pragma unroll
        for (int k = 0; k < 6; k++) nbv[k] = nb_self[k] ? p : a.p_in[nb_slot[k]];
    }
    const float4 pn = a.full_masks ? slot_update<TV, true>(a, j, tv_on, p, nbv, g, m, vv, inv_bc1, inv_bc2, lr_density)
                                   : slot_update<TV>(a, j, tv_on, p, nbv, g, m, vv, inv_bc1, inv_bc2, lr_density);
    a.p_out[sl] = pn;
    a.m[sl] = m;
    a.v[sl] = vv;
    if (tch) a.grad[sl] = g;
    if (j == 0) {
        a.density_out[v] = pn.x;
        if (a.dense_mirror) a.dense_mirror[a.compact_to_dense[v]] = pn.x;
    }
}

__device__ __forceinline__ void bias_corrections(int t, const int* t_dev, float* s_bc)
{
    if (threadIdx.x == 0) {
        if (t_dev) t = *t_dev + 1;
        // bias corrections as the reference forms them (powf of the float betas)
        s_bc[0] = 1.f / (float)(1. - powf(0.9f, t));
        s_bc[1] = 1.f / (float)(1. - powf(0.999f, t));
    }
    __syncthreads();
}

// Dense grid: one block per (y, z) row of W vertices, S slots each.
// One (y, z) row of W vertices, S slots each, by a block (s_bc: the bias corrections).
template <int S, bool TV>
__device__ __forceinline__ void sweep_dense_row(const SweepArgs& a, int row, const float* s_bc)
{
    const int y = row % a.H;
    const int z = row / a.H;
    const uint32_t WH = (uint32_t)a.W * a.H;
    const uint32_t v0 = (uint32_t)z * WH + (uint32_t)y * a.W;
    const bool row_interior = y >= 1 && y <= a.H - 2 && z >= 1 && z <= a.D - 2;
    const uint32_t n_slots = (uint32_t)a.W * S;
    for (uint32_t li = threadIdx.x; li < n_slots; li += blockDim.x) {
        const uint32_t x = li / S;
        const int j = (int)(li - x * S);
        const uint32_t v = v0 + x;
        const uint32_t sl = v * S + j;
        const bool tv_on = row_interior && x >= 1 && x + 2 <= (uint32_t)a.W;
        uint32_t nb_slot[6];
        const bool nb_self[6] = {false, false, false, false, false, false};
        nb_slot[0] = sl - WH * S;
        nb_slot[1] = sl - (uint32_t)a.W * S;
        nb_slot[2] = sl - S;
        nb_slot[3] = sl + S;
        nb_slot[4] = sl + (uint32_t)a.W * S;
        nb_slot[5] = sl + WH * S;
        const float lr_d = a.adaptive_lr ? a.lr * a.adaptive_lr[v] : a.lr;
        sweep_slot<TV>(a, sl, v, j, tv_on, nb_slot, nb_self, s_bc[0], s_bc[1], lr_d);
    }
}

// Dense grid: one block per (y, z) row of W vertices, S slots each.
template <int S, bool TV>
__global__ void __launch_bounds__(256) k_sweep_dense(SweepArgs a)
{
    __shared__ float s_bc[2];
    bias_corrections(a.timestep, a.t_dev, s_bc);
    sweep_dense_row<S, TV>(a, blockIdx.x, s_bc);
}

// The density each vertex of a dense FP32 grid will have after the next sweep, written to the
// density mirror ahead of that sweep: slot 0's TV + Adam (slot_update on the same operands, so
// the same bits the sweep writes), nothing else stored.  A look-ahead step places the next
// batch's samples on these densities while the sweep itself runs.
template <int S, bool TV>
__global__ void __launch_bounds__(256) k_density_preview(SweepArgs a)
{
    __shared__ float s_bc[2];
    bias_corrections(a.timestep, a.t_dev, s_bc);
    const uint32_t WH = (uint32_t)a.W * a.H;
    const uint32_t n = WH * (uint32_t)a.D;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t x = v % (uint32_t)a.W;
        const uint32_t y = (v / (uint32_t)a.W) % (uint32_t)a.H;
        const uint32_t z = v / WH;
        const bool tv_on = y >= 1 && y + 2 <= (uint32_t)a.H && z >= 1 && z + 2 <= (uint32_t)a.D && x >= 1 &&
                           x + 2 <= (uint32_t)a.W;
        const uint32_t sl = v * S;
        const float4 p = a.p_in[sl];
        float4 g = touched_bit(a.touched, v) ? a.grad[sl] : make_float4(0.f, 0.f, 0.f, 0.f);
        float4 m = a.m[sl];
        float4 vv = a.v[sl];
        float4 nbv[6];
        if (TV && tv_on) {
            nbv[0] = a.p_in[sl - WH * S];
            nbv[1] = a.p_in[sl - (uint32_t)a.W * S];
            nbv[2] = a.p_in[sl - S];
            nbv[3] = a.p_in[sl + S];
            nbv[4] = a.p_in[sl + (uint32_t)a.W * S];
            nbv[5] = a.p_in[sl + WH * S];
        }
        const float lr_d = a.adaptive_lr ? a.lr * a.adaptive_lr[v] : a.lr;
        const float4 pn = slot_update<TV>(a, 0, tv_on, p, nbv, g, m, vv, s_bc[0], s_bc[1], lr_d);
        a.density_out[v] = pn.x;
    }
}

// The row sweeps of many dense FP32 grids (the batched form) in one launch: block b takes row b
// of the concatenated row lists, its grid found by binary search over the first rows.
struct SweepBatch {
    const SweepArgs* args;  // [n]
    const int* first;       // [n + 1]: first row of each grid, then the total
    int n;
};

template <int S>
__global__ void __launch_bounds__(256) k_sweep_dense_batched(SweepBatch sb)
{
    __shared__ float s_bc[2];
    __shared__ SweepArgs s_args;
    __shared__ int s_row;
    const int item = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = sb.n - 1;  // the last grid whose first row is <= item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sb.first[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        s_args = sb.args[lo];
        s_row = item - sb.first[lo];
    }
    __syncthreads();
    bias_corrections(s_args.timestep, s_args.t_dev, s_bc);
    sweep_dense_row<S, true>(s_args, s_row, s_bc);
}

// Dense grid, TV on: the 2.5-D form.  A block owns a kZTX x kZTY tile of vertex columns and
// walks a chunk of kZChunk planes in z.  A thread owns one 16-byte slot of one column and keeps
// the column's z-1, z and z+1 slots in registers; the tile's current plane (with a one-vertex
// halo in x and y, loaded by the edge threads) is staged in shared memory, where the x- and
// y-neighbours are read.  Every parameter slot then leaves L2 once per block (plus the halo),
// instead of once for itself and once for each neighbour that needs it.  The arithmetic is
// slot_update's, so the results equal k_sweep_dense's bit for bit.
constexpr int kZTX = 16, kZTY = 8, kZChunk = 32;
static_assert(kZTX > 1 && kZTY > 1, "a column is at most one of left/right and of top/bottom");

template <int S>
struct ZPlane {
    float4 v[kZTY + 2][kZTX + 2][S];
};

// One block's work: tile (bx, by), chunk bz of grid a; s_bc holds a's bias corrections.
template <int S>
__device__ __forceinline__ void sweep_dense_z_tile(const SweepArgs& a, int bx, int by, int bz, const float* s_bc,
                                                   ZPlane<S>& pl)
{
    auto& plane = pl.v;
    const int t = threadIdx.x;
    const int col = t / S;
    const int j = t - col * S;
    const int tx = col % kZTX, ty = col / kZTX;
    const int x = bx * kZTX + tx, y = by * kZTY + ty;
    const int z0 = bz * kZChunk;
    const int z1 = z0 + kZChunk < a.D ? z0 + kZChunk : a.D;
    const bool in = x < a.W && y < a.H;
    const uint32_t W = (uint32_t)a.W, WH = W * (uint32_t)a.H;
    const uint32_t cv = (uint32_t)y * W + (uint32_t)x;  // the column's vertex in a plane
    const bool xy_interior = x >= 1 && x + 2 <= a.W && y >= 1 && y <= a.H - 2;
    const bool left = in && tx == 0 && x >= 1;
    const bool right = in && tx == kZTX - 1 && x + 1 < a.W;
    const bool top = in && ty == 0 && y >= 1;
    const bool bottom = in && ty == kZTY - 1 && y + 1 < a.H;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 p_prev = zero, p_cur = zero;
    if (in) {
        if (z0 >= 1) p_prev = a.p_in[((uint32_t)(z0 - 1) * WH + cv) * S + j];
        p_cur = a.p_in[((uint32_t)z0 * WH + cv) * S + j];
    }
    for (int z = z0; z < z1; z++) {
        const uint32_t v = (uint32_t)z * WH + cv;
        const uint32_t sl = v * S + j;
        // every load of this plane first: the next plane's slot, the halo, the optimizer state
        // (a column is at most one of left/right and one of top/bottom: the tile is wider and
        // taller than one vertex)
        float4 p_next = zero, hx = zero, hy = zero;
        float4 g = zero, m = zero, vv = zero;
        bool tch = false;
        float lr = a.lr;
        if (in) {
            if (z + 1 < a.D) p_next = a.p_in[sl + WH * S];
            if (left) hx = a.p_in[sl - S];
            else if (right) hx = a.p_in[sl + S];
            if (top) hy = a.p_in[sl - W * S];
            else if (bottom) hy = a.p_in[sl + W * S];
            tch = touched_bit(a.touched, v);
            if (tch) g = a.grad[sl];
            m = a.m[sl];
            vv = a.v[sl];
            if (a.adaptive_lr) lr = a.lr * a.adaptive_lr[v];
        }
        plane[ty + 1][tx + 1][j] = p_cur;
        if (left) plane[ty + 1][0][j] = hx;
        else if (right) plane[ty + 1][kZTX + 1][j] = hx;
        if (top) plane[0][tx + 1][j] = hy;
        else if (bottom) plane[kZTY + 1][tx + 1][j] = hy;
        __syncthreads();
        if (in) {
            if (a.clear && j == 0 && (v & 31u) == 0) a.clear[v >> 5] = 0u;
            const bool tv_on = xy_interior && z >= 1 && z <= a.D - 2;
            float4 nbv[6];
            if (tv_on) {
                nbv[0] = p_prev;
                nbv[1] = plane[ty][tx + 1][j];
                nbv[2] = plane[ty + 1][tx][j];
                nbv[3] = plane[ty + 1][tx + 2][j];
                nbv[4] = plane[ty + 2][tx + 1][j];
                nbv[5] = p_next;
            }
            const float4 pn = slot_update<true>(a, j, tv_on, p_cur, nbv, g, m, vv, s_bc[0], s_bc[1], lr);
            a.p_out[sl] = pn;
            a.m[sl] = m;
            a.v[sl] = vv;
            if (tch) a.grad[sl] = g;
            if (j == 0) a.density_out[v] = pn.x;
        }
        __syncthreads();
        p_prev = p_cur;
        p_cur = p_next;
    }
}

template <int S>
__global__ void __launch_bounds__(kZTX * kZTY * S, 1) k_sweep_dense_z(SweepArgs a)
{
    __shared__ float s_bc[2];
    __shared__ ZPlane<S> plane;
    bias_corrections(a.timestep, a.t_dev, s_bc);
    sweep_dense_z_tile<S>(a, blockIdx.x, blockIdx.y, blockIdx.z, s_bc, plane);
}

// Tiles of a dense grid for k_sweep_dense_z: (x tiles, y tiles, z chunks).
__host__ __device__ __forceinline__ dim3 z_tiles(int W, int H, int D)
{
    return dim3((unsigned)((W + kZTX - 1) / kZTX), (unsigned)((H + kZTY - 1) / kZTY),
                (unsigned)((D + kZChunk - 1) / kZChunk));
}

// Sparse grid: blocks tile the compact slots; positions from the compact->dense table.
template <int S, bool TV>
__global__ void __launch_bounds__(256) k_sweep_sparse(SweepArgs a)
{
    // A warp takes 32 consecutive compact vertices: each lane works out one vertex's TV
    // neighbourhood once (the dense position, its flags and six neighbour lookups), and the
    // warp's 32 * S slots -- consecutive slots on consecutive lanes -- take it by shuffle.
    __shared__ float s_bc[2];
    bias_corrections(a.timestep, a.t_dev, s_bc);
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t v0 = warp * 32u;
    if (v0 >= a.n_act) return;  // warp-uniform
    SparseTv mine;
    mine.flags = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) mine.nb[k] = 0;
    if (TV && v0 + lane < a.n_act)
        mine = sparse_tv(v0 + lane, a.compact_to_dense, a.in_cage, a.index_offsets, a.W, a.H, a.D);
#pragma unroll
    for (int it = 0; it < S; it++) {
        const uint32_t i = it * 32u + lane;
        const uint32_t vl = i / S;
        const int j = (int)(i - vl * S);
        const SparseTv t = TV ? shfl_tv(mine, (int)vl) : mine;
        const uint32_t v = v0 + vl;
        if (v >= a.n_act) continue;
        uint32_t nb_slot[6];
        bool nb_self[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            nb_self[k] = (t.flags >> k) & 1u;
            nb_slot[k] = t.nb[k] * S + j;
        }
        sweep_slot<TV>(a, v * S + j, v, j, (t.flags >> 6) & 1u, nb_slot, nb_self, s_bc[0], s_bc[1], a.lr);
    }
}

template <int S>
static void launch_sweep(const cpx_grid* g, const SweepArgs& a, bool tv, cudaStream_t st)
{
    if (!g->sparse) {
        const unsigned rows = (unsigned)((int64_t)g->H * g->D);
        if (tv && S == 7 && (g->options & CPX_OPT_PLANE_SWEEP) && !g->sparse) {
            k_sweep_dense_z<S><<<z_tiles(g->W, g->H, g->D), kZTX * kZTY * S, 0, st>>>(a);
        } else if (tv) {
            k_sweep_dense<S, true><<<rows, 256, 0, st>>>(a);
        } else {
            k_sweep_dense<S, false><<<rows, 256, 0, st>>>(a);
        }
    } else {
        const unsigned blocks = (unsigned)(((int64_t)g->n_act + 255) / 256);  // a warp per 32 vertices
        if (tv)
            k_sweep_sparse<S, true><<<blocks, 256, 0, st>>>(a);
        else
            k_sweep_sparse<S, false><<<blocks, 256, 0, st>>>(a);
    }
}

// Element masks of a record (element e: 0 density, 1 + c*sh_dim + k SH, >= n_arrays padding).
static void element_masks(const cpx_grid* g, uint32_t* tv_mask, uint32_t* adam_mask)
{
    uint32_t tvm = 0, am = 0;
    const int lo_tv = g->hierarchy ? g->band * g->band : 0;
    const int hi = (g->band + 1) * (g->band + 1);
    for (int e = 0; e < g->rec; e++) {
        bool t = false, ad = false;
        if (e == 0) {
            t = ad = true;
        } else if (e < g->n_arrays) {
            const int k = (e - 1) % g->sh_dim;
            t = k >= lo_tv && k < hi;
            ad = !g->hierarchy || (k >= g->band * g->band && k < hi);
        }
        if (t) tvm |= 1u << e;
        if (ad) am |= 1u << e;
    }
    *tv_mask = tvm;
    *adam_mask = am;
}

static SweepArgs sweep_args(const cpx_grid* g, double lam_d, double lam_sh, double lr, double sh_lr, int timestep,
                            const int* t_dev);

cpx_status sweep_adam(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr,
                      double sh_lr, int timestep, cudaStream_t st, const int* t_dev)
{
    ++g->epoch;  // new densities: a placement done in advance on the old ones is stale
    if (g->n_act == 0) return CPX_OK;
    if (g->prec != kPrecFP32) {
        uint32_t tvm, am;
        element_masks(g, &tvm, &am);
        cpx_status rc = sweep_adam_lowp(g, fused_tv, lam_d, lam_sh, lr, sh_lr, timestep, tvm, am, st, t_dev);
        return rc == CPX_OK ? refresh_dense_skip(g, st) : rc;  // the new density's empty cells
    }
    const int S = g->rec / 4;
    if (g->n_act * S >= ((int64_t)1 << 32)) {
        set_error("grid too large for 32-bit slot indices");
        return CPX_ERR_UNSUPPORTED;
    }
    const SweepArgs a = sweep_args(g, lam_d, lam_sh, lr, sh_lr, timestep, t_dev);
    switch (S) {
    case 1: launch_sweep<1>(g, a, fused_tv, st); break;
    case 4: launch_sweep<4>(g, a, fused_tv, st); break;
    case 7: launch_sweep<7>(g, a, fused_tv, st); break;
    default:
        set_error("record of %d slots unsupported", S);
        return CPX_ERR_UNSUPPORTED;
    }
    count_launch();
    g->cur ^= 1;
    g->tcur ^= 1;
    g->all_touched = 0;
    cpx_status rc = cuda_status(cudaGetLastError(), "adam sweep");
    return rc == CPX_OK ? refresh_dense_skip(g, st) : rc;
}

// The arguments of a grid's FP32 sweep in its current state.
static SweepArgs sweep_args(const cpx_grid* g, double lam_d, double lam_sh, double lr, double sh_lr, int timestep,
                            const int* t_dev)
{
    SweepArgs a;
    a.W = g->W;
    a.H = g->H;
    a.D = g->D;
    a.n_act = (uint32_t)g->n_act;
    a.p_in = reinterpret_cast<const float4*>(g->params[g->cur]);
    a.p_out = reinterpret_cast<float4*>(g->params[g->cur ^ 1]);
    a.grad = reinterpret_cast<float4*>(g->grad);
    a.m = reinterpret_cast<float4*>(g->m);
    a.v = reinterpret_cast<float4*>(g->v);
    a.density_out = g->density;
    a.dense_mirror = g->sparse ? g->dense_mirror : nullptr;
    a.adaptive_lr = g->sparse ? nullptr : g->adaptive_lr;
    a.index_offsets = g->index_offsets;
    a.compact_to_dense = g->compact_to_dense;
    a.in_cage = g->in_cage;
    a.touched = g->all_touched ? nullptr : g->touched[g->tcur];
    a.clear = g->touched[g->tcur ^ 1];
    element_masks(g, &a.tv_mask, &a.adam_mask);
    const uint32_t all = g->rec >= 32 ? 0xffffffffu : (1u << g->rec) - 1u;
    a.full_masks = (a.tv_mask & all) == all && (a.adam_mask & all) == all ? 1 : 0;
    a.lam_d = (float)lam_d;
    a.lam_sh = (float)lam_sh;
    a.lr = (float)lr;
    a.sh_lr = (float)sh_lr;
    a.timestep = timestep;
    a.t_dev = t_dev;
    a.pass = 0;
    return a;
}

cpx_status sweep_adam_pass(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, int pass, cudaStream_t st)
{
    if (g->prec != kPrecFP32 || g->sparse || g->rec != 28 || g->n_act * 7 >= ((int64_t)1 << 32) ||
        (g->options & CPX_OPT_PLANE_SWEEP) || g->all_touched || (pass != 1 && pass != 2)) {
        set_error("the split sweep runs on dense FP32 grids of SH band 2 with a touched map");
        return CPX_ERR_UNSUPPORTED;
    }
    ++g->epoch;
    if (g->n_act == 0) return CPX_OK;
    SweepArgs a = sweep_args(g, lam_d, lam_sh, lr, sh_lr, timestep, nullptr);
    a.pass = pass;
    launch_sweep<7>(g, a, fused_tv, st);
    count_launch();
    cpx_status rc = cuda_status(cudaGetLastError(), "adam sweep pass");
    if (rc != CPX_OK || pass == 1) return rc;
    g->cur ^= 1;
    g->tcur ^= 1;
    g->all_touched = 0;
    return refresh_dense_skip(g, st);
}

cpx_status density_preview(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, cudaStream_t st)
{
    if (g->prec != kPrecFP32 || g->sparse || g->rec != 28 || g->n_act * 7 >= ((int64_t)1 << 32)) {
        set_error("the density preview runs on dense FP32 grids of SH band 2");
        return CPX_ERR_UNSUPPORTED;
    }
    const SweepArgs a = sweep_args(g, lam_d, lam_sh, lr, sh_lr, timestep, nullptr);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (g->n_act + 255) / 256;
    const unsigned blocks = (unsigned)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
    if (fused_tv)
        k_density_preview<7, true><<<blocks, 256, 0, st>>>(a);
    else
        k_density_preview<7, false><<<blocks, 256, 0, st>>>(a);
    count_launch();
    return cuda_status(cudaGetLastError(), "density preview");
}

bool sweep_batchable(const cpx_grid* g, bool fused_tv)
{
    return fused_tv && g->prec == kPrecFP32 && !g->sparse && g->rec == 28 && g->n_act > 0 &&
           g->n_act * 7 < ((int64_t)1 << 32);
}

size_t sweep_table_bytes(int n) { return (size_t)n * sizeof(SweepArgs) + ((size_t)n + 1) * sizeof(int); }

int sweep_table_fill(cpx_grid* const* grids, int n, double lam_d, double lam_sh, double lr, double sh_lr,
                     const int* t_dev, void* host_image)
{
    SweepArgs* args = static_cast<SweepArgs*>(host_image);
    int* first = reinterpret_cast<int*>(args + n);
    int items = 0;
    for (int i = 0; i < n; i++) {
        args[i] = sweep_args(grids[i], lam_d, lam_sh, lr, sh_lr, 1, t_dev);
        first[i] = items;
        items += grids[i]->H * grids[i]->D;  // rows
    }
    first[n] = items;
    return items;
}

cpx_status sweep_batched_launch(cpx_grid* const* grids, int n, const void* dev_table, int items, cudaStream_t st)
{
    if (n == 0) return CPX_OK;
    SweepBatch sb;
    sb.args = static_cast<const SweepArgs*>(dev_table);
    sb.first = reinterpret_cast<const int*>(sb.args + n);
    sb.n = n;
    k_sweep_dense_batched<7><<<(unsigned)items, 256, 0, st>>>(sb);
    count_launch();
    for (int i = 0; i < n; i++) {
        cpx_grid* g = grids[i];
        ++g->epoch;
        g->cur ^= 1;
        g->tcur ^= 1;
        g->all_touched = 0;
        cpx_status rc = refresh_dense_skip(g, st);
        if (rc != CPX_OK) return rc;
    }
    return cuda_status(cudaGetLastError(), "batched sweep");
}

// ---------------------------------------------------------------------------
// Standalone TV gradient (RenderUtils::addVarianceLoss, RenderUtils.cu:2815-2851).
// ---------------------------------------------------------------------------
struct TvArgs {
    int W, H, D, rec, n_arrays, sh_dim, band, hierarchy, sparse, optimize_step;
    const float* __restrict__ p;
    float* grad;
    const uint32_t* __restrict__ index_offsets;
    const uint8_t* __restrict__ in_cage;
    const uint8_t* __restrict__ occ;
    float lam_d, lam_sh;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t nb_index(const TvArgs& a, int x, int y, int z)
{
    x = clampi(x, 0, a.W - 1);
    y = clampi(y, 0, a.H - 1);
    z = clampi(z, 0, a.D - 1);
    uint32_t v = (uint32_t)(z * a.W * a.H + y * a.W + x);
    return a.sparse ? a.index_offsets[v] : v;
}

// Type 0: one thread per vertex (x,y interior, z in the reference's range), all
// parameters of the vertex, 3 / 6 / 26 neighbours with the reference's quirks.
__global__ void k_tv_type0(TvArgs a, int nbrs)
{
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nplane = (int64_t)a.W * a.H;
    if (tid >= nplane * a.D) return;
    const int z = (int)(tid / nplane);
    const int y = (int)((tid / a.W) % a.H);
    const int x = (int)(tid % a.W);
    if (y == 0 || y == a.H - 1 || x == 0 || x == a.W - 1) return;
    if (nbrs == 3) {
        if (z > a.D - 2) return;  // depth 0 .. D-2 (RenderUtils.cu:2608)
    } else if (z < 1 || z > a.D - 2) {
        return;
    }
    uint32_t ix[27];
    for (int dz = -1; dz < 2; dz++)
        for (int dy = -1; dy < 2; dy++)
            for (int dx = -1; dx < 2; dx++)
                ix[(dz + 1) * 9 + (dy + 1) * 3 + dx + 1] = nb_index(a, x + dx, y + dy, z + dz);
    if (a.sparse) {
        // the reference's gate inCageInfo[indexOffsets[v]] (RenderUtils.cu:2669, 2608, 2770):
        // the dense flag array read at the compact index.  Non-caged vertices (compact index 0)
        // are skipped outright: when dense vertex 0 is in cage the reference would add racy
        // terms to compact vertex 0 from every such position, which is not reproduced.
        const uint32_t dv = (uint32_t)(z * a.W * a.H + y * a.W + x);
        if (!a.in_cage[dv] || !a.in_cage[ix[13]]) return;
    }
    const int startSH = a.hierarchy ? a.band * a.band : 0;
    const int endSH = (a.band + 1) * (a.band + 1);
    float slot4 = 0.f;  // neighbour array slot 4 as left by the previous parameter (26 case)
    for (int e = 0; e < a.n_arrays; e++) {
        if (e > 0) {
            const int k = (e - 1) % a.sh_dim;
            if (k < startSH || k >= endSH) continue;
        }
        const float lam = e == 0 ? a.lam_d : a.lam_sh;
        auto val = [&](uint32_t i) { return a.p[(size_t)i * a.rec + e]; };
        const float self = val(ix[13]);
        float sum = 0.f, disp = 0.f, sd;
        if (nbrs == 3) {
            const float n14 = ix[14] != 0 ? val(ix[14]) : self;
            sum += (self - n14) * (self - n14);
            const float n16 = ix[16] != 0 ? val(ix[16]) : self;
            sum += (self - n16) * (self - n16);
            const bool have22 = e == 0 ? ix[22] != 0 : ix[4] != 0;  // RenderUtils.cu:2650
            const float n22 = have22 ? val(ix[22]) : self;
            disp = self - n22;
            sum += (self - n22) * (self - n22);
            sd = sqrtf(sum) / 3.f;
        } else if (nbrs == 6) {
            const int nb[6] = {4, 10, 12, 14, 16, 22};
            for (int j = 0; j < 6; j++) {
                const float nv = ix[nb[j]] != 0 ? val(ix[nb[j]]) : self;
                sum += (self - nv) * (self - nv);
                disp = j == 0 ? self - nv : disp + (self - nv);
            }
            sd = sqrtf(sum) / 6.f;
        } else {
            for (int j = 0; j < 27; j++) {
                if (j == 13) continue;
                const float nv = ix[j] != 0 ? val(ix[j]) : self;
                if (j == 4) slot4 = nv;
                sum += (self - nv) * (self - nv);
                disp += e == 0 ? self - nv : self - slot4;
            }
            sd = sqrtf(sum) / 26.f;
        }
        float* gp = a.grad + (size_t)ix[13] * a.rec + e;
        *gp = *gp + lam / (sd + 1.e-6f) * disp;
    }
}

// Type 1 voxel disparity (RenderUtils.cu:2469-2547): one thread per cell; the shared
// corners are accumulated with atomics (the reference's unsynchronised += is racy).
__global__ void k_tv_type1(TvArgs a)
{
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int Wc = a.W - 1, Hc = a.H - 1, Dc = a.D - 1;
    if (tid >= (int64_t)Wc * Hc * Dc) return;
    const int x = (int)(tid % Wc);
    const int y = (int)((tid / Wc) % Hc);
    const int z = (int)(tid / ((int64_t)Wc * Hc));
    if (a.sparse && !a.occ[tid]) return;
    uint32_t ix[8];
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) ix[dz * 4 + dy * 2 + dx] = nb_index(a, x + dx, y + dy, z + dz);
    const int startSH = a.hierarchy ? a.band * a.band : 0;
    const int endSH = (a.band + 1) * (a.band + 1);
    for (int e = 0; e < a.n_arrays; e++) {
        float lam = a.lam_d;
        if (e > 0) {
            if (a.optimize_step > 1) continue;
            const int k = (e - 1) % a.sh_dim;
            if (k < startSH || k >= endSH) continue;
            lam = a.lam_sh;
        }
        float mean = 0.f;
        for (int i = 0; i < 8; i++) {
            const float pv = a.p[(size_t)ix[i] * a.rec + e];
            mean += e == 0 ? pv : pv / 8.f;
        }
        if (e == 0) mean /= 8.f;
        for (int i = 0; i < 8; i++)
            atomicAdd(a.grad + (size_t)ix[i] * a.rec + e, lam * (a.p[(size_t)ix[i] * a.rec + e] - mean));
    }
}

cpx_status tv_launch(cpx_grid* g, double lam_d, double lam_sh, int type, int nbrs,
                     cudaStream_t st)
{
    if (type < 0 || type > 2 || (type != 1 && nbrs != 3 && nbrs != 6 && nbrs != 26)) {
        set_error("TV type %d with %d neighbours is not defined", type, nbrs);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse && !g->have_occupancy) {
        set_error("sparse grid without occupancy");
        return CPX_ERR_NOT_READY;
    }
    if (g->prec != kPrecFP32) {
        set_error("the mixed forms run TV type 0 / 6 neighbours fused into the optimizer sweep only");
        return CPX_ERR_UNSUPPORTED;
    }
    g->all_touched = 1;  // TV writes gradients of vertices no ray touched
    TvArgs a;
    a.W = g->W;
    a.H = g->H;
    a.D = g->D;
    a.rec = g->rec;
    a.n_arrays = g->n_arrays;
    a.sh_dim = g->sh_dim;
    a.band = g->band;
    a.hierarchy = g->hierarchy;
    a.sparse = g->sparse;
    a.optimize_step = g->optimize_step;
    a.p = g->params[g->cur];
    a.grad = g->grad;
    a.index_offsets = g->index_offsets;
    a.in_cage = g->in_cage;
    a.occ = g->occ_bytes;
    a.lam_d = (float)lam_d;
    a.lam_sh = (float)lam_sh;
    if (type == 0 || type == 2) {
        const int64_t n = g->n_dense;
        k_tv_type0<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, nbrs);
        count_launch();
    }
    if (type == 1 || type == 2) {
        const int64_t c = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
        k_tv_type1<<<(unsigned)((c + 255) / 256), 256, 0, st>>>(a);
        count_launch();
    }
    return cuda_status(cudaGetLastError(), "tv");
}

}  // namespace cpx
