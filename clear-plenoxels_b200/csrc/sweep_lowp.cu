// sweep_lowp.cu -- fused TV (type 0, 6 neighbours) + Adam sweep of the mixed forms.
//
// Same order of operations as the FP32 sweep (TV term added to the gradient, then Adam
// with the reference's bias corrections and density clamp, Optimizer.cu:359-415), over the
// mixed storage: density FP32, SH in 16-bit records, gradients in FP32 records, moments in
// bfloat16 records.  Like the FP32 sweep, a thread owns 4 consecutive parameters (one quad)
// of one vertex: it reads their SH (8 B), gradients (16 B), moments (2 x 8 B), and for quad 0
// the density, applies TV and Adam in FP32, and writes the new SH, moments and density back
// with stochastic rounding to 16 bits, zeroing the gradients it consumed.  Per vertex at SH
// band 2: density r+w 8 B, SH r+w 112 B, gradients r + zero-w 224 B, moments r+w 224 B
// (+4 B learning-rate multiplier on dense grids): 572 B against the FP32 form's 904 B.
#include "cpx_internal.cuh"

namespace cpx {

struct LowpArgs {
    int W, H, D;
    uint32_t n_act;
    const float* __restrict__ d_in;
    float* d_out;
    float* dense_mirror;  // sparse grids: density at dense positions (or null)
    const uint2* __restrict__ sh_in;  // 4 x 16-bit per quad
    uint2* sh_out;
    float4* grad;  // FP32 gradient records, S float4 per vertex
    uint2* m;      // bfloat16 moments, 4 per quad
    uint2* v;
    const float* __restrict__ adaptive_lr;
    const uint32_t* __restrict__ index_offsets;
    const uint32_t* __restrict__ compact_to_dense;
    const uint8_t* __restrict__ in_cage;
    const uint32_t* __restrict__ touched;  // vertices whose gradients may be non-zero; null = all
    uint32_t* clear;                       // the other touched map, cleared for the next batch
    uint32_t tv_mask, adam_mask;
    float lam_d, lam_sh, lr, sh_lr;
    int timestep;
    uint32_t step_key;  // hash of (stochastic-rounding seed, timestep)
    const int* t_dev;   // when set, the timestep is *t_dev + 1 (a replayed CUDA graph)
    uint32_t seed;
};

__device__ __forceinline__ void bits4(const uint2& q, uint16_t* h)
{
    h[0] = (uint16_t)(q.x & 0xffffu);
    h[1] = (uint16_t)(q.x >> 16);
    h[2] = (uint16_t)(q.y & 0xffffu);
    h[3] = (uint16_t)(q.y >> 16);
}

// Square root through the hardware reciprocal square root (about 2 ulp; the results are
// stored in 16 bits), 0 for 0.
__device__ __forceinline__ float fast_sqrt(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

// Quad j (record slots 4j..4j+3) of vertex v; S quads per record.  The six-neighbour TV term (RenderUtils.cu:2672-2757, neighbours in
// the reference's order z-1, y-1, x-1, x+1, y+1, z+1) streams one neighbour quad at a time.
template <int PREC, int S, bool TV>
__device__ __forceinline__ void lowp_quad(const LowpArgs& a, uint32_t v, int j, bool tv_on,
                                          const uint32_t* nb_v, const bool* nb_self, float inv_bc1,
                                          float inv_bc2, float lr_density, uint32_t step_key)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1.e-6f;
    const size_t q = (size_t)v * S + j;
    const uint2 sh_raw = a.sh_in[q];
    uint16_t sh_bits[4];
    bits4(sh_raw, sh_bits);
    float p[4];
    unpack4<PREC>(sh_raw, p);
    if (j == 0) p[0] = a.d_in[v];  // slot 0 of an SH record is unused: density is FP32
    // untouched vertices have zero gradients: their records are neither read nor written
    const bool tch = touched_bit(a.touched, v);
    if (a.clear && j == 0 && (v & 31u) == 0) a.clear[v >> 5] = 0u;
    const float4 g4 = tch ? a.grad[(size_t)v * S + j] : make_float4(0.f, 0.f, 0.f, 0.f);
    float g[4] = {g4.x, g4.y, g4.z, g4.w};
    uint16_t m_bits[4], v_bits[4];
    bits4(a.m[q], m_bits);
    bits4(a.v[q], v_bits);
    if (TV && tv_on) {
        float sum[4] = {0.f, 0.f, 0.f, 0.f}, disp[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float nb[4];
            if (nb_self[k]) {
#pragma unroll
                for (int c = 0; c < 4; c++) nb[c] = p[c];
            } else {
                const size_t nq = (size_t)nb_v[k] * S + j;
                unpack4<PREC>(a.sh_in[nq], nb);
                if (j == 0) nb[0] = a.d_in[nb_v[k]];
            }
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float d = p[c] - nb[c];
                sum[c] += d * d;
                disp[c] = (k == 0) ? d : disp[c] + d;
            }
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int e = 4 * j + c;
            if ((a.tv_mask >> e) & 1u) {
                const float sd = fast_sqrt(sum[c]) * (1.f / 6.f);
                g[c] += __fdividef((e == 0 ? a.lam_d : a.lam_sh) * disp[c], sd + 1.e-6f);
            }
        }
    }
    // random bits: one hash of (launch key, vertex, quad), then one cheap draw per element
    const uint32_t h1 = fmix32(step_key ^ (v * 0x632BE5ABu) ^ ((uint32_t)j << 28));
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int e = 4 * j + c;
        if (!((a.adam_mask >> e) & 1u)) continue;
        const float gc = g[c];
        const float mc = fmaf(1.f - beta1, gc, beta1 * bf16_to_f(m_bits[c]));
        const float vc = fmaf((1.f - beta2) * gc, gc, beta2 * bf16_to_f(v_bits[c]));
        const float lr = e == 0 ? lr_density : a.sh_lr;
        float np = p[c] - __fdividef(lr * (mc * inv_bc1), fast_sqrt(vc * inv_bc2) + eps);
        // one 32-bit draw per element: the low half rounds the parameter, the high half
        // both moments
        const uint32_t r = draw32(h1 + (uint32_t)c * 0x9E3779B9u, 0x85EBCA6Bu);
        if (e == 0) {
            np = np < 0.f ? 0.f : np;  // density clamp (Optimizer.cu:384)
            a.d_out[v] = np;
            if (a.dense_mirror) a.dense_mirror[a.compact_to_dense[v]] = np;
        } else {
            sh_bits[c] = f_to_sh_sr<PREC>(np, r & 0xffffu);
        }
        m_bits[c] = f_to_bf16_sr(mc, r >> 16);
        v_bits[c] = f_to_bf16_sr(vc, r >> 16);
        g[c] = 0.f;
    }
    if (j == 0 && !(a.adam_mask & 1u)) {
        a.d_out[v] = p[0];
        if (a.dense_mirror) a.dense_mirror[a.compact_to_dense[v]] = p[0];
    }
    a.sh_out[q] = pack4(sh_bits);
    a.m[q] = pack4(m_bits);
    a.v[q] = pack4(v_bits);
    if (tch) a.grad[(size_t)v * S + j] = make_float4(g[0], g[1], g[2], g[3]);
}

// Bias corrections and the stochastic-rounding key of this step into shared memory.
__device__ __forceinline__ void lowp_bias_corrections(const LowpArgs& a, float* s_bc, uint32_t* s_key)
{
    if (threadIdx.x == 0) {
        const int t = a.t_dev ? *a.t_dev + 1 : a.timestep;
        s_bc[0] = 1.f / (float)(1. - powf(0.9f, t));
        s_bc[1] = 1.f / (float)(1. - powf(0.999f, t));
        *s_key = a.t_dev ? fmix32(a.seed ^ ((uint32_t)t * 0x9E3779B9u)) : a.step_key;
    }
    __syncthreads();
}

// Dense grid: one block per (y, z) row of W vertices, S quads each.
template <int PREC, int S, bool TV>
__global__ void __launch_bounds__(256) k_sweep_lowp_dense(LowpArgs a)
{
    __shared__ float s_bc[2];
    __shared__ uint32_t s_key;
    lowp_bias_corrections(a, s_bc, &s_key);
    const int row = blockIdx.x;
    const int y = row % a.H;
    const int z = row / a.H;
    const uint32_t WH = (uint32_t)a.W * a.H;
    const uint32_t v0 = (uint32_t)z * WH + (uint32_t)y * a.W;
    const bool row_interior = y >= 1 && y <= a.H - 2 && z >= 1 && z <= a.D - 2;
    const uint32_t n = (uint32_t)a.W * S;
    for (uint32_t li = threadIdx.x; li < n; li += blockDim.x) {
        const uint32_t x = li / S;
        const int j = (int)(li - x * S);
        const uint32_t v = v0 + x;
        const bool tv_on = row_interior && x >= 1 && x + 2 <= (uint32_t)a.W;
        const uint32_t nb_v[6] = {v - WH, v - (uint32_t)a.W, v - 1u, v + 1u, v + (uint32_t)a.W, v + WH};
        const bool nb_self[6] = {false, false, false, false, false, false};
        const float lr_d = a.adaptive_lr ? a.lr * a.adaptive_lr[v] : a.lr;
        lowp_quad<PREC, S, TV>(a, v, j, tv_on, nb_v, nb_self, s_bc[0], s_bc[1], lr_d, s_key);
    }
}

// Sparse grid: blocks tile the compact (vertex, quad) pairs.
template <int PREC, int S, bool TV>
__global__ void __launch_bounds__(256) k_sweep_lowp_sparse(LowpArgs a)
{
    // A warp takes 32 consecutive compact vertices; each lane works out one vertex's TV
    // neighbourhood and the warp's 32 * S quads take it by shuffle (as the FP32 sparse sweep).
    __shared__ float s_bc[2];
    __shared__ uint32_t s_key;
    lowp_bias_corrections(a, s_bc, &s_key);
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
        bool nb_self[6];
#pragma unroll
        for (int k = 0; k < 6; k++) nb_self[k] = (t.flags >> k) & 1u;
        lowp_quad<PREC, S, TV>(a, v, j, (t.flags >> 6) & 1u, t.nb, nb_self, s_bc[0], s_bc[1], a.lr, s_key);
    }
}

template <int PREC, int S>
static void launch_lowp(const cpx_grid* g, const LowpArgs& a, bool tv, cudaStream_t st)
{
    if (!g->sparse) {
        const unsigned rows = (unsigned)((int64_t)g->H * g->D);
        if (tv)
            k_sweep_lowp_dense<PREC, S, true><<<rows, 256, 0, st>>>(a);
        else
            k_sweep_lowp_dense<PREC, S, false><<<rows, 256, 0, st>>>(a);
    } else {
        const unsigned blocks = (unsigned)(((int64_t)g->n_act + 255) / 256);  // a warp per 32 vertices
        if (tv)
            k_sweep_lowp_sparse<PREC, S, true><<<blocks, 256, 0, st>>>(a);
        else
            k_sweep_lowp_sparse<PREC, S, false><<<blocks, 256, 0, st>>>(a);
    }
}

template <int PREC>
static cpx_status launch_lowp_shape(const cpx_grid* g, const LowpArgs& a, bool tv, cudaStream_t st)
{
    // quads per record: 4 parameters -> 1, 13 -> 4, 28 -> 7
    switch (g->sh_dim) {
    case 1: launch_lowp<PREC, 1>(g, a, tv, st); break;
    case 4: launch_lowp<PREC, 4>(g, a, tv, st); break;
    case 9: launch_lowp<PREC, 7>(g, a, tv, st); break;
    default:
        set_error("sh_dim %d unsupported", g->sh_dim);
        return CPX_ERR_UNSUPPORTED;
    }
    return CPX_OK;
}

cpx_status sweep_adam_lowp(cpx_grid* g, bool fused_tv, double lam_d, double lam_sh, double lr, double sh_lr,
                           int timestep, uint32_t tv_mask, uint32_t adam_mask, cudaStream_t st, const int* t_dev)
{
    if (g->n_act * (g->rec / 4) >= ((int64_t)1 << 32)) {
        set_error("grid too large for 32-bit quad indices");
        return CPX_ERR_UNSUPPORTED;
    }
    LowpArgs a;
    a.W = g->W;
    a.H = g->H;
    a.D = g->D;
    a.n_act = (uint32_t)g->n_act;
    a.d_in = g->dens[g->cur];
    a.d_out = g->dens[g->cur ^ 1];
    a.dense_mirror = g->sparse ? g->dense_mirror : nullptr;
    a.sh_in = reinterpret_cast<const uint2*>(g->sh16[g->cur]);
    a.sh_out = reinterpret_cast<uint2*>(g->sh16[g->cur ^ 1]);
    a.grad = reinterpret_cast<float4*>(g->grad);
    a.m = reinterpret_cast<uint2*>(g->m16);
    a.v = reinterpret_cast<uint2*>(g->v16);
    a.adaptive_lr = g->sparse ? nullptr : g->adaptive_lr;
    a.index_offsets = g->index_offsets;
    a.compact_to_dense = g->compact_to_dense;
    a.in_cage = g->in_cage;
    a.touched = g->all_touched ? nullptr : g->touched[g->tcur];
    a.clear = g->touched[g->tcur ^ 1];
    a.tv_mask = tv_mask;
    a.adam_mask = adam_mask;
    a.lam_d = (float)lam_d;
    a.lam_sh = (float)lam_sh;
    a.lr = (float)lr;
    a.sh_lr = (float)sh_lr;
    a.timestep = timestep;
    a.step_key = fmix32(g->sr_seed ^ ((uint32_t)timestep * 0x9E3779B9u));
    a.t_dev = t_dev;
    a.seed = g->sr_seed;
    cpx_status rc = g->prec == kPrecFP16 ? launch_lowp_shape<kPrecFP16>(g, a, fused_tv, st)
                                         : launch_lowp_shape<kPrecBF16>(g, a, fused_tv, st);
    if (rc != CPX_OK) return rc;
    count_launch();
    g->cur ^= 1;
    g->density = g->dens[g->cur];
    g->tcur ^= 1;
    g->all_touched = 0;
    return cuda_status(cudaGetLastError(), "mixed adam sweep");
}

}  // namespace cpx
