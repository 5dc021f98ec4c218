// proposal.cu -- learned sample-interval proposal for the march (no reference counterpart).
//
// Each ray's [near, far] is cut into 32 equal segments.  A small MLP (48 -> 64 -> 64 -> 64
// -> 1, ReLU) predicts from the segment midpoint (position in box coordinates and its
// 4-octave sin/cos encoding), the ray direction and the ray origin whether the segment holds
// visible density (label: the samples of a full march inside the segment carry total weight
// above a threshold -- empty and occluded segments are both 0).  The march skips the segments
// predicted empty with confidence (sigmoid(logit) <= 1 - confidence) and marches every other
// segment in full, so a ray whose predictions are all uncertain runs the plain full march.
//
// Inference runs on the 5th-generation tensor cores: a persistent CTA of 128 threads takes
// tiles of 128 points (4 rays x 32 segments); each thread writes its point's features to
// shared memory as BF16 in the MMA's canonical K-major layout, one thread issues
// tcgen05.mma (M=128, N=64, K=16 steps, FP32 accumulators in tensor memory), and after the
// commit's mbarrier arrives every thread reads its row back with tcgen05.ld, adds the bias,
// applies ReLU and writes the next layer's BF16 operand.  The last layer (64 -> 1) is a dot
// product in FP32 registers, and each warp (= one ray) turns its 32 logits into a segment
// mask with a ballot.  Training uses FP32 CUDA cores (the network is 11.5k parameters): a
// block takes 128 points, runs forward and backward through shared memory, reduces the
// weight gradients over its points and adds them to the global gradient, then Adam.
#include "cpx_internal.cuh"

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace cpx {
namespace prop {

constexpr int kSeg = kProposalSegments;  // 32
constexpr int kFeat = 33;                // used input features
constexpr int kIn = 48;                  // input width, padded to the MMA's K step (16)
constexpr int kHid = 64;
constexpr int kRows = 128;  // points per tile = 4 rays

// FP32 parameter block, offsets in floats
constexpr int oW1 = 0;                 // [64][48] (row n = output, column k = input)
constexpr int oB1 = oW1 + kHid * kIn;  // [64]
constexpr int oW2 = oB1 + kHid;        // [64][64]
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;  // [64][64]
constexpr int oB3 = oW3 + kHid * kHid;
constexpr int oW4 = oB3 + kHid;  // [64]
constexpr int oB4 = oW4 + kHid;  // [1]
constexpr int kParams = oB4 + 1;

// BF16 weight pack: W1, W2, W3 in the canonical K-major layout (no swizzle)
constexpr int kW1Elems = kHid * kIn;
constexpr int kW2Elems = kHid * kHid;
constexpr int kPackElems = kW1Elems + 2 * kW2Elems;

// Shared memory of the inference kernel (bytes).  The operand regions sit at the start of
// a 100 KB allocation, so every address an MMA descriptor can form from them stays inside.
constexpr int sW1 = 0;
constexpr int sW2 = sW1 + kW1Elems * 2;  // 6144
constexpr int sW3 = sW2 + kW2Elems * 2;  // 14336
constexpr int sA0 = sW3 + kW2Elems * 2;  // 22528
constexpr int sA1 = sA0 + kRows * kHid * 2;  // 38912
constexpr int kInferSmem = 100 * 1024;
// The last MMA step of an A operand starts at sA1 + 3 * 4096; read with the leading and stride
// offsets exchanged it would reach 15 * 2048 + 256 bytes further.
static_assert(sA1 + 3 * 2 * kRows * 16 + 15 * kRows * 16 + 256 <= kInferSmem, "operand guard space");

// Element offset of (row r, column k) in a canonical K-major BF16 operand of R rows: core
// matrices of 8 rows x 8 columns (16 B rows), 8-row groups 128 B apart, 8-column chunks
// R*16 B apart.
__host__ __device__ constexpr int canon(int r, int k, int R) { return (k >> 3) * (R * 8) + (r >> 3) * 64 + (r & 7) * 8 + (k & 7); }

struct Args {
    RaysView r;
    const int32_t* sidx;
    int start, len;
    int64_t n_rays;
    float sx, sy, sz;  // 2 / (axis vertices - 1): voxel -> [-1, 1]
    float conf_logit;  // |logit| of a decided segment
    const float* __restrict__ params;
    const uint16_t* __restrict__ wpack;
    uint32_t* seg_mask;  // [len] (or null)
    float* logits;       // [len][32] (or null)
    int* err;
    unsigned long long* n_skipped;  // segments predicted confidently empty
};

// ---------------------------------------------------------------------------
// Features
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ray_of(const Args& a, int b, int64_t& ri, bool& valid)
{
    valid = b < a.len;
    ri = 0;
    if (!valid) return;
    ri = a.sidx ? (int64_t)a.sidx[a.start + b] : (int64_t)a.start + b;
    if (ri < 0 || ri >= a.n_rays) {
        valid = false;
        ri = 0;
    }
}

// Features of segment s of ray ri (zero for an invalid ray), f[0..47].
__device__ __forceinline__ void features(const Args& a, int64_t ri, bool valid, int s, float* f)
{
#pragma unroll
    for (int i = 0; i < kIn; i++) f[i] = 0.f;
    if (!valid) return;
    const float o[3] = {a.r.ox[ri], a.r.oy[ri], a.r.oz[ri]};
    const float d[3] = {a.r.dx[ri], a.r.dy[ri], a.r.dz[ri]};
    const float nr = a.r.near_t[ri], fr = a.r.far_t[ri];
    const float t = nr + ((float)s + 0.5f) * (fr - nr) * (1.f / kSeg);
    const float sc[3] = {a.sx, a.sy, a.sz};
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        const float x = (o[ax] + t * d[ax]) * sc[ax] - 1.f;
        f[ax] = x;
        float w = 3.14159265358979f * x;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float sn, cs;
            sincosf(w, &sn, &cs);
            f[3 + 6 * k + 2 * ax] = sn;
            f[4 + 6 * k + 2 * ax] = cs;
            w *= 2.f;
        }
        f[27 + ax] = d[ax];
        f[30 + ax] = (o[ax] * sc[ax] - 1.f) * 0.25f;
    }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (canonical K-major core matrices).
__device__ __forceinline__ uint64_t mat_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: kind::f16, D = F32, A = B = BF16, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHid >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for phase `parity` of the mbarrier, for about a second at most.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

// Row `row` (128-row operand) <- 8 values of chunk c, as one 16-byte store.
__device__ __forceinline__ void store_chunk(uint16_t* A, int row, int c, const float* v)
{
    uint4 q;
    q.x = (uint32_t)bf16_bits(v[0]) | ((uint32_t)bf16_bits(v[1]) << 16);
    q.y = (uint32_t)bf16_bits(v[2]) | ((uint32_t)bf16_bits(v[3]) << 16);
    q.z = (uint32_t)bf16_bits(v[4]) | ((uint32_t)bf16_bits(v[5]) << 16);
    q.w = (uint32_t)bf16_bits(v[6]) | ((uint32_t)bf16_bits(v[7]) << 16);
    *reinterpret_cast<uint4*>(A + canon(row, 8 * c, kRows)) = q;
}

// D[128 x 64] = A[128 x K] * W[64 x K]^T into TMEM; every thread returns once it has landed.
__device__ __forceinline__ bool mma_layer(uint32_t a_base, uint32_t w_base, int ksteps, uint32_t tmem,
                                          uint32_t mbar, uint32_t& phase)
{
    if (threadIdx.x == 0) {
        fence_after();
        for (int ks = 0; ks < ksteps; ks++) {
            // a 16-column step covers two 8-column chunks
            const uint64_t ad = mat_desc(a_base + ks * 2 * (kRows * 16), kRows * 16, 128);
            const uint64_t bd = mat_desc(w_base + ks * 2 * (kHid * 16), kHid * 16, 128);
            mma_bf16(tmem, ad, bd, ks > 0 ? 1u : 0u);
        }
        mma_commit(mbar);
    }
    const bool ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    fence_after();
    // block-uniform, so the .sync.aligned TMEM loads that follow run on whole warps
    return __syncthreads_and(ok) != 0;
}

// This thread's row of the accumulator, bias, ReLU -> next operand (8 chunks of 8).
__device__ __forceinline__ void epilogue_hidden(uint32_t tmem, const float* bias, uint16_t* A_next, int row)
{
    const uint32_t taddr = tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
    float v[kHid];
#pragma unroll
    for (int q = 0; q < 4; q++) tmem_ld16(taddr + 16 * q, v + 16 * q);
    tmem_wait_ld();
#pragma unroll
    for (int c = 0; c < 8; c++) {
        float h[8];
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = fmaxf(v[8 * c + i] + bias[8 * c + i], 0.f);
        store_chunk(A_next, row, c, h);
    }
}

// ---------------------------------------------------------------------------
// Inference on the tensor cores
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_infer_tc(Args a)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar_store;
    __shared__ uint32_t tmem_slot;
    __shared__ float s_b[3][kHid];
    __shared__ float s_w4[kHid];
    __shared__ float s_b4;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint16_t* A0 = reinterpret_cast<uint16_t*>(smem + sA0);
    uint16_t* A1 = reinterpret_cast<uint16_t*>(smem + sA1);
    const uint32_t base = smem_addr(smem);
    const uint32_t mbar = smem_addr(&mbar_store);

    // weights (BF16, canonical) and the FP32 vectors
    for (int i = tid; i < kPackElems / 8; i += blockDim.x)
        reinterpret_cast<uint4*>(smem)[i] = reinterpret_cast<const uint4*>(a.wpack)[i];
    for (int i = tid; i < kHid; i += blockDim.x) {
        s_b[0][i] = a.params[oB1 + i];
        s_b[1][i] = a.params[oB2 + i];
        s_b[2][i] = a.params[oB3 + i];
        s_w4[i] = a.params[oW4 + i];
    }
    if (tid == 0) {
        s_b4 = a.params[oB4];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(kHid)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    uint32_t phase = 0;
    bool failed = false;
    const int n_tiles = (a.len + 3) / 4;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int b = tile * 4 + warp;  // this warp's ray; lane = segment
        int64_t ri;
        bool valid;
        ray_of(a, b, ri, valid);
        {
            float f[kIn];
            features(a, ri, valid, lane, f);
#pragma unroll
            for (int c = 0; c < kIn / 8; c++) store_chunk(A0, tid, c, f + 8 * c);
        }
        fence_async_smem();
        __syncthreads();
        if (!mma_layer(base + sA0, base + sW1, kIn / 16, tmem, mbar, phase)) {
            failed = true;
            break;
        }
        epilogue_hidden(tmem, s_b[0], A1, tid);
        fence_async_smem();
        fence_before();
        __syncthreads();
        if (!mma_layer(base + sA1, base + sW2, kHid / 16, tmem, mbar, phase)) {
            failed = true;
            break;
        }
        epilogue_hidden(tmem, s_b[1], A0, tid);
        fence_async_smem();
        fence_before();
        __syncthreads();
        if (!mma_layer(base + sA0, base + sW3, kHid / 16, tmem, mbar, phase)) {
            failed = true;
            break;
        }
        float logit = s_b4;
        {
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
            float v[kHid];
#pragma unroll
            for (int q = 0; q < 4; q++) tmem_ld16(taddr + 16 * q, v + 16 * q);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < kHid; i++) logit = fmaf(fmaxf(v[i] + s_b[2][i], 0.f), s_w4[i], logit);
        }
        fence_before();
        __syncthreads();
        // march every segment that is not confidently empty
        const uint32_t mask = __ballot_sync(0xffffffffu, !(logit <= -a.conf_logit));
        if (valid) {
            if (a.logits) a.logits[(size_t)b * kSeg + lane] = logit;
            if (lane == 0) {
                if (a.seg_mask) a.seg_mask[b] = mask;
                if (a.n_skipped) atomicAdd(a.n_skipped, (unsigned long long)(kSeg - __popc(mask)));
            }
        }
    }
    if (failed) {
        // an MMA did not complete within the wait's limit: report it, give the outstanding
        // commit one more bounded wait, then release the tensor memory
        if (tid == 0) atomicOr(a.err, 4);
        mbar_wait(mbar, phase ^ 1u);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kHid) : "memory");
}

// ---------------------------------------------------------------------------
// FP32 forward on the CUDA cores (training, and the check of the tensor-core path)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float forward_f32(const float* P, const float* x, float* h1, float* h2, float* h3)
{
    for (int n = 0; n < kHid; n++) {
        float s = P[oB1 + n];
        for (int k = 0; k < kIn; k++) s = fmaf(P[oW1 + n * kIn + k], x[k], s);
        h1[n] = fmaxf(s, 0.f);
    }
    for (int n = 0; n < kHid; n++) {
        float s = P[oB2 + n];
        for (int k = 0; k < kHid; k++) s = fmaf(P[oW2 + n * kHid + k], h1[k], s);
        h2[n] = fmaxf(s, 0.f);
    }
    float z = P[oB4];
    for (int n = 0; n < kHid; n++) {
        float s = P[oB3 + n];
        for (int k = 0; k < kHid; k++) s = fmaf(P[oW3 + n * kHid + k], h2[k], s);
        h3[n] = fmaxf(s, 0.f);
        z = fmaf(h3[n], P[oW4 + n], z);
    }
    return z;
}

__global__ void __launch_bounds__(128) k_infer_f32(Args a)
{
    extern __shared__ float sP[];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sP[i] = a.params[i];
    __syncthreads();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n_tiles = (a.len + 3) / 4;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int b = tile * 4 + warp;
        int64_t ri;
        bool valid;
        ray_of(a, b, ri, valid);
        float f[kIn], h1[kHid], h2[kHid], h3[kHid];
        features(a, ri, valid, lane, f);
        const float logit = forward_f32(sP, f, h1, h2, h3);
        const uint32_t mask = __ballot_sync(0xffffffffu, !(logit <= -a.conf_logit));
        if (valid) {
            if (a.logits) a.logits[(size_t)b * kSeg + lane] = logit;
            if (lane == 0 && a.seg_mask) a.seg_mask[b] = mask;
        }
    }
}

// ---------------------------------------------------------------------------
// Training: forward + backward of 128 points per block, weight gradients reduced per block
// ---------------------------------------------------------------------------
struct TrainArgs {
    Args a;                  // rays, batch and parameters
    const float* seg_w;      // [len][32] segment weights of a full march (labels)
    float label_weight;      // label = seg_w > label_weight
    float inv_points;        // 1 / points of this step (mean loss)
    float* grad;             // [kParams], accumulated
    double* loss;            // sum of the points' losses, accumulated
};

// Dynamic shared memory of k_train (floats): the parameter block, then one row per point of
// the input and of every hidden activation.  Row strides are odd, so the 32 lanes of a warp,
// each reading its own row at the same column, fall in 32 different banks.
constexpr int kSX = kIn + 1;
constexpr int kSH = kHid + 1;
constexpr int tP = 0;
constexpr int tX = tP + ((kParams + 3) & ~3);
constexpr int tH1 = tX + kRows * kSX;
constexpr int tH2 = tH1 + kRows * kSH;
constexpr int tH3 = tH2 + kRows * kSH;
constexpr int tD = tH3 + kRows * kSH;
constexpr int tDz = tD + kRows * kSH;
constexpr int kTrainSmemFloats = tDz + kRows;
static_assert(kTrainSmemFloats * 4 <= 227 * 1024, "k_train shared memory");
static_assert(oW1 % 4 == 0 && oW2 % 4 == 0 && oW3 % 4 == 0 && kIn % 4 == 0, "float4 weight rows");

// out[n] = relu(b[n] + sum_k W[n][k] r[k]) for the thread's own point, its input row r held in
// registers.  Four outputs advance together (four independent FMA chains) on float4 broadcast
// loads of the weight rows; each output still sums bias first, then k ascending, as
// forward_f32 does.  With Z, also returns b4 + sum_n out[n] w4[n] in n order.
template <int KI, bool Z>
__device__ __forceinline__ float layer_fwd(const float* P, int oW, int oB, const float (&r)[KI], float* out)
{
    float z = Z ? P[oB4] : 0.f;
#pragma unroll 1
    for (int n = 0; n < kHid; n += 4) {
        float s[4];
#pragma unroll
        for (int u = 0; u < 4; u++) s[u] = P[oB + n + u];
#pragma unroll
        for (int k = 0; k < KI; k += 4) {
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float4 w = *reinterpret_cast<const float4*>(P + oW + (n + u) * KI + k);
                s[u] = fmaf(w.x, r[k], s[u]);
                s[u] = fmaf(w.y, r[k + 1], s[u]);
                s[u] = fmaf(w.z, r[k + 2], s[u]);
                s[u] = fmaf(w.w, r[k + 3], s[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float h = fmaxf(s[u], 0.f);
            out[n + u] = h;
            if (Z) z = fmaf(h, P[oW4 + n + u], z);
        }
    }
    return z;
}

// out[k] = act[k] > 0 ? sum_n W[n][k] g[n] : 0 (W is kHid x kHid, row n = output), the
// back-propagated gradient of one point, g in registers; four k together on float4 loads, n
// ascending.
__device__ __forceinline__ void layer_bwd(const float* P, int oW, const float (&g)[kHid], const float* act, float* out)
{
#pragma unroll 1
    for (int k = 0; k < kHid; k += 4) {
        float s[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int n = 0; n < kHid; n++) {
            const float4 w = *reinterpret_cast<const float4*>(P + oW + n * kHid + k);
            s[0] = fmaf(w.x, g[n], s[0]);
            s[1] = fmaf(w.y, g[n], s[1]);
            s[2] = fmaf(w.z, g[n], s[2]);
            s[3] = fmaf(w.w, g[n], s[3]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) out[k + u] = act[k + u] > 0.f ? s[u] : 0.f;
    }
}

// out[i][j] += sum_p A[p][i] * B[p][j] for i < kHid, j < NJ over the block's 128 points (row
// strides sa, sb): each thread sums a 4 x NJ/8 tile in registers, p ascending, and adds it to
// the global gradient with atomics.  Points whose four A values are all zero (ReLU) are
// skipped; a zero A value adds nothing to the other sums either.
template <int NJ>
__device__ __forceinline__ void outer_reduce(const float* A, int sa, const float* B, int sb, float* out)
{
    constexpr int TJ = NJ / 8;
    static_assert(NJ % 8 == 0 && kHid == 4 * 16 && kRows == 128, "tile split");
    const int i0 = (threadIdx.x >> 3) * 4, j0 = (threadIdx.x & 7) * TJ;
    float acc[4][TJ];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < TJ; b++) acc[a][b] = 0.f;
    for (int p = 0; p < kRows; p++) {
        float av[4], bv[TJ];
#pragma unroll
        for (int a = 0; a < 4; a++) av[a] = A[p * sa + i0 + a];
        if (av[0] == 0.f && av[1] == 0.f && av[2] == 0.f && av[3] == 0.f) continue;
#pragma unroll
        for (int b = 0; b < TJ; b++) bv[b] = B[p * sb + j0 + b];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < TJ; b++) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < TJ; b++)
            if (acc[a][b] != 0.f) atomicAdd(out + (i0 + a) * NJ + j0 + b, acc[a][b]);
}

// column sum over the block's points of a hidden-activation region (bias gradients)
__device__ __forceinline__ void column_sum(const float* R, float* out)
{
    const int tid = threadIdx.x;
    if (tid < kHid) {
        float s = 0.f;
        for (int p = 0; p < kRows; p++) s += R[p * kSH + tid];
        if (s != 0.f) atomicAdd(out + tid, s);
    }
}

__global__ void __launch_bounds__(128) k_train(TrainArgs t)
{
    extern __shared__ float4 train_smem[];
    float* sm = reinterpret_cast<float*>(train_smem);
    const Args& a = t.a;
    float* P = sm + tP;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) P[i] = a.params[i];
    __syncthreads();
    const int tid = threadIdx.x, lane = tid & 31;
    const int b = blockIdx.x * 4 + (tid >> 5);
    int64_t ri;
    bool valid;  // one ray per warp: uniform across the warp
    ray_of(a, b, ri, valid);
    float* x = sm + tX + tid * kSX;
    float* h1 = sm + tH1 + tid * kSH;
    float* h2 = sm + tH2 + tid * kSH;
    float* h3 = sm + tH3 + tid * kSH;
    float* d = sm + tD + tid * kSH;
    float z;
    {
        float r[kIn];
        features(a, ri, valid, lane, r);
#pragma unroll
        for (int k = 0; k < kIn; k++) x[k] = r[k];
        layer_fwd<kIn, false>(P, oW1, oB1, r, h1);
    }
    {
        float r[kHid];
#pragma unroll
        for (int k = 0; k < kHid; k++) r[k] = h1[k];
        layer_fwd<kHid, false>(P, oW2, oB2, r, h2);
    }
    {
        float r[kHid];
#pragma unroll
        for (int k = 0; k < kHid; k++) r[k] = h2[k];
        z = layer_fwd<kHid, true>(P, oW3, oB3, r, h3);
    }
    float dz = 0.f;
    double l = 0.;
    if (valid) {
        const float y = t.seg_w[(size_t)b * kSeg + lane] > t.label_weight ? 1.f : 0.f;
        const float sg = 1.f / (1.f + expf(-z));
        dz = (sg - y) * t.inv_points;
        // binary cross-entropy with logits: softplus(z) - y z
        l = fmaxf(z, 0.f) - y * z + log1pf(expf(-fabsf(z)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (valid && lane == 0) atomicAdd(t.loss, l);
    sm[tDz + tid] = dz;
    // layer 4 and d3 = dz * w4 * relu'(h3)
#pragma unroll 4
    for (int n = 0; n < kHid; n++) d[n] = h3[n] > 0.f ? dz * P[oW4 + n] : 0.f;
    __syncthreads();
    // dW4 = sum dz h3, db4 = sum dz
    if (tid < kHid) {
        float s = 0.f;
        for (int p = 0; p < kRows; p++) s = fmaf(sm[tDz + p], sm[tH3 + p * kSH + tid], s);
        if (s != 0.f) atomicAdd(t.grad + oW4 + tid, s);
    } else if (tid == kHid) {
        float s = 0.f;
        for (int p = 0; p < kRows; p++) s += sm[tDz + p];
        if (s != 0.f) atomicAdd(t.grad + oB4, s);
    }
    // dW3 = sum d3 x h2, db3 = sum d3
    outer_reduce<kHid>(sm + tD, kSH, sm + tH2, kSH, t.grad + oW3);
    column_sum(sm + tD, t.grad + oB3);
    __syncthreads();
    // d2 = (W3^T d3) * relu'(h2), kept in h3's place
    {
        float g[kHid];
#pragma unroll
        for (int n = 0; n < kHid; n++) g[n] = d[n];
        layer_bwd(P, oW3, g, h2, h3);
    }
    __syncthreads();
    outer_reduce<kHid>(sm + tH3, kSH, sm + tH1, kSH, t.grad + oW2);
    column_sum(sm + tH3, t.grad + oB2);
    __syncthreads();
    // d1 = (W2^T d2) * relu'(h1), kept in d
    {
        float g[kHid];
#pragma unroll
        for (int n = 0; n < kHid; n++) g[n] = h3[n];
        layer_bwd(P, oW2, g, h1, d);
    }
    __syncthreads();
    outer_reduce<kIn>(sm + tD, kSH, sm + tX, kSX, t.grad + oW1);
    column_sum(sm + tD, t.grad + oB1);
}

__global__ void k_adam(float* p, float* g, float* m, float* v, int n, float lr, float inv_bc1, float inv_bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * inv_bc1) / (sqrtf(vi * inv_bc2) + 1e-8f);
    g[i] = 0.f;
}

// W1, W2, W3 of the FP32 block -> BF16 canonical operands
__global__ void k_pack(const float* P, uint16_t* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kPackElems) return;
    int n, k, R = kHid, base, src;
    if (i < kW1Elems) {
        n = i / kIn;
        k = i % kIn;
        base = 0;
        src = oW1 + n * kIn + k;
    } else {
        const int j = i - kW1Elems;
        const int layer = j / kW2Elems, e = j % kW2Elems;
        n = e / kHid;
        k = e % kHid;
        base = kW1Elems + layer * kW2Elems;
        src = (layer == 0 ? oW2 : oW3) + n * kHid + k;
    }
    out[base + canon(n, k, R)] = bf16_bits(P[src]);
}

}  // namespace prop
}  // namespace cpx

using namespace cpx;
using namespace cpx::prop;

struct cpx_proposal {
    cpx_proposal_desc desc;
    float* params = nullptr;  // [kParams] FP32 master
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    uint16_t* wpack = nullptr;
    int* err = nullptr;
    double* loss = nullptr;
    unsigned long long* n_skipped = nullptr;
    int adam_t = 0;
    int rounds = 0;  // completed training rounds
    uint32_t* seg_mask = nullptr;
    int mask_cap = 0;
    float* seg_w = nullptr;
    int segw_cap = 0;
    int sms = 0;
};

namespace cpx {

// Seeded parameter initialisation (uniform He init of the ReLU layers; the output bias starts
// at -2 so an untrained network decides no segment with confidence 0.9).
static void init_params(uint32_t seed, std::vector<float>& P)
{
    P.assign(kParams, 0.f);
    uint64_t s = 0x9E3779B97F4A7C15ull ^ seed;
    auto uni = [&s]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int n_out, int n_in, int used_in) {
        const double bound = std::sqrt(6.0 / used_in);
        for (int o = 0; o < n_out; o++)
            for (int i = 0; i < n_in; i++) P[off + o * n_in + i] = i < used_in ? (float)((2 * uni() - 1) * bound) : 0.f;
    };
    fill(oW1, kHid, kIn, kFeat);
    fill(oW2, kHid, kHid, kHid);
    fill(oW3, kHid, kHid, kHid);
    for (int i = 0; i < kHid; i++) P[oW4 + i] = (float)((2 * uni() - 1) * std::sqrt(1.0 / kHid));
    P[oB4] = -2.f;
}

static cpx_status pack(cpx_proposal* p, cudaStream_t st)
{
    k_pack<<<(kPackElems + 255) / 256, 256, 0, st>>>(p->params, p->wpack);
    count_launch();
    return cuda_status(cudaGetLastError(), "proposal pack");
}

static Args make_args(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len)
{
    Args a;
    a.r = rays_view(r);
    a.sidx = sidx;
    a.start = start;
    a.len = len;
    a.n_rays = r->n;
    a.sx = 2.f / (float)(g->W - 1);
    a.sy = 2.f / (float)(g->H - 1);
    a.sz = 2.f / (float)(g->D - 1);
    const double c = p->desc.confidence;
    a.conf_logit = (float)std::log(c / (1.0 - c));
    a.params = p->params;
    a.wpack = p->wpack;
    a.seg_mask = nullptr;
    a.logits = nullptr;
    a.err = p->err;
    a.n_skipped = p->n_skipped;
    return a;
}

static cpx_status check_batch(cpx_rays* r, const int32_t* sidx, int start, int len)
{
    if (!r || len < 0 || start < 0 || (!sidx && (int64_t)start + len > r->n)) {
        set_error("batch [%d, %d) outside the ray table", start, start + len);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return CPX_OK;
}

cpx_status proposal_masks(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                          cudaStream_t st, uint32_t** masks_out)
{
    if (p->mask_cap < len) {
        cudaFree(p->seg_mask);
        p->seg_mask = nullptr;
        p->mask_cap = 0;
        if (cudaMalloc((void**)&p->seg_mask, (size_t)(len > 0 ? len : 1) * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            set_error("proposal masks could not be allocated");
            return CPX_ERR_OUT_OF_MEMORY;
        }
        p->mask_cap = len;
    }
    *masks_out = p->seg_mask;
    if (len == 0) return CPX_OK;
    Args a = make_args(p, g, r, sidx, start, len);
    a.seg_mask = p->seg_mask;
    const int tiles = (len + 3) / 4;
    const int grid = tiles < 2 * p->sms ? tiles : 2 * p->sms;
    k_infer_tc<<<grid, 128, kInferSmem, st>>>(a);
    count_launch();
    return cuda_status(cudaGetLastError(), "proposal inference");
}

float* proposal_label_buffer(cpx_proposal* p, int len)
{
    if (p->segw_cap < len) {
        cudaFree(p->seg_w);
        p->seg_w = nullptr;
        p->segw_cap = 0;
        if (cudaMalloc((void**)&p->seg_w, (size_t)(len > 0 ? len : 1) * kSeg * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        p->segw_cap = len;
    }
    return p->seg_w;
}

cpx_status proposal_train(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                          const float* seg_w, int steps, int rays_per_step, bool adam, cudaStream_t st)
{
    if (len == 0 || steps <= 0) return CPX_OK;
    if (rays_per_step <= 0 || rays_per_step > len) rays_per_step = len;
    rays_per_step = (rays_per_step + 3) & ~3;
    cudaMemsetAsync(p->loss, 0, sizeof(double), st);
    for (int s = 0; s < steps; s++) {
        const int first = (int)(((int64_t)s * rays_per_step) % len);
        const int n = first + rays_per_step <= len ? rays_per_step : len - first;
        TrainArgs t;
        t.a = make_args(p, g, r, sidx, start + first, n);
        t.seg_w = seg_w + (size_t)first * kSeg;
        t.label_weight = p->desc.label_weight;
        t.inv_points = 1.f / (float)(n * kSeg);
        t.grad = p->grad;
        t.loss = p->loss;
        k_train<<<(n + 3) / 4, 128, kTrainSmemFloats * sizeof(float), st>>>(t);
        count_launch();
        if (!adam) break;
        p->adam_t++;
        const float bc1 = 1.f / (1.f - std::pow(0.9f, (float)p->adam_t));
        const float bc2 = 1.f / (1.f - std::pow(0.999f, (float)p->adam_t));
        k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(p->params, p->grad, p->m, p->v, kParams, p->desc.learning_rate,
                                                     bc1, bc2);
        count_launch();
    }
    if (adam) {
        p->rounds++;
        return pack(p, st);
    }
    return cuda_status(cudaGetLastError(), "proposal training");
}

}  // namespace cpx

extern "C" {

int cpx_proposal_param_count(void) { return kParams; }

cpx_status cpx_proposal_create(const cpx_proposal_desc* d, cpx_proposal** out)
{
    if (!d || !out) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (!(d->confidence > 0.5f && d->confidence < 1.f) || !(d->label_weight >= 0.f) || !(d->learning_rate > 0.f)) {
        set_error("proposal confidence must lie in (0.5, 1), label weight >= 0, learning rate > 0");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
        cudaFuncSetAttribute(k_infer_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, kParams * (int)sizeof(float));
        cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmemFloats * (int)sizeof(float));
        attr_set = true;
    }
    cpx_proposal* p = new (std::nothrow) cpx_proposal();
    if (!p) return CPX_ERR_OUT_OF_MEMORY;
    p->desc = *d;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaSuccess;
    const size_t pb = kParams * sizeof(float);
    float** bufs[4] = {&p->params, &p->grad, &p->m, &p->v};
    for (auto b : bufs) {
        if (e == cudaSuccess) e = cudaMalloc((void**)b, pb);
        if (e == cudaSuccess) e = cudaMemset(*b, 0, pb);
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->wpack, kPackElems * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->loss, sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->n_skipped, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(p->n_skipped, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        std::vector<float> P;
        init_params(d->seed, P);
        e = cudaMemcpy(p->params, P.data(), pb, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        cpx_status s = pack(p, 0);
        if (s == CPX_OK) e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        cpx_proposal_destroy(p);
        return cuda_status(e, "proposal create");
    }
    *out = p;
    return CPX_OK;
}

cpx_status cpx_proposal_destroy(cpx_proposal* p)
{
    if (!p) return CPX_OK;
    cudaDeviceSynchronize();
    cudaFree(p->params);
    cudaFree(p->grad);
    cudaFree(p->m);
    cudaFree(p->v);
    cudaFree(p->wpack);
    cudaFree(p->err);
    cudaFree(p->loss);
    cudaFree(p->n_skipped);
    cudaFree(p->seg_mask);
    cudaFree(p->seg_w);
    delete p;
    return CPX_OK;
}

cpx_status cpx_proposal_params(cpx_proposal* p, float* host, int upload)
{
    if (!p || !host) return CPX_ERR_INVALID_ARGUMENT;
    cudaError_t e;
    if (upload) {
        e = cudaMemcpy(p->params, host, kParams * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && pack(p, 0) == CPX_OK) e = cudaDeviceSynchronize();
    } else {
        e = cudaMemcpy(host, p->params, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    }
    return cuda_status(e, "proposal params");
}

cpx_status cpx_proposal_infer(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start,
                              int len, float* logits_dev, uint32_t* masks_dev, int tensor_cores, cpx_stream stream)
{
    if (!p || !g) return CPX_ERR_INVALID_ARGUMENT;
    if (check_batch(r, sidx, start, len)) return CPX_ERR_INVALID_ARGUMENT;
    if (len == 0) return CPX_OK;
    cudaStream_t st = (cudaStream_t)stream;
    Args a = make_args(p, g, r, sidx, start, len);
    a.logits = logits_dev;
    a.seg_mask = masks_dev;
    const int tiles = (len + 3) / 4;
    if (tensor_cores) {
        const int grid = tiles < 2 * p->sms ? tiles : 2 * p->sms;
        k_infer_tc<<<grid, 128, kInferSmem, st>>>(a);
    } else {
        const int grid = tiles < 8 * p->sms ? tiles : 8 * p->sms;
        k_infer_f32<<<grid, 128, kParams * sizeof(float), st>>>(a);
    }
    count_launch();
    return cuda_status(cudaGetLastError(), "proposal inference");
}

cpx_status cpx_proposal_gradient(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start,
                                 int len, const float* seg_weights_dev, float* grad_host, double* loss_out)
{
    if (!p || !g || !seg_weights_dev || !grad_host) return CPX_ERR_INVALID_ARGUMENT;
    if (check_batch(r, sidx, start, len)) return CPX_ERR_INVALID_ARGUMENT;
    cudaMemset(p->grad, 0, kParams * sizeof(float));
    cpx_status s = proposal_train(p, g, r, sidx, start, len, seg_weights_dev, 1, len, false, 0);
    if (s != CPX_OK) return s;
    cudaError_t e = cudaMemcpy(grad_host, p->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    double l = 0.;
    if (e == cudaSuccess) e = cudaMemcpy(&l, p->loss, sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemset(p->grad, 0, kParams * sizeof(float));
    if (loss_out) *loss_out = l / ((double)len * kSeg);
    return cuda_status(e, "proposal gradient");
}

cpx_status cpx_proposal_train(cpx_proposal* p, const cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start,
                              int len, const float* seg_weights_dev, int steps, int rays_per_step, double* loss_out,
                              cpx_stream stream)
{
    if (!p || !g || !seg_weights_dev) return CPX_ERR_INVALID_ARGUMENT;
    if (check_batch(r, sidx, start, len)) return CPX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    cpx_status s = proposal_train(p, g, r, sidx, start, len, seg_weights_dev, steps, rays_per_step, true, st);
    if (s != CPX_OK || !loss_out) return s;
    double l = 0.;
    cudaError_t e = cudaMemcpyAsync(&l, p->loss, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const int per = rays_per_step <= 0 || rays_per_step > len ? len : rays_per_step;
    *loss_out = l / ((double)steps * per * kSeg);
    return cuda_status(e, "proposal training");
}

cpx_status cpx_proposal_stats(cpx_proposal* p, int* rounds, int64_t* skipped_segments, int* error_flags)
{
    if (!p) return CPX_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaDeviceSynchronize();
    unsigned long long c = 0;
    int f = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&c, p->n_skipped, sizeof(c), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&f, p->err, sizeof(f), cudaMemcpyDeviceToHost);
    if (rounds) *rounds = p->rounds;
    if (skipped_segments) *skipped_segments = (int64_t)c;
    if (error_flags) *error_flags = f;
    return cuda_status(e, "proposal stats");
}

}  // extern "C"
