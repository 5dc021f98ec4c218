// sweep_lowp.cu -- fused TV (type 0, 6 neighbours) + Adam sweep of the mixed forms.
//
// Same order of operations as the FP32 sweep (TV term added to the gradient, then Adam
// with the reference's bias corrections and density clamp, Optimizer.cu:359-415), over the
// mixed storage: density FP32, SH in 16-bit records, gradients in FP32 records, moments in
// bfloat16 records.  A warp takes 32 consecutive vertices: each lane first works out one
// vertex's own part (touched bit, learning rate, the FP32 density and its TV term), then the
// warp's lanes each update one quad (4 consecutive slots) of those vertices, taking the vertex
// part by shuffle: the quad's SH (8 B), gradients (16 B, touched vertices only), moments
// (2 x 8 B) and its six TV neighbours' SH quads; TV and Adam run in FP32 (packed FP32 pairs
// where every slot takes both), and the new SH and moments go back to 16 bits by the
// hardware's stochastic-rounding conversion, the consumed gradients zeroed.  Per vertex at SH
// band 2: density r+w 8 B, SH r+w 112 B, moments r+w 224 B (+4 B learning-rate multiplier on
// dense grids), gradients r + zero-w 224 B where touched: 348 B (+224 B) against the FP32
// form's 680 B (+224 B).
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
    int full_masks;     // TV and Adam apply to every slot of every quad (no padding, no hierarchy)
    int sparse_adam;    // CPX_OPT_SPARSE_ADAM: untouched vertices are skipped, the rest updated in place
};

// Square root through the hardware reciprocal square root (about 2 ulp; the results are
// stored in 16 bits), 0 for 0.
__device__ __forceinline__ float fast_sqrt(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

// Per-vertex part of the sweep, worked out once by the lane that owns the vertex and handed
// to the lanes of its quads by shuffle: the touched bit, whether the TV term applies, the
// density learning rate, the density itself and its TV term (RenderUtils.cu:2672-2757,
// neighbours in the reference's order z-1, y-1, x-1, x+1, y+1, z+1).
struct LowpVertex {
    float dens;     // FP32 density
    float tv0;      // TV term of the density (0 when it does not apply)
    float lr_d;     // density learning rate (adaptive multiplier included)
    uint32_t bits;  // bit 0: touched; bit 1: TV applies; bits 2..7: neighbour k reads the vertex itself;
                    // bit 8: skipped (sparse Adam, untouched)
};

constexpr uint32_t kSkipBit = 1u << 8;

template <bool TV>
__device__ __forceinline__ LowpVertex lowp_vertex(const LowpArgs& a, uint32_t v, bool tv_on, const uint32_t* nb_v,
                                                  uint32_t self_bits, float lr_d)
{
    LowpVertex r;
    r.tv0 = 0.f;
    r.lr_d = lr_d;
    const bool tch = touched_bit(a.touched, v);
    if (a.sparse_adam && !tch) {  // sparse Adam: a zero gradient leaves the vertex as it is
        r.dens = 0.f;
        r.bits = kSkipBit;
        return r;
    }
    r.dens = __ldg(a.d_in + v);
    r.bits = (tch ? 1u : 0u) | (tv_on ? 2u : 0u) | (self_bits << 2);
    if (TV && tv_on && (a.tv_mask & 1u)) {
        float sum = 0.f, disp = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const float nb = ((self_bits >> k) & 1u) ? r.dens : __ldg(a.d_in + nb_v[k]);
            const float d = r.dens - nb;
            sum += d * d;
            disp = (k == 0) ? d : disp + d;
        }
        const float sd = fast_sqrt(sum) * (1.f / 6.f);
        r.tv0 = __fdividef(a.lam_d * disp, sd + 1.e-6f);
    }
    return r;
}

__device__ __forceinline__ LowpVertex shfl_vertex(const LowpVertex& mine, int from_lane)
{
    LowpVertex r;
    r.dens = __shfl_sync(0xffffffffu, mine.dens, from_lane);
    r.tv0 = __shfl_sync(0xffffffffu, mine.tv0, from_lane);
    r.lr_d = __shfl_sync(0xffffffffu, mine.lr_d, from_lane);
    r.bits = __shfl_sync(0xffffffffu, mine.bits, from_lane);
    return r;
}

// A thread's unit of a record: E = 4 slots (a quad: 8 B of 16-bit values, 16 B of gradients)
// or E = 2 slots (a pair: 4 B and 8 B).
template <int E> struct Unit;
template <> struct Unit<4> {
    using H = uint2;   // E 16-bit values
    using F = float4;  // E floats
    __device__ static void unpack_bf16(const H& w, float* f) { unpack2<kPrecBF16>(w.x, f[0], f[1]); unpack2<kPrecBF16>(w.y, f[2], f[3]); }
    template <int PREC> __device__ static void unpack(const H& w, float* f) { unpack2<PREC>(w.x, f[0], f[1]); unpack2<PREC>(w.y, f[2], f[3]); }
    template <int PREC> __device__ static H pack(const float* f, uint32_t r0, uint32_t r1)
    {
        return make_uint2(sr_pack2<PREC>(f[0], f[1], r0), sr_pack2<PREC>(f[2], f[3], r1));
    }
    __device__ static void floats(const F& g, float* f) { f[0] = g.x; f[1] = g.y; f[2] = g.z; f[3] = g.w; }
    __device__ static F make(const float* f) { return make_float4(f[0], f[1], f[2], f[3]); }
    template <int PREC> __device__ static void unpack_m(const H& w, float* f) { mom1_unpack2<PREC>(w.x, f[0], f[1]); mom1_unpack2<PREC>(w.y, f[2], f[3]); }
    template <int PREC> __device__ static void unpack_v(const H& w, float* f) { mom2_unpack2<PREC>(w.x, f[0], f[1]); mom2_unpack2<PREC>(w.y, f[2], f[3]); }
    template <int PREC> __device__ static H pack_m(const float* f, uint32_t r0, uint32_t r1) { return make_uint2(mom1_pack2<PREC>(f[0], f[1], r0), mom1_pack2<PREC>(f[2], f[3], r1)); }
    template <int PREC> __device__ static H pack_v(const float* f, uint32_t r0, uint32_t r1) { return make_uint2(mom2_pack2<PREC>(f[0], f[1], r0), mom2_pack2<PREC>(f[2], f[3], r1)); }
};
template <> struct Unit<2> {
    using H = uint32_t;
    using F = float2;
    __device__ static void unpack_bf16(const H& w, float* f) { unpack2<kPrecBF16>(w, f[0], f[1]); }
    template <int PREC> __device__ static void unpack(const H& w, float* f) { unpack2<PREC>(w, f[0], f[1]); }
    template <int PREC> __device__ static H pack(const float* f, uint32_t r0, uint32_t) { return sr_pack2<PREC>(f[0], f[1], r0); }
    __device__ static void floats(const F& g, float* f) { f[0] = g.x; f[1] = g.y; }
    __device__ static F make(const float* f) { return make_float2(f[0], f[1]); }
    template <int PREC> __device__ static void unpack_m(const H& w, float* f) { mom1_unpack2<PREC>(w, f[0], f[1]); }
    template <int PREC> __device__ static void unpack_v(const H& w, float* f) { mom2_unpack2<PREC>(w, f[0], f[1]); }
    template <int PREC> __device__ static H pack_m(const float* f, uint32_t r0, uint32_t) { return mom1_pack2<PREC>(f[0], f[1], r0); }
    template <int PREC> __device__ static H pack_v(const float* f, uint32_t r0, uint32_t) { return mom2_pack2<PREC>(f[0], f[1], r0); }
};

// Unit u (record slots E*u .. E*u+E-1) of vertex v, unit index q = v * U + u; nbq: the same
// unit of the six TV neighbours.  Slot 0 is the density: its value, TV term and learning rate
// come from the vertex's LowpVertex, its moments from the unit's moment records.
template <int PREC, int E, bool TV>
__device__ __forceinline__ void lowp_unit(const LowpArgs& a, uint32_t v, uint32_t q, int u, const LowpVertex& vx,
                                          const uint32_t* nbq, float inv_bc1, float inv_bc2, uint32_t step_key)
{
    using UT = Unit<E>;
    using H = typename UT::H;
    using F = typename UT::F;
    const H* sh_in = reinterpret_cast<const H*>(a.sh_in);
    H* sh_out = reinterpret_cast<H*>(a.sh_out);
    H* mrec = reinterpret_cast<H*>(a.m);
    H* vrec = reinterpret_cast<H*>(a.v);
    F* grad = reinterpret_cast<F*>(a.grad);
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1.e-6f;
    // every record a unit reads is written only by the same thread after the read (or not at
    // all), so all of them load through the non-coherent path
    float p[E];
    constexpr int SHP = sh_prec<PREC>();
    UT::template unpack<SHP>(__ldg(sh_in + q), p);
    if (u == 0) p[0] = vx.dens;  // slot 0 of an SH record is unused: density is FP32
    // untouched vertices have zero gradients: their records are neither read nor written
    const bool tch = vx.bits & 1u;
    float g[E];
    if (tch) {
        UT::floats(__ldg(grad + q), g);
    } else {
#pragma unroll
        for (int c = 0; c < E; c++) g[c] = 0.f;
    }
    float mo[E], vo[E];
    UT::template unpack_m<PREC>(__ldg(mrec + q), mo);
    UT::template unpack_v<PREC>(__ldg(vrec + q), vo);
    if (TV && (vx.bits & 2u)) {
        float sum[E], disp[E];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float nb[E];
            if ((vx.bits >> (2 + k)) & 1u) {
#pragma unroll
                for (int c = 0; c < E; c++) nb[c] = p[c];
            } else {
                UT::template unpack<SHP>(__ldg(sh_in + nbq[k]), nb);
            }
#pragma unroll
            for (int c = 0; c < E; c++) {
                const float d = p[c] - nb[c];
                sum[c] = (k == 0) ? d * d : fmaf(d, d, sum[c]);
                disp[c] = (k == 0) ? d : disp[c] + d;
            }
        }
#pragma unroll
        for (int c = 0; c < E; c++) {
            const int e = E * u + c;
            if (e != 0 && ((a.tv_mask >> e) & 1u)) {
                const float sd = fast_sqrt(sum[c]) * (1.f / 6.f);
                g[c] += __fdividef(a.lam_sh * disp[c], sd + 1.e-6f);
            }
        }
    }
    if (u == 0) g[0] += vx.tv0;
    // Adam; elements outside the mask keep their values, which convert back exactly
    float np[E], mn[E], vn[E];
#pragma unroll
    for (int c = 0; c < E; c++) {
        const int e = E * u + c;
        np[c] = p[c];
        mn[c] = mo[c];
        vn[c] = vo[c];
        if (!((a.adam_mask >> e) & 1u)) continue;
        const float gc = g[c];
        mn[c] = fmaf(1.f - beta1, gc, beta1 * mo[c]);
        vn[c] = fmaf((1.f - beta2) * gc, gc, beta2 * vo[c]);
        const float lr = e == 0 ? vx.lr_d : a.sh_lr;
        np[c] = p[c] - __fdividef(lr * (mn[c] * inv_bc1), fast_sqrt(vn[c] * inv_bc2) + eps);
        g[c] = 0.f;
    }
    if (u == 0) {
        const float d = (a.adam_mask & 1u) ? (np[0] < 0.f ? 0.f : np[0]) : p[0];  // density clamp (Optimizer.cu:384)
        a.d_out[v] = d;
        if (a.dense_mirror) a.dense_mirror[a.compact_to_dense[v]] = d;
    }
    // random words: one hash of (launch key, vertex, unit) and one cheap draw; the parameters
    // and the two moments take them in rotated forms
    const uint32_t r0 = fmix32(step_key ^ (v * 0x632BE5ABu) ^ ((uint32_t)u << 27));
    const uint32_t r1 = draw32(r0, 0x85EBCA6Bu);
    sh_out[q] = UT::template pack<SHP>(np, r0, r1);
    mrec[q] = UT::template pack_m<PREC>(mn, __funnelshift_l(r0, r0, 11), __funnelshift_l(r1, r1, 11));
    vrec[q] = UT::template pack_v<PREC>(vn, __funnelshift_l(r0, r0, 22), __funnelshift_l(r1, r1, 22));
    if (tch) grad[q] = UT::make(g);
}

// Hardware approximations (about 1 ulp) of the square root and of the reciprocal of each half
// of a pair, denormal arguments flushed to zero (a TV sum or second moment that small adds
// nothing a 16-bit value can hold); the reciprocal takes arguments of at least 1e-6 here.
__device__ __forceinline__ float2 sqrt2_approx(float2 x)
{
    float2 r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(x.x));
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(x.y));
    return r;
}
__device__ __forceinline__ float2 rcp2_approx(float2 x)
{
    float2 r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(x.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(x.y));
    return r;
}

// The quad update of lowp_unit<PREC, 4, TV> for records whose every slot takes TV and Adam,
// with the element arithmetic in packed FP32 pairs (sm_100 FFMA2 / FMUL2 / FADD2: each pair
// element rounds exactly as the scalar operation) and the square roots and reciprocals from the
// hardware approximations.
// Operand sources of lowp_quad_x2.  From global memory: every record a quad reads is written
// only by the same thread after the read, or not at all, so all of them load through the
// non-coherent path.
struct QuadGlobal {
    const LowpArgs& a;
    uint32_t q;
    const uint32_t* nbq;
    __device__ uint2 self() const { return __ldg(a.sh_in + q); }
    __device__ uint2 nb(int k) const { return __ldg(a.sh_in + nbq[k]); }
    __device__ uint2 m() const { return __ldg(a.m + q); }
    __device__ uint2 v() const { return __ldg(a.v + q); }
    __device__ float4 grad() const { return __ldg(a.grad + q); }
};

// From the lane's own shared-memory slots, filled by its cp.async copies: slot k of 8 bytes at
// s8 + k * stride (SH, m, v, the six neighbours), the gradient quad at g16.
struct QuadStaged {
    uint32_t s8, stride, g16;
    __device__ static uint2 ld8(uint32_t addr)
    {
        uint2 r;
        asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "r"(addr));
        return r;
    }
    __device__ uint2 self() const { return ld8(s8); }
    __device__ uint2 m() const { return ld8(s8 + stride); }
    __device__ uint2 v() const { return ld8(s8 + 2 * stride); }
    __device__ uint2 nb(int k) const { return ld8(s8 + (3 + k) * stride); }
    __device__ float4 grad() const
    {
        float4 r;
        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "r"(g16));
        return r;
    }
};

// NB_SELF: a TV neighbour may be the vertex itself (bits 2..7 of the LowpVertex, the sparse
// grid's missing neighbours); false where no neighbour ever is (the dense grid applies TV to
// interior vertices only), which drops the per-neighbour tests.
// (lo(w) + a.x, hi(w) + a.y) for a word of two 16-bit values: the mixed-precision add converts
// the 16-bit operand exactly and rounds the sum once
template <int PREC>
__device__ __forceinline__ float2 add2_h16(uint32_t w, float2 a)
{
    float2 r;
    if (PREC == kPrecBF16)
        asm("{.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\tadd.rn.f32.bf16 %0, lo, %3;\n\tadd.rn.f32.bf16 %1, hi, %4;}"
            : "=f"(r.x), "=f"(r.y) : "r"(w), "f"(a.x), "f"(a.y));
    else
        asm("{.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\tadd.rn.f32.f16 %0, lo, %3;\n\tadd.rn.f32.f16 %1, hi, %4;}"
            : "=f"(r.x), "=f"(r.y) : "r"(w), "f"(a.x), "f"(a.y));
    return r;
}

template <int PREC, bool TV, class Src, bool NB_SELF = true>
__device__ __forceinline__ void lowp_quad_x2(const LowpArgs& a, uint32_t v, uint32_t q, int u, const LowpVertex& vx,
                                             const Src& src, float inv_bc1, float inv_bc2, uint32_t step_key)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1.e-6f;
    const float2 neg1 = make_float2(-1.f, -1.f);
    constexpr int SHP = sh_prec<PREC>();
    const uint2 sh_raw = src.self();
    float2 p01, p23;
    unpack2<SHP>(sh_raw.x, p01.x, p01.y);
    unpack2<SHP>(sh_raw.y, p23.x, p23.y);
    if (u == 0) p01.x = vx.dens;  // slot 0 of an SH record is unused: density is FP32
    const bool tch = vx.bits & 1u;
    float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tch) g4 = src.grad();
    float2 g01 = make_float2(g4.x, g4.y), g23 = make_float2(g4.z, g4.w);
    const uint2 m_raw = src.m(), v_raw = src.v();
    float2 mo01, mo23, vo01, vo23;
    mom1_unpack2<PREC>(m_raw.x, mo01.x, mo01.y);
    mom1_unpack2<PREC>(m_raw.y, mo23.x, mo23.y);
    mom2_unpack2<PREC>(v_raw.x, vo01.x, vo01.y);
    mom2_unpack2<PREC>(v_raw.y, vo23.x, vo23.y);
    if (TV && (vx.bits & 2u)) {
        float2 s01, s23, d01s, d23s;
        const float2 mp01 = __fmul2_rn(p01, neg1), mp23 = __fmul2_rn(p23, neg1);
#pragma unroll
        for (int k = 0; k < 6; k++) {
            // n - p, exactly the negation of p - n (one rounding either way); a neighbour that is
            // the vertex itself gives +0, as p - p does
            float2 d01 = make_float2(0.f, 0.f), d23 = make_float2(0.f, 0.f);
            if (!NB_SELF || !((vx.bits >> (2 + k)) & 1u)) {
                const uint2 w = src.nb(k);
                d01 = add2_h16<SHP>(w.x, mp01);
                d23 = add2_h16<SHP>(w.y, mp23);
            }
            s01 = k == 0 ? __fmul2_rn(d01, d01) : __ffma2_rn(d01, d01, s01);
            s23 = k == 0 ? __fmul2_rn(d23, d23) : __ffma2_rn(d23, d23, s23);
            d01s = k == 0 ? d01 : __fadd2_rn(d01s, d01);
            d23s = k == 0 ? d23 : __fadd2_rn(d23s, d23);
        }
        // lam * disp / (sqrt(sum) / 6 + 1e-6), the denominator at least 1e-6
        const float2 lam = make_float2(-a.lam_sh, -a.lam_sh);  // the sums hold n - p
        const float2 sixth = make_float2(1.f / 6.f, 1.f / 6.f), tiny = make_float2(1.e-6f, 1.e-6f);
        const float2 e01 = __ffma2_rn(sqrt2_approx(s01), sixth, tiny), e23 = __ffma2_rn(sqrt2_approx(s23), sixth, tiny);
        g01 = __ffma2_rn(__fmul2_rn(lam, d01s), rcp2_approx(e01), g01);
        g23 = __ffma2_rn(__fmul2_rn(lam, d23s), rcp2_approx(e23), g23);
    }
    if (u == 0) g01.x = g4.x + vx.tv0;  // the density's own TV term (slot 0 of the SH pass is void)
    // Adam
    const float2 b1 = make_float2(beta1, beta1), ob1 = make_float2(1.f - beta1, 1.f - beta1);
    const float2 b2 = make_float2(beta2, beta2), ob2 = make_float2(1.f - beta2, 1.f - beta2);
    const float2 bc1 = make_float2(inv_bc1, inv_bc1), bc2 = make_float2(inv_bc2, inv_bc2);
    const float2 mn01 = __ffma2_rn(ob1, g01, __fmul2_rn(b1, mo01));
    const float2 mn23 = __ffma2_rn(ob1, g23, __fmul2_rn(b1, mo23));
    const float2 vn01 = __ffma2_rn(__fmul2_rn(ob2, g01), g01, __fmul2_rn(b2, vo01));
    const float2 vn23 = __ffma2_rn(__fmul2_rn(ob2, g23), g23, __fmul2_rn(b2, vo23));
    const float2 lr01 = make_float2(u == 0 ? vx.lr_d : a.sh_lr, a.sh_lr), lr23 = make_float2(a.sh_lr, a.sh_lr);
    const float2 a01 = __fmul2_rn(lr01, __fmul2_rn(mn01, bc1)), a23 = __fmul2_rn(lr23, __fmul2_rn(mn23, bc1));
    const float2 e2 = make_float2(eps, eps);
    const float2 den01 = __fadd2_rn(sqrt2_approx(__fmul2_rn(vn01, bc2)), e2);
    const float2 den23 = __fadd2_rn(sqrt2_approx(__fmul2_rn(vn23, bc2)), e2);
    const float2 q01 = __fmul2_rn(a01, rcp2_approx(den01)), q23 = __fmul2_rn(a23, rcp2_approx(den23));
    const float2 np01 = __ffma2_rn(q01, neg1, p01), np23 = __ffma2_rn(q23, neg1, p23);  // p - step
    if (u == 0) {
        const float d = np01.x < 0.f ? 0.f : np01.x;  // density clamp (Optimizer.cu:384)
        a.d_out[v] = d;
        if (a.dense_mirror) a.dense_mirror[a.compact_to_dense[v]] = d;
    }
    const uint32_t r0 = fmix32(step_key ^ (v * 0x632BE5ABu) ^ ((uint32_t)u << 27));
    const uint32_t r1 = draw32(r0, 0x85EBCA6Bu);
    a.sh_out[q] = make_uint2(sr_pack2<SHP>(np01.x, np01.y, r0), sr_pack2<SHP>(np23.x, np23.y, r1));
    a.m[q] = make_uint2(mom1_pack2<PREC>(mn01.x, mn01.y, __funnelshift_l(r0, r0, 11)),
                        mom1_pack2<PREC>(mn23.x, mn23.y, __funnelshift_l(r1, r1, 11)));
    a.v[q] = make_uint2(mom2_pack2<PREC>(vn01.x, vn01.y, __funnelshift_l(r0, r0, 22)),
                        mom2_pack2<PREC>(vn23.x, vn23.y, __funnelshift_l(r1, r1, 22)));
    if (tch) a.grad[q] = make_float4(0.f, 0.f, 0.f, 0.f);
}

template <int PREC, int E, bool TV>
__device__ __forceinline__ void lowp_step(const LowpArgs& a, uint32_t v, uint32_t q, int u, const LowpVertex& vx,
                                          const uint32_t* nbq, float inv_bc1, float inv_bc2, uint32_t step_key)
{
    if (E == 4 && a.full_masks)
        lowp_quad_x2<PREC, TV>(a, v, q, u, vx, QuadGlobal{a, q, nbq}, inv_bc1, inv_bc2, step_key);
    else
        lowp_unit<PREC, E, TV>(a, v, q, u, vx, nbq, inv_bc1, inv_bc2, step_key);
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

// Dense grid: one block per (y, z) row; a warp takes 32 consecutive vertices of the row, each
// lane works out one vertex's LowpVertex, and the warp's 32 * U units (consecutive units on
// consecutive lanes, U = 4 S / E per vertex) take it by shuffle.
template <int PREC, int S, bool TV, int E>
__global__ void __launch_bounds__(256, 4) k_sweep_lowp_dense(LowpArgs a)
{
    constexpr int U = 4 * S / E;
    __shared__ float s_bc[2];
    __shared__ uint32_t s_key;
    lowp_bias_corrections(a, s_bc, &s_key);
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x;
    const int y = row % a.H;
    const int z = row / a.H;
    const uint32_t WH = (uint32_t)a.W * a.H;
    const uint32_t v0 = (uint32_t)z * WH + (uint32_t)y * a.W;
    const bool row_interior = y >= 1 && y <= a.H - 2 && z >= 1 && z <= a.D - 2;
    // neighbour units lie a fixed number of units away (unsigned wrap-around; only read where
    // the TV term applies, i.e. inside the grid)
    const uint32_t off[6] = {0u - WH * U, 0u - (uint32_t)a.W * U, 0u - (uint32_t)U, (uint32_t)U,
                             (uint32_t)a.W * U, WH * U};
    for (uint32_t x0 = (threadIdx.x >> 5) * 32u; x0 < (uint32_t)a.W; x0 += blockDim.x) {
        const uint32_t x = x0 + lane;
        const uint32_t v = v0 + x;
        LowpVertex mine;
        mine.dens = mine.tv0 = mine.lr_d = 0.f;
        mine.bits = 0;
        if (x < (uint32_t)a.W) {
            const bool tv_on = row_interior && x >= 1 && x + 2 <= (uint32_t)a.W;
            const uint32_t nb_v[6] = {v - WH, v - (uint32_t)a.W, v - 1u, v + 1u, v + (uint32_t)a.W, v + WH};
            const float lr_d = a.adaptive_lr ? a.lr * a.adaptive_lr[v] : a.lr;
            mine = lowp_vertex<TV>(a, v, tv_on, nb_v, 0u, lr_d);
            if (a.clear && (v & 31u) == 0) a.clear[v >> 5] = 0u;
        }
        const uint32_t nx = min(32u, (uint32_t)a.W - x0);  // vertices of this chunk
#pragma unroll
        for (int it = 0; it < U; it++) {
            const uint32_t i = it * 32u + lane;
            const uint32_t vl = i / U;
            const int u = (int)(i - vl * U);
            const LowpVertex vx = shfl_vertex(mine, (int)vl);
            if (vl >= nx || (vx.bits & kSkipBit)) continue;
            const uint32_t vv = v0 + x0 + vl;
            const uint32_t q = vv * U + u;
            const uint32_t nbq[6] = {q + off[0], q + off[1], q + off[2], q + off[3], q + off[4], q + off[5]};
            lowp_step<PREC, E, TV>(a, vv, q, u, vx, nbq, s_bc[0], s_bc[1], s_key);
        }
    }
}

// Sparse grid: a warp takes 32 consecutive compact vertices; each lane works out one vertex's
// TV neighbourhood and LowpVertex, and the warp's 32 * U units take them by shuffle (as the
// FP32 sparse sweep).
template <int PREC, int S, bool TV, int E>
__global__ void __launch_bounds__(256) k_sweep_lowp_sparse(LowpArgs a)
{
    constexpr int U = 4 * S / E;
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
    LowpVertex mv;
    mv.dens = mv.tv0 = mv.lr_d = 0.f;
    mv.bits = 0;
    if (v0 + lane < a.n_act) {
        if (TV) mine = sparse_tv(v0 + lane, a.compact_to_dense, a.in_cage, a.index_offsets, a.W, a.H, a.D);
        mv = lowp_vertex<TV>(a, v0 + lane, (mine.flags >> 6) & 1u, mine.nb, mine.flags & 63u, a.lr);
        if (a.clear && ((v0 + lane) & 31u) == 0) a.clear[(v0 + lane) >> 5] = 0u;
    }
#pragma unroll
    for (int it = 0; it < U; it++) {
        const uint32_t i = it * 32u + lane;
        const uint32_t vl = i / U;
        const int u = (int)(i - vl * U);
        const SparseTv t = TV ? shfl_tv(mine, (int)vl) : mine;
        const LowpVertex vx = shfl_vertex(mv, (int)vl);
        const uint32_t v = v0 + vl;
        if (v >= a.n_act || (vx.bits & kSkipBit)) continue;
        uint32_t nbq[6];
#pragma unroll
        for (int k = 0; k < 6; k++) nbq[k] = t.nb[k] * U + u;
        lowp_step<PREC, E, TV>(a, v, v * U + u, u, vx, nbq, s_bc[0], s_bc[1], s_key);
    }
}

// Dense grid, every slot under TV and Adam, copies one quad ahead.  The layout of work is that
// of k_sweep_lowp_dense (block per row, warp per 32 vertices, lane per quad); each lane copies
// its next quad's operands -- SH, moments, the gradients of a touched vertex, the six TV
// neighbours' SH -- into its own shared-memory slots with cp.async while it updates the
// current quad from the slots the previous copies filled.  A lane reads only the slots it
// filled itself (after cp.async.wait_group), so no barrier is involved, and the operands in
// flight take no registers.
constexpr int kAsyncThreads = 256;
constexpr int kAsyncSlots = 9;  // 8-byte slots per quad: SH, m, v, six neighbours

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// Waits until at most n of this thread's copy groups are still in flight (n a constant once
// the caller's loop is unrolled).
__device__ __forceinline__ void cp_async_wait(int n)
{
    switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    }
}

// Quads in flight per lane, the one in use included.  Measured at 256^3: 2 stages (4 blocks per
// SM) 1.56 ms, 3 or 4 stages (fewer resident blocks) 1.89 ms.
constexpr int kAsyncStages = 2;
constexpr int kAsyncStageBytes = kAsyncSlots * kAsyncThreads * 8 + kAsyncThreads * 16;
constexpr int kAsyncSmem = kAsyncStages * kAsyncStageBytes;
constexpr int kAsyncBlocks = (226 * 1024) / (kAsyncSmem + 1152) < 4 ? (226 * 1024) / (kAsyncSmem + 1152) : 4;

template <int PREC, int S, bool TV>
__global__ void __launch_bounds__(kAsyncThreads, kAsyncBlocks) k_sweep_lowp_dense_async(LowpArgs a)
{
    constexpr int U = S;  // quads per vertex
    constexpr int NS = kAsyncStages;
    extern __shared__ __align__(16) unsigned char async_smem[];
    __shared__ float s_bc[2];
    __shared__ uint32_t s_key;
    lowp_bias_corrections(a, s_bc, &s_key);
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x;
    const int y = row % a.H;
    const int z = row / a.H;
    const uint32_t WH = (uint32_t)a.W * a.H;
    const uint32_t v0 = (uint32_t)z * WH + (uint32_t)y * a.W;
    const bool row_interior = y >= 1 && y <= a.H - 2 && z >= 1 && z <= a.D - 2;
    const uint32_t off[6] = {0u - WH * U, 0u - (uint32_t)a.W * U, 0u - (uint32_t)U, (uint32_t)U,
                             (uint32_t)a.W * U, WH * U};
    // stage k: 9 slot rows of 8 bytes per thread, then the thread's 16-byte gradient slot
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(async_smem);
    const uint32_t stride = kAsyncThreads * 8;  // bytes between a thread's slots
    const uint32_t slot0 = base + threadIdx.x * 8;
    const uint32_t g0 = base + kAsyncSlots * kAsyncThreads * 8 + threadIdx.x * 16;
    for (uint32_t x0 = (threadIdx.x >> 5) * 32u; x0 < (uint32_t)a.W; x0 += blockDim.x) {
        const uint32_t x = x0 + lane;
        const uint32_t v = v0 + x;
        LowpVertex mine;
        mine.dens = mine.tv0 = mine.lr_d = 0.f;
        mine.bits = 0;
        if (x < (uint32_t)a.W) {
            const bool tv_on = row_interior && x >= 1 && x + 2 <= (uint32_t)a.W;
            const uint32_t nb_v[6] = {v - WH, v - (uint32_t)a.W, v - 1u, v + 1u, v + (uint32_t)a.W, v + WH};
            const float lr_d = a.adaptive_lr ? a.lr * a.adaptive_lr[v] : a.lr;
            mine = lowp_vertex<TV>(a, v, tv_on, nb_v, 0u, lr_d);
            if (a.clear && (v & 31u) == 0) a.clear[v >> 5] = 0u;
        }
        const uint32_t nx = min(32u, (uint32_t)a.W - x0);
        // the copies of quad `it` into stage it % NS (every lane commits a group, empty or not)
        auto issue = [&](int it) {
            const uint32_t i = it * 32u + lane;
            const uint32_t vl = i / U;
            const LowpVertex vx = shfl_vertex(mine, (int)vl);
            if (vl < nx && !(vx.bits & kSkipBit)) {
                const uint32_t q = (v0 + x0 + vl) * U + (i - vl * U);
                const uint32_t d = slot0 + (it % NS) * kAsyncStageBytes;
                cp_async8(d, a.sh_in + q);
                cp_async8(d + stride, a.m + q);
                cp_async8(d + 2 * stride, a.v + q);
                if (vx.bits & 1u) cp_async16(g0 + (it % NS) * kAsyncStageBytes, a.grad + q);
                if (TV && (vx.bits & 2u)) {
#pragma unroll
                    for (int k = 0; k < 6; k++) cp_async8(d + (3 + k) * stride, a.sh_in + (q + off[k]));
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
#pragma unroll
        for (int it = 0; it < NS - 1 && it < U; it++) issue(it);
#pragma unroll
        for (int it = 0; it < U; it++) {
            if (it + NS - 1 < U) issue(it + NS - 1);
            // groups committed after quad it's: min(NS - 1, U - 1 - it)
            cp_async_wait(U - 1 - it < NS - 1 ? U - 1 - it : NS - 1);
            const uint32_t i = it * 32u + lane;
            const uint32_t vl = i / U;
            const int u = (int)(i - vl * U);
            const LowpVertex vx = shfl_vertex(mine, (int)vl);
            if (vl >= nx || (vx.bits & kSkipBit)) continue;
            const uint32_t vv = v0 + x0 + vl;
            const uint32_t q = vv * U + u;
            const QuadStaged src{slot0 + (it % NS) * kAsyncStageBytes, stride, g0 + (it % NS) * kAsyncStageBytes};
            lowp_quad_x2<PREC, TV, QuadStaged, false>(a, vv, q, u, vx, src, s_bc[0], s_bc[1], s_key);
        }
    }
}

// Sparse grid, copies one quad ahead: the work of k_sweep_lowp_sparse (a warp per 32 compact
// vertices, lane per quad, neighbourhoods shared by shuffle) with the operands of each lane's
// next quad -- including its gathered TV neighbours -- copied into its own shared-memory slots
// by cp.async while it updates the current one (as k_sweep_lowp_dense_async).
template <int PREC, int S, bool TV>
__global__ void __launch_bounds__(kAsyncThreads, kAsyncBlocks) k_sweep_lowp_sparse_async(LowpArgs a)
{
    constexpr int U = S;
    constexpr int NS = kAsyncStages;
    extern __shared__ __align__(16) unsigned char async_smem[];
    __shared__ float s_bc[2];
    __shared__ uint32_t s_key;
    lowp_bias_corrections(a, s_bc, &s_key);
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t v0 = warp * 32u;
    if (v0 >= a.n_act) return;  // warp-uniform; no copy is in flight yet
    SparseTv mine;
    mine.flags = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) mine.nb[k] = 0;
    LowpVertex mv;
    mv.dens = mv.tv0 = mv.lr_d = 0.f;
    mv.bits = 0;
    if (v0 + lane < a.n_act) {
        if (TV) mine = sparse_tv(v0 + lane, a.compact_to_dense, a.in_cage, a.index_offsets, a.W, a.H, a.D);
        mv = lowp_vertex<TV>(a, v0 + lane, (mine.flags >> 6) & 1u, mine.nb, mine.flags & 63u, a.lr);
        if (a.clear && ((v0 + lane) & 31u) == 0) a.clear[(v0 + lane) >> 5] = 0u;
    }
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(async_smem);
    const uint32_t stride = kAsyncThreads * 8;
    const uint32_t slot0 = base + threadIdx.x * 8;
    const uint32_t g0 = base + kAsyncSlots * kAsyncThreads * 8 + threadIdx.x * 16;
    auto issue = [&](int it) {
        const uint32_t i = it * 32u + lane;
        const uint32_t vl = i / U;
        const uint32_t u = i - vl * U;
        const SparseTv t = TV ? shfl_tv(mine, (int)vl) : mine;
        const LowpVertex vx = shfl_vertex(mv, (int)vl);
        const uint32_t v = v0 + vl;
        if (v < a.n_act && !(vx.bits & kSkipBit)) {
            const uint32_t q = v * U + u;
            const uint32_t d = slot0 + (it % NS) * kAsyncStageBytes;
            cp_async8(d, a.sh_in + q);
            cp_async8(d + stride, a.m + q);
            cp_async8(d + 2 * stride, a.v + q);
            if (vx.bits & 1u) cp_async16(g0 + (it % NS) * kAsyncStageBytes, a.grad + q);
            if (TV && (vx.bits & 2u)) {
#pragma unroll
                for (int k = 0; k < 6; k++)
                    if (!((vx.bits >> (2 + k)) & 1u)) cp_async8(d + (3 + k) * stride, a.sh_in + (t.nb[k] * U + u));
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
#pragma unroll
    for (int it = 0; it < NS - 1 && it < U; it++) issue(it);
#pragma unroll
    for (int it = 0; it < U; it++) {
        if (it + NS - 1 < U) issue(it + NS - 1);
        cp_async_wait(U - 1 - it < NS - 1 ? U - 1 - it : NS - 1);
        const uint32_t i = it * 32u + lane;
        const uint32_t vl = i / U;
        const int u = (int)(i - vl * U);
        const LowpVertex vx = shfl_vertex(mv, (int)vl);
        const uint32_t v = v0 + vl;
        if (v >= a.n_act || (vx.bits & kSkipBit)) continue;
        const QuadStaged src{slot0 + (it % NS) * kAsyncStageBytes, stride, g0 + (it % NS) * kAsyncStageBytes};
        lowp_quad_x2<PREC, TV>(a, v, v * U + u, u, vx, src, s_bc[0], s_bc[1], s_key);
    }
}

// Once per process, before any graph capture: the async sweep's dynamic shared-memory opt-in.
template <int PREC, int S>
static bool async_opt_in()
{
    return cudaFuncSetAttribute(k_sweep_lowp_dense_async<PREC, S, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kAsyncSmem) == cudaSuccess &&
           cudaFuncSetAttribute(k_sweep_lowp_dense_async<PREC, S, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kAsyncSmem) == cudaSuccess &&
           cudaFuncSetAttribute(k_sweep_lowp_sparse_async<PREC, S, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kAsyncSmem) == cudaSuccess &&
           cudaFuncSetAttribute(k_sweep_lowp_sparse_async<PREC, S, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kAsyncSmem) == cudaSuccess;
}

static int g_async_ready = -1;  // -1: not yet asked; 0: unavailable (the row sweep serves); 1: ready

cpx_status lowp_prepare()
{
    if (g_async_ready >= 0) return CPX_OK;
    const bool ok = async_opt_in<kPrecBF16, 1>() && async_opt_in<kPrecBF16, 4>() && async_opt_in<kPrecBF16, 7>() &&
                    async_opt_in<kPrecFP16, 1>() && async_opt_in<kPrecFP16, 4>() && async_opt_in<kPrecFP16, 7>() &&
                    async_opt_in<kPrecFP16M, 1>() && async_opt_in<kPrecFP16M, 4>() && async_opt_in<kPrecFP16M, 7>();
    if (!ok) cudaGetLastError();
    g_async_ready = ok ? 1 : 0;
    return CPX_OK;
}

// slots a thread updates: quads (pairs measured slower: twice the loads for the same bytes)
constexpr int kLowpUnit = 4;

template <int PREC, int S>
static void launch_lowp(const cpx_grid* g, const LowpArgs& a, bool tv, cudaStream_t st)
{
    if (!g->sparse && a.full_masks && g_async_ready == 1) {
        const unsigned rows = (unsigned)((int64_t)g->H * g->D);
        if (tv)
            k_sweep_lowp_dense_async<PREC, S, true><<<rows, kAsyncThreads, kAsyncSmem, st>>>(a);
        else
            k_sweep_lowp_dense_async<PREC, S, false><<<rows, kAsyncThreads, kAsyncSmem, st>>>(a);
        return;
    }
    if (!g->sparse) {
        const unsigned rows = (unsigned)((int64_t)g->H * g->D);
        if (tv)
            k_sweep_lowp_dense<PREC, S, true, kLowpUnit><<<rows, 256, 0, st>>>(a);
        else
            k_sweep_lowp_dense<PREC, S, false, kLowpUnit><<<rows, 256, 0, st>>>(a);
    } else if (a.full_masks && g_async_ready == 1) {
        const unsigned blocks = (unsigned)(((int64_t)g->n_act + kAsyncThreads - 1) / kAsyncThreads);
        if (tv)
            k_sweep_lowp_sparse_async<PREC, S, true><<<blocks, kAsyncThreads, kAsyncSmem, st>>>(a);
        else
            k_sweep_lowp_sparse_async<PREC, S, false><<<blocks, kAsyncThreads, kAsyncSmem, st>>>(a);
    } else {
        const unsigned blocks = (unsigned)(((int64_t)g->n_act + 255) / 256);  // a warp per 32 vertices
        if (tv)
            k_sweep_lowp_sparse<PREC, S, true, kLowpUnit><<<blocks, 256, 0, st>>>(a);
        else
            k_sweep_lowp_sparse<PREC, S, false, kLowpUnit><<<blocks, 256, 0, st>>>(a);
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
    a.sparse_adam = (g->options & CPX_OPT_SPARSE_ADAM) && !g->all_touched ? 1 : 0;
    if (a.sparse_adam) {  // in place: the skipped vertices' values stay where they are
        a.d_out = g->dens[g->cur];
        a.sh_out = reinterpret_cast<uint2*>(g->sh16[g->cur]);
    }
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
    const uint32_t all = (g->rec >= 32) ? 0xffffffffu : ((1u << g->rec) - 1u);
    a.full_masks = (tv_mask & all) == all && (adam_mask & all) == all ? 1 : 0;
    cpx_status rc = g->prec != kPrecFP16 ? launch_lowp_shape<kPrecBF16>(g, a, fused_tv, st)
                    : g->mom_h           ? launch_lowp_shape<kPrecFP16M>(g, a, fused_tv, st)
                                         : launch_lowp_shape<kPrecFP16>(g, a, fused_tv, st);
    if (rc != CPX_OK) return rc;
    count_launch();
    if (!a.sparse_adam) g->cur ^= 1;
    g->density = g->dens[g->cur];
    g->tcur ^= 1;
    g->all_touched = 0;
    return cuda_status(cudaGetLastError(), "mixed adam sweep");
}

}  // namespace cpx
