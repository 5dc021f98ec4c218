// lowp.cuh -- 16-bit storage of the mixed-precision grid form.
//
// The mixed form keeps density (and the march: positions, transmittance, weights,
// colour accumulation and gradients) in FP32 and stores the SH coefficients and both
// Adam moments as 16-bit values:
//   * BF16: SH and moments in bfloat16;
//   * FP16: SH in half, moments in bfloat16 (a second moment g^2 of 1e-10 is far below
//     half's smallest subnormal, 6e-8; bfloat16 has FP32's exponent range).
// Records of `slots` 16-bit values per vertex (slots = n_arrays rounded up to 4, the FP32
// record's length, so a record is a whole number of 8-byte quads: 56 B at SH band 2 and
// quad j lines up with float4 j of the FP32 gradient record); slot e holds parameter e of
// the reference's order (0 = density, 1..3*sh_dim = R, G, B coefficients), so SH records
// leave slot 0 unused and moment records use it for the density's moments.
//
// Optimizer write-back rounds stochastically: a value lands on either neighbouring
// 16-bit number with probability proportional to closeness, so small Adam steps are not
// lost to round-to-nearest.  The random bits come from a counter-based hash of (seed,
// timestep, vertex, record quad, element): MurmurHash3's 32-bit finaliser (Appleby, public
// domain) applied in a chain, then a multiply-xorshift draw per element whose low 16 bits
// round the parameter and whose high 16 bits round both moments.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

namespace cpx {

constexpr int kPrecFP32 = 0;
constexpr int kPrecBF16 = 1;
constexpr int kPrecFP16 = 2;

inline int lowp_slots(int n_arrays) { return (n_arrays + 3) & ~3; }

__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// bfloat16 bits -> float
__device__ __forceinline__ float bf16_to_f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ float h16_to_f(uint16_t b) { return __half2float(__ushort_as_half(b)); }

template <int PREC>
__device__ __forceinline__ float sh_to_f(uint16_t b)
{
    return PREC == kPrecFP16 ? h16_to_f(b) : bf16_to_f(b);
}

__device__ __forceinline__ uint16_t f_to_bf16_rn(float x)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ uint16_t f_to_h16_rn(float x) { return __half_as_ushort(__float2half_rn(x)); }

template <int PREC>
__device__ __forceinline__ uint16_t f_to_sh_rn(float x)
{
    return PREC == kPrecFP16 ? f_to_h16_rn(x) : f_to_bf16_rn(x);
}

// Cheap 32-bit mixer for words drawn from one hashed counter (multiply, xorshift).
__device__ __forceinline__ uint32_t draw32(uint32_t h, uint32_t k)
{
    uint32_t w = (h ^ (h >> 15)) * k;
    return w ^ (w >> 13);
}

// 4 packed 16-bit values (one quad) <-> floats
template <int PREC>
__device__ __forceinline__ void unpack4(const uint2& q, float* f)
{
    f[0] = sh_to_f<PREC>((uint16_t)(q.x & 0xffffu));
    f[1] = sh_to_f<PREC>((uint16_t)(q.x >> 16));
    f[2] = sh_to_f<PREC>((uint16_t)(q.y & 0xffffu));
    f[3] = sh_to_f<PREC>((uint16_t)(q.y >> 16));
}

// Two floats -> one 32-bit word of two 16-bit values (lo in bits 0..15) with stochastic
// rounding by the sm_100a conversion cvt.rs, which rounds each magnitude up with probability
// equal to the dropped fraction, drawing on the random word rbits.  Values already
// representable convert exactly; NaN stays NaN and overflow goes to infinity.
template <int PREC>
__device__ __forceinline__ uint32_t sr_pack2(float lo, float hi, uint32_t rbits)
{
    uint32_t d;
    if (PREC == kPrecFP16)
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    else
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// One 32-bit word of two 16-bit values -> floats (lo from bits 0..15).
template <int PREC>
__device__ __forceinline__ void unpack2(uint32_t w, float& lo, float& hi)
{
    if (PREC == kPrecFP16) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
        lo = f.x;
        hi = f.y;
    } else {
        lo = __uint_as_float(w << 16);
        hi = __uint_as_float(w & 0xffff0000u);
    }
}

// Stochastic rounding as sr_pack2, saturating: a value beyond the largest finite 16-bit number
// lands on that number instead of infinity.
template <int PREC>
__device__ __forceinline__ uint32_t sr_pack2_sat(float lo, float hi, uint32_t rbits)
{
    uint32_t d;
    if (PREC == kPrecFP16)
        asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    else
        asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// The optimizer sweep's form "FP16 with half moments" (grid precision CPX_PRECISION_FP16_FULL):
// SH in half as the FP16 form, and both Adam moments in half too.  Half spans about 12
// decades (subnormals included) and the second moment v = E[g^2] of gradients between 1e-8
// and 1 spans 16, so v is kept through its root: the records hold m * 2^8 and sqrt(v) * 2^8
// (exact power-of-two scalings), with room for |m| and sqrt(v) from about 2.3e-10 (subnormal)
// and 2.4e-7 (normal) up to 255.9, where the store saturates.  Internal to the sweeps; grids
// carry it as precision FP16 with mom_h set.
constexpr int kPrecFP16M = 3;
constexpr float kMomScale = 256.f;

// The SH storage of a sweep form.
template <int PREC>
__host__ __device__ constexpr int sh_prec()
{
    return PREC == kPrecFP16M ? kPrecFP16 : PREC;
}

__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// One 32-bit word of two first-moment values of sweep form PREC <-> floats.
template <int PREC>
__device__ __forceinline__ void mom1_unpack2(uint32_t w, float& lo, float& hi)
{
    if (PREC == kPrecFP16M) {
        unpack2<kPrecFP16>(w, lo, hi);
        lo *= 1.f / kMomScale;
        hi *= 1.f / kMomScale;
    } else {
        unpack2<kPrecBF16>(w, lo, hi);
    }
}
template <int PREC>
__device__ __forceinline__ uint32_t mom1_pack2(float lo, float hi, uint32_t rbits)
{
    if (PREC == kPrecFP16M) return sr_pack2_sat<kPrecFP16>(lo * kMomScale, hi * kMomScale, rbits);
    return sr_pack2<kPrecBF16>(lo, hi, rbits);
}
// ... and of two second-moment values (stored through their roots in the half form).
template <int PREC>
__device__ __forceinline__ void mom2_unpack2(uint32_t w, float& lo, float& hi)
{
    if (PREC == kPrecFP16M) {
        unpack2<kPrecFP16>(w, lo, hi);
        lo *= 1.f / kMomScale;
        hi *= 1.f / kMomScale;
        lo *= lo;
        hi *= hi;
    } else {
        unpack2<kPrecBF16>(w, lo, hi);
    }
}
template <int PREC>
__device__ __forceinline__ uint32_t mom2_pack2(float lo, float hi, uint32_t rbits)
{
    if (PREC == kPrecFP16M)
        return sr_pack2_sat<kPrecFP16>(sqrt_approx(lo) * kMomScale, sqrt_approx(hi) * kMomScale, rbits);
    return sr_pack2<kPrecBF16>(lo, hi, rbits);
}

__device__ __forceinline__ uint2 pack4(const uint16_t* h)
{
    return make_uint2((uint32_t)h[0] | ((uint32_t)h[1] << 16), (uint32_t)h[2] | ((uint32_t)h[3] << 16));
}

}  // namespace cpx
