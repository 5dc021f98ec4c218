// march.cu -- forward and backward volume march on sm_100a.
//
// The reference marches each ray in one thread and interleaves everything
// (RenderUtils.cu:1582-1718 forward, 2051-2256 backward): at every sample it
// gathers 8 corners x 28 parameters from 28 planar arrays and, backward, issues
// 224 float atomics.  Sample placement is the only part that is inherently
// sequential -- t advances by |step - w| and w depends on the transmittance --
// and it needs only the density.  So the march is split:
//
//  1. place (thread per ray): replays the reference's placement recurrence with
//     the same FP64/FP32 operations in the same order (t, transmittance and
//     weights in double, the trilinear density rounded to float after every
//     corner, softplus and exp in float), reading only the packed density
//     mirror.  Sample positions, counts, weights and accumulated density are
//     therefore the reference's bit for bit.  Each evaluated sample is stored
//     as a 32-byte record.
//  2. shade (warp per ray, lane per sample): gathers the SH records of the
//     samples in parallel (7 aligned 16-byte loads per corner), evaluates the
//     colour, reduces the forward colour over the warp, then runs the backward
//     with warp prefix scans for the running colour/weight sums and scatters the
//     gradients with 16-byte vector atomics (7 per corner instead of 28).
//
// Reference citations: file:line in SparseVolumeRadianceField/.
#include "cpx_internal.cuh"

#include <cstdlib>
#include <mutex>
#include <type_traits>

namespace cpx {

// getSceneIndex (RenderUtils.cu:3-13).
__device__ __forceinline__ int scene_index(int col, int row, int depth, int W, int H, int D)
{
    col = col < 0 ? 0 : (col > W - 1 ? W - 1 : col);
    row = row < 0 ? 0 : (row > H - 1 ? H - 1 : row);
    depth = depth < 0 ? 0 : (depth > D - 1 ? D - 1 : depth);
    return depth * W * H + row * W + col;
}

__device__ __forceinline__ bool cell_occupied(const GridView& g, unsigned b0, unsigned b1,
                                              unsigned b2)
{
    const int ci = scene_index((int)b0, (int)b1, (int)b2, g.W - 1, g.H - 1, g.D - 1);
    return (g.occ_bits[ci >> 5] >> (ci & 31)) & 1u;
}

__device__ __forceinline__ bool dense_cell_open(const uint32_t* __restrict__ cells, const GridView& g, unsigned b0,
                                                unsigned b1, unsigned b2)
{
    const int ci = scene_index((int)b0, (int)b1, (int)b2, g.W - 1, g.H - 1, g.D - 1);
    return (__ldg(cells + (ci >> 5)) >> (ci & 31)) & 1u;
}

__device__ __forceinline__ int clamp_axis(unsigned b, int n)
{
    const int v = (int)b;  // getSceneIndex takes int coordinates (RenderUtils.cu:3-13)
    return v < 0 ? 0 : (v > n - 1 ? n - 1 : v);
}

// The 8 corner vertices of cell (b0,b1,b2) in the reference's order 000,010,100,110,001,011,
// 101,111 (x,y,z), each coordinate clamped to the grid as getSceneIndex does; sparse grids
// map them through index_offsets (RenderUtils.cu:855-990).
__device__ __forceinline__ void cell_corners_dense(const GridView& g, unsigned b0, unsigned b1, unsigned b2,
                                                   unsigned* idx)
{
    const int x0 = clamp_axis(b0, g.W), x1 = clamp_axis(b0 + 1u, g.W);
    const int y0 = clamp_axis(b1, g.H), y1 = clamp_axis(b1 + 1u, g.H);
    const int z0 = clamp_axis(b2, g.D), z1 = clamp_axis(b2 + 1u, g.D);
    const int WH = g.W * g.H;
    const int r00 = z0 * WH + y0 * g.W, r01 = z0 * WH + y1 * g.W;
    const int r10 = z1 * WH + y0 * g.W, r11 = z1 * WH + y1 * g.W;
    idx[0] = (unsigned)(r00 + x0);
    idx[1] = (unsigned)(r01 + x0);
    idx[2] = (unsigned)(r00 + x1);
    idx[3] = (unsigned)(r01 + x1);
    idx[4] = (unsigned)(r10 + x0);
    idx[5] = (unsigned)(r11 + x0);
    idx[6] = (unsigned)(r10 + x1);
    idx[7] = (unsigned)(r11 + x1);
}

__device__ __forceinline__ void cell_corners(const GridView& g, unsigned b0, unsigned b1, unsigned b2,
                                             unsigned* idx)
{
    cell_corners_dense(g, b0, b1, b2, idx);
    if (g.sparse) {
#pragma unroll
        for (int q = 0; q < 8; q++) idx[q] = g.index_offsets[idx[q]];
    }
}

// L1 prefetch of the four 32-byte sectors of a dense-indexed density array (the density of a
// dense grid, or the dense mirror of a sparse one) that hold a cell's 8 corners (corners q and
// q+2 differ only in x and share a sector).
__device__ __forceinline__ void prefetch_cell(const GridView& g, const float* dens, unsigned b0, unsigned b1,
                                              unsigned b2)
{
    unsigned idx[8];
    cell_corners_dense(g, b0, b1, b2, idx);
#pragma unroll
    for (int q = 0; q < 8; q += 2) asm volatile("prefetch.global.L1 [%0];" ::"l"(dens + idx[q]));
}

// Brick occupancy of a sparse grid (8x8x8 cells per bit), read by the FP32 march.
// (struct Skip: cpx_internal.cuh)

// FP32 march on a sparse grid, at an empty cell (b0, b1, b2) with position bc: the number of
// steps that carry the sample position out of that cell -- or out of its whole 8x8x8 brick
// when the brick is empty.  Every position the reference's step-by-step march would visit
// before that point lies in the same empty cell or brick, so jumping by whole steps keeps
// the reference's sample sequence: the samples after the jump sit where step-by-step
// stepping would have put them.
template <typename Real>
__device__ __forceinline__ int empty_steps(const Skip& sk, const Real* bc, unsigned b0, unsigned b1, unsigned b2,
                                           float dx, float dy, float dz, float step)
{
    int kx = (int)(b0 >> 3), ky = (int)(b1 >> 3), kz = (int)(b2 >> 3);
    kx = kx < sk.bx ? kx : sk.bx - 1;
    ky = ky < sk.by ? ky : sk.by - 1;
    kz = kz < sk.bz ? kz : sk.bz - 1;
    const unsigned k = ((unsigned)kz * sk.by + ky) * sk.bx + kx;
    const bool brick_empty = !((__ldg(sk.bits + (k >> 5)) >> (k & 31u)) & 1u);
    const unsigned base[3] = {b0, b1, b2};
    const int kb[3] = {kx, ky, kz};
    const float d[3] = {dx, dy, dz};
    Real exit = (Real)3.0e38f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const Real lo = brick_empty ? (Real)(8 * kb[a]) : (Real)base[a];
        const Real hi = brick_empty ? (Real)(8 * kb[a] + 8) : (Real)(base[a] + 1u);
        if (d[a] > 0.f) {
            const Real e = (hi - bc[a]) / (Real)d[a];
            exit = e < exit ? e : exit;
        } else if (d[a] < 0.f) {
            const Real e = (lo - bc[a]) / (Real)d[a];
            exit = e < exit ? e : exit;
        }
    }
    const Real n = ceil(exit / (Real)step);
    return n < (Real)1 ? 1 : (n > (Real)1.0e6f ? 1000000 : (int)n);
}

// exp in the march's precision.  The FP32 march of the mixed forms (not bound to the reference's
// bits) takes the hardware approximations (__expf, __logf: a few ulp), which shorten its
// per-sample dependent chain; the FP64/FP32 placement of the FP32 form keeps the reference's
// exp / expf / logf.
__device__ __forceinline__ double real_exp(double x) { return exp(x); }
__device__ __forceinline__ float real_exp(float x) { return __expf(x); }
__device__ __forceinline__ float march_expf(double, float x) { return expf(x); }
__device__ __forceinline__ float march_expf(float, float x) { return __expf(x); }
__device__ __forceinline__ float march_logf(double, float x) { return logf(x); }
__device__ __forceinline__ float march_logf(float, float x) { return __logf(x); }

// ---------------------------------------------------------------------------
// Sample placement: one thread per ray.  With Real = double this is the reference's
// recurrence operation for operation (the FP32 form); the mixed forms march in FP32
// (Real = float): the same recurrence with t, transmittance and weights in float.
// ---------------------------------------------------------------------------
// PROP: the proposal-aware march of the mixed forms.  seg_mask holds one bit per segment of
// 32 equal segments of [near, far]: the march jumps over segments whose bit is clear and
// stops after the last set one (all bits set = the full march).  seg_w, when non-null,
// receives the summed sample weights of each segment (the proposal's labels).
//
// The march of one ray is a state (PlaceRay) with three steps -- begin, one iteration of the
// sample loop, end -- so that the same arithmetic runs either as a loop per ray (place_ray)
// or inside the fused march, where a lane that finishes a ray takes the next one without
// waiting for the other lanes of its warp.
template <typename Real>
struct PlaceRay {
    float ox, oy, oz, dx, dy, dz, near_t, far_t;
    Real t, acc, accD, seg_len, inv_seg;
    float accDen;
    int intT, n, it, it_cap, b;
    int64_t ri;
    unsigned cb0, cb1, cb2;
    float cd[8];
    uint32_t seg_mask;
    float* seg_w;
    SampleRec* out;
    // The last sample's record waits here for its transmittance, exp(-accD), which is worked
    // out with the next sample (or at the ray's end): the double exp then overlaps the next
    // sample's trilinear chain instead of stalling the in-order issue on its own.
    SampleRec pend;
};

// renderRaysGPU's set-up of one ray (RenderUtils.cu:1927-1946).  Returns false for a ray with
// no samples (near > far), whose outputs are then complete.
template <typename Real, bool PROP>
__device__ __forceinline__ bool place_begin(PlaceRay<Real>& st, const GridView& g, const RaysView& r, int b,
                                            int64_t ri, SampleRec* samples, int maxs, int* counts,
                                            double* acc_out, bool write_fwd, uint32_t seg_mask, float* seg_w)
{
    // renderRaysGPU zeroes the outputs first (RenderUtils.cu:1927-1941); the backward alone
    // leaves the forward's outputs as they are
    if (write_fwd) {
        r.acc_den[ri] = 0.f;
        r.acc_w[ri] = 0.f;
    }
    st.near_t = r.near_t[ri];
    st.far_t = r.far_t[ri];
    if (st.near_t > st.far_t) {  // RenderUtils.cu:1943-1946: no samples, no background
        counts[b] = -1;
        acc_out[b] = 0.;
        return false;
    }
    st.b = b;
    st.ri = ri;
    st.ox = r.ox[ri];
    st.oy = r.oy[ri];
    st.oz = r.oz[ri];
    st.dx = r.dx[ri];
    st.dy = r.dy[ri];
    st.dz = r.dz[ri];
    // maxs bounds every ray inside the grid box; longer (or non-finite) rays stop there with
    // the error flag set instead of marching on.
    const double bound = floor(((double)st.far_t - (double)st.near_t + 2.0) / (double)g.step) + 4.0;
    // the guided march also spends an iteration on every jump over a skipped segment (two when
    // the jump's end rounds back into the skipped segment)
    st.it_cap = (bound < (double)(maxs + 16) ? (int)bound : maxs + 16) + (PROP ? 2 * kProposalSegments : 0);
    st.out = samples + (size_t)b * maxs;
    st.t = st.near_t;
    st.acc = 0;
    st.accD = 0;
    st.accDen = 0.f;
    st.intT = 0;
    st.n = 0;
    st.it = 0;
    // densities of the last cell visited (consecutive samples mostly share a cell)
    st.cb0 = 0xffffffffu;
    st.cb1 = 0;
    st.cb2 = 0;
    st.seg_mask = seg_mask;
    st.seg_w = seg_w;
    st.seg_len = PROP ? ((Real)st.far_t - (Real)st.near_t) * (Real)(1.0 / kProposalSegments) : (Real)0;
    st.inv_seg = PROP && st.seg_len > (Real)0 ? (Real)1 / st.seg_len : (Real)0;
    return true;
}

// One iteration of the sample loop (RenderUtils.cu:1674-1705), entered with t < far.  Returns
// true when the ray ends here (the loop's breaks).
template <typename Real, bool PROP>
__device__ __forceinline__ bool place_iter(PlaceRay<Real>& st, const GridView& g, int maxs, int* err,
                                           const Skip& sk)
{
    const float step = g.step;
    if (++st.it > st.it_cap || st.n >= maxs) {
        // not an overrun when the last sample already ended the ray (the stop of the FP32 march)
        if (!(st.n > 0 && real_exp(-st.accD) < (Real)sk.t_stop)) atomicOr(err, 1);
        return true;
    }
    Real t = st.t;
    int seg = 0;
    if (PROP) {
        seg = (int)((t - (Real)st.near_t) * st.inv_seg);
        seg = seg < 0 ? 0 : (seg > kProposalSegments - 1 ? kProposalSegments - 1 : seg);
        if (!((st.seg_mask >> seg) & 1u)) {
            if ((st.seg_mask >> seg) == 0u) return true;  // no predicted segment ahead
            Real tn = (Real)st.near_t + (Real)(seg + 1) * st.seg_len;
            st.t = tn > t ? tn : t + (Real)step;
            ++st.intT;
            return false;
        }
    }
    Real ofx = 0, ofy = 0, ofz = 0;
    if (st.intT < g.n_off) {
        ofx = (Real)g.off_x[st.intT];
        ofy = (Real)g.off_y[st.intT];
        ofz = (Real)g.off_z[st.intT];
    }
    // RenderUtils.cu:1676-1678
    const Real bc0 = st.ox + t * st.dx + ofx;
    const Real bc1 = st.oy + t * st.dy + ofy;
    const Real bc2 = st.oz + t * st.dz + ofz;
    const unsigned b0 = (unsigned int)bc0;
    const unsigned b1 = (unsigned int)bc1;
    const unsigned b2 = (unsigned int)bc2;
    // a sparse grid's unoccupied cell (RenderUtils.cu:1681-1686), or -- FP32 march on a
    // dense grid -- a cell whose corner densities are all at or below kEmptyDensity
    const bool empty = g.sparse ? !cell_occupied(g, b0, b1, b2)
                                : (sk.cells != nullptr && !dense_cell_open(sk.cells, g, b0, b1, b2));
    if (empty) {
        if (sizeof(Real) == sizeof(float) && sk.bits) {
            // FP32 march: all the steps through the empty cell (or brick) at once
            const Real bc[3] = {bc0, bc1, bc2};
            const int k = empty_steps<Real>(sk, bc, b0, b1, b2, st.dx, st.dy, st.dz, step);
            st.t = t + (Real)k * (Real)step;
            st.intT += k;
        } else {
            st.t = t + step;
            ++st.intT;
        }
        return false;
    }
    if (b0 != st.cb0 || b1 != st.cb1 || b2 != st.cb2) {
        unsigned idx[8];
        if (g.sparse && sk.dense) {
            // the same values as density[index_offsets[corner]], one load each
            cell_corners_dense(g, b0, b1, b2, idx);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float v = __ldg(sk.dense + idx[q]);
                st.cd[q] = __float_as_uint(v) == kMirrorEmpty ? g.density[0] : v;
            }
        } else {
            cell_corners(g, b0, b1, b2, idx);
#pragma unroll
            for (int q = 0; q < 8; q++) st.cd[q] = g.density[idx[q]];
        }
        st.cb0 = b0;
        st.cb1 = b1;
        st.cb2 = b2;
        // the march waits on every new cell's densities; fetch the cells one and two
        // voxels further along the ray into L1 now, while this sample is evaluated
        if (!g.sparse || sk.dense) {
            const float* src = g.sparse ? sk.dense : g.density;
#pragma unroll
            for (int k = 1; k <= 2; k++) {
                const Real ta = t + (Real)k;
                prefetch_cell(g, src, (unsigned)(st.ox + ta * st.dx), (unsigned)(st.oy + ta * st.dy),
                              (unsigned)(st.oz + ta * st.dz));
            }
        }
    }
    const Real x = bc0 - b0;
    const Real y = bc1 - b1;
    const Real z = bc2 - b2;
    const Real one = 1;
    // trilerpRGB density term (RenderUtils.cu:855-990), corners in the reference's order
    float tri0 = 0.f;
    Real c;
    c = (one - x) * (one - y) * (one - z);
    tri0 += c * st.cd[0];
    c = (one - x) * y * (one - z);
    tri0 += c * st.cd[1];
    c = x * (one - y) * (one - z);
    tri0 += c * st.cd[2];
    c = x * y * (one - z);
    tri0 += c * st.cd[3];
    c = (one - x) * (one - y) * z;
    tri0 += c * st.cd[4];
    c = (one - x) * y * z;
    tri0 += c * st.cd[5];
    c = x * (one - y) * z;
    tri0 += c * st.cd[6];
    c = x * y * z;
    tri0 += c * st.cd[7];
    // the transmittance before this sample, exp(-sum sigma step) of the samples so far (the
    // reference's T, RenderUtils.cu:1693-1704; exactly 1 before the first sample)
    const Real Ti = real_exp(-st.accD);
    if (st.n > 0) {
        st.pend.tn = (float)Ti;  // the previous sample's transmittance after it
        st.out[st.n - 1] = st.pend;
        if (Ti < (Real)sk.t_stop) return true;  // FP32 march: nothing visible remains behind
    }
    // density_activation (RenderUtils.cu:491) and the weight (RenderUtils.cu:1693-1704)
    const float sigma = march_logf(one, 1.f + march_expf(one, tri0 - 13.f));
    const Real w = Ti * (one - march_expf(one, -sigma * step));
    st.acc += w;
    st.accDen += sigma;
    st.accD += sigma * step;
    if (PROP && st.seg_w) st.seg_w[seg] += (float)w;
    SampleRec& rec = st.pend;
    rec.bx = (uint16_t)(b0 < 65535u ? b0 : 65535u);
    rec.by = (uint16_t)(b1 < 65535u ? b1 : 65535u);
    rec.bz = (uint16_t)(b2 < 65535u ? b2 : 65535u);
    rec.pad = 0;
    rec.fx = (float)x;
    rec.fy = (float)y;
    rec.fz = (float)z;
    rec.raw = tri0;
    rec.w = (float)w;
    st.t = t + fabs(step - w);  // fabs(float) is the float overload
    ++st.intT;
    ++st.n;
    return false;
}

template <typename Real>
__device__ __forceinline__ void place_end(PlaceRay<Real>& st, const RaysView& r, int* counts,
                                          double* acc_out, bool write_fwd)
{
    if (st.n > 0) {  // the last sample's record, with its transmittance
        st.pend.tn = (float)real_exp(-st.accD);
        st.out[st.n - 1] = st.pend;
    }
    if (write_fwd) {
        r.acc_den[st.ri] = st.accDen;
        r.acc_w[st.ri] = (float)st.acc;
    }
    acc_out[st.b] = (double)st.acc;
    counts[st.b] = st.n;
}

template <typename Real, bool PROP>
__device__ __forceinline__ void place_ray(const GridView& g, const RaysView& r, int b, int64_t ri,
                                          SampleRec* samples, int maxs, int* counts,
                                          double* acc_out, int* err, bool write_fwd,
                                          uint32_t seg_mask, float* seg_w, const Skip& sk)
{
    PlaceRay<Real> st;
    if (!place_begin<Real, PROP>(st, g, r, b, ri, samples, maxs, counts, acc_out, write_fwd, seg_mask, seg_w))
        return;
    while (st.t < st.far_t) {
        if (place_iter<Real, PROP>(st, g, maxs, err, sk)) break;
    }
    place_end<Real>(st, r, counts, acc_out, write_fwd);
}

// ---------------------------------------------------------------------------
// Stage 2: shading and gradients (warp per ray, lane per sample).
// ---------------------------------------------------------------------------

// The reference's unnormalised SH basis on the float direction (RenderUtils.cu:1646-1656).
template <int NSH>
__device__ __forceinline__ void sh_basis(float dx, float dy, float dz, float* shs)
{
    const float dir[3] = {dx, dy, dz};
    shs[0] = 1.f;
    if (NSH > 1) {
        shs[1] = dir[1];
        shs[2] = dir[2];
        shs[3] = dir[0];
    }
    if (NSH > 4) {
        shs[4] = dir[0] * dir[1];
        shs[5] = dir[1] * dir[2];
        shs[6] = (3.f * dir[2] * dir[2] - 1.f);
        shs[7] = dir[0] * dir[2];
        shs[8] = (dir[0] * dir[0] - dir[1] * dir[1]);
    }
}

// sigmoid / sigmoid_derivative (RenderUtils.cu:480-489), evaluated in double as there.
__device__ __forceinline__ float colour_act(float x) { return 1.f / (1.f + exp(-0.1 * x)); }
__device__ __forceinline__ float colour_deriv_from_act(float s)
{
    return 0.1 * s * (1.f - s);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_inclusive_scan(double v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

struct Corners {
    unsigned idx[8];
    float w[8];
};

__device__ __forceinline__ void sample_corners(const GridView& g, const SampleRec& s, Corners& c)
{
    const float x = s.fx, y = s.fy, z = s.fz;
    const float x0 = 1.f - x, y0 = 1.f - y, z0 = 1.f - z;
    c.w[0] = x0 * y0 * z0;
    c.w[1] = x0 * y * z0;
    c.w[2] = x * y0 * z0;
    c.w[3] = x * y * z0;
    c.w[4] = x0 * y0 * z;
    c.w[5] = x0 * y * z;
    c.w[6] = x * y0 * z;
    c.w[7] = x * y * z;
    cell_corners(g, s.bx, s.by, s.bz, c.idx);
}

template <int NSH>
struct RecShape {
    static constexpr int NA = 1 + 3 * NSH;
    static constexpr int REC = (NA + 3) & ~3;
    static constexpr int NV4 = REC / 4;
};

// Per-warp table of the distinct corner vertices of one 32-sample chunk (about 100 of the
// 256 corner references): key = vertex index.  In the forward the values hold each vertex's
// view-dependent raw colour sum_k SH_ck * basis_k (the basis is constant along a ray, so a
// sample's raw colour is the trilinear blend of its corners' raw colours); in the backward
// they accumulate (density grad, R, G, B colour grads) before the scatter.  Values are four
// separate arrays so neighbouring slots sit in different banks.
constexpr int kHashSlots = 256;
constexpr uint32_t kEmpty = 0xffffffffu;

struct WarpTable {
    uint32_t* keys;  // [n]
    float* va;       // [n] x4
    float* vb0;
    float* vb1;
    float* vb2;
    int n = kHashSlots;       // slots: kHashSlots per sample a lane takes per chunk (a power of 2)
    uint32_t shift = 24;      // 32 - log2(n): the hash's top bits index the table
};

__device__ __forceinline__ int table_slot(const WarpTable& t, uint32_t key)
{
    uint32_t h = (key * 0x9E3779B1u) >> t.shift;
    for (int probe = 0; probe < t.n; probe++) {
        const uint32_t old = atomicCAS(&t.keys[h], kEmpty, key);
        if (old == kEmpty || old == key) return (int)h;
        h = (h + 1) & (uint32_t)(t.n - 1);
    }
    return -1;  // unreachable: a chunk references at most 8 vertices per sample
}

// The slot of a key already in the table (read-only probe).
__device__ __forceinline__ int table_find(const WarpTable& t, uint32_t key)
{
    uint32_t h = (key * 0x9E3779B1u) >> t.shift;
    for (int probe = 0; probe < t.n; probe++) {
        const uint32_t k = t.keys[h];
        if (k == key) return (int)h;
        h = (h + 1) & (uint32_t)(t.n - 1);
    }
    return 0;  // unreachable: every key looked up was inserted
}

__device__ __forceinline__ void table_clear(const WarpTable& t, int lane)
{
    __syncwarp();
    for (int s = lane; s < t.n; s += 32) {
        if (t.keys[s] == kEmpty) continue;
        t.keys[s] = kEmpty;
        t.va[s] = 0.f;
        t.vb0[s] = 0.f;
        t.vb1[s] = 0.f;
        t.vb2[s] = 0.f;
    }
    __syncwarp();
}

// Raw view-dependent colour of every vertex in the table (forward).  PREC selects the SH
// storage: FP32 parameter records, or 16-bit SH records of the mixed forms.
template <int NSH, int PREC>
__device__ __forceinline__ void table_colours(const WarpTable& t, const GridView& g, const float* shs,
                                              int lane)
{
    using RS = RecShape<NSH>;
    __syncwarp();
    for (int s = lane; s < t.n; s += 32) {
        const uint32_t key = t.keys[s];
        if (key == kEmpty) continue;
        float col[3] = {0.f, 0.f, 0.f};
        if (PREC == kPrecFP32) {
            const float4* rec = reinterpret_cast<const float4*>(g.params + (size_t)key * RS::REC);
#pragma unroll
            for (int v = 0; v < RS::NV4; v++) {
                const float4 p = __ldg(rec + v);
                const float pv[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int e = 4 * v + k;
                    if (e >= 1 && e < RS::NA) {
                        const int ch = (e - 1) / NSH;
                        const int kk = (e - 1) % NSH;
                        if (kk < g.n_sh_fwd) col[ch] = fmaf(pv[k], shs[kk], col[ch]);
                    }
                }
            }
        } else {
            // 16-bit record of REC slots: NV4 quads of 8 bytes
            const uint2* rec = reinterpret_cast<const uint2*>(sh16_records(g) + (size_t)key * RS::REC);
#pragma unroll
            for (int v = 0; v < RS::NV4; v++) {
                float pv[4];
                unpack4<PREC>(__ldg(rec + v), pv);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int e = 4 * v + k;
                    if (e >= 1 && e < RS::NA) {
                        const int ch = (e - 1) / NSH;
                        const int kk = (e - 1) % NSH;
                        if (kk < g.n_sh_fwd) col[ch] = fmaf(pv[k], shs[kk], col[ch]);
                    }
                }
            }
        }
        t.vb0[s] = col[0];
        t.vb1[s] = col[1];
        t.vb2[s] = col[2];
    }
    __syncwarp();
}

// Flush the table: one vertex record of gradients per distinct key, 16-byte vector atomics.
template <int NSH>
__device__ __forceinline__ void table_flush(const WarpTable& t, const GridView& g, const float* shs,
                                            uint32_t* touched, int lane)
{
    using RS = RecShape<NSH>;
    __syncwarp();
    for (int s = lane; s < t.n; s += 32) {
        const uint32_t key = t.keys[s];
        if (key == kEmpty) continue;
        const float va = t.va[s];
        const float bch[3] = {t.vb0[s], t.vb1[s], t.vb2[s]};
        float4* dst = reinterpret_cast<float4*>(g.grad + (size_t)key * RS::REC);
#pragma unroll
        for (int q = 0; q < RS::NV4; q++) {
            float e4[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int e = 4 * q + k;
                float val = 0.f;
                if (e == 0) {
                    val = va;
                } else if (e < RS::NA) {
                    const int ch = (e - 1) / NSH;
                    const int kk = (e - 1) % NSH;
                    bool on = true;
                    if (g.hierarchy) on = kk >= g.band * g.band && kk < g.n_sh_fwd;
                    val = on ? bch[ch] * shs[kk] : 0.f;
                }
                e4[k] = val;
            }
            atomicAdd(dst + q, make_float4(e4[0], e4[1], e4[2], e4[3]));
        }
        atomicOr(touched + (key >> 5), 1u << (key & 31u));
        t.keys[s] = kEmpty;
        t.va[s] = 0.f;
        t.vb0[s] = 0.f;
        t.vb1[s] = 0.f;
        t.vb2[s] = 0.f;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Record passes through the copy engine (k_shade / k_shade_dyn).  A lane that gathers a
// 112-byte vertex record with seven 16-byte loads costs the L1 one wavefront per load, and the
// 32 lanes of a warp touch 32 different records, so the record passes dominated the shading's
// L1 traffic.  Here each lane moves a whole record with one bulk copy instead: the forward
// pulls the record into the lane's slot of a per-warp shared-memory stage (cp.async.bulk,
// completing on the warp's mbarrier) and reads it back with conflict-free 16-byte shared loads
// (records 112 B apart: the 8 lanes of a quarter-warp hit 8 distinct 4-bank groups); the flush
// writes the gradient record into the slot and adds it to global memory with one bulk
// reduction (cp.reduce.async.bulk .add.f32, element-wise atomic adds in L2) in place of seven
// vector atomics.  The occupied table slots are listed first, so a pass moves up to 32 records
// and a chunk's ~100 distinct vertices take about four passes.  Addresses and sizes are
// multiples of 16 bytes.
// ---------------------------------------------------------------------------
struct Stage {
    uint32_t smem;   // shared-window address of lane 0's record slot (lane l's at smem + l * record bytes)
    uint32_t mbar;   // the warp's mbarrier (arrival count 1)
    uint32_t phase;  // parity of the mbarrier phase the next pass waits for
    int* err;        // error word: 32 = a record copy did not complete within the wait's limit
    uint8_t* list;   // the warp's list of occupied table slots (tables of at most 256 slots)
    bool ok;
};

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void bulk_reduce_add(float* dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(dst), "r"(src),
                 "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// This thread's bulk reductions have read their shared-memory sources (the slot is free).
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void proxy_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect(uint32_t mbar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
}

// Waits for phase `parity` of the mbarrier, for about a second at most.  Each try suspends the
// thread until the phase completes or for up to the hint (about 0.1 ms), so a wait costs a try
// or two instead of a polling loop.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity)
{
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity), "r"(100000u)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

__device__ __forceinline__ float4 lds128(uint32_t addr)
{
    float4 r;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "r"(addr));
    return r;
}

__device__ __forceinline__ uint2 lds64(uint32_t addr)
{
    uint2 r;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "r"(addr));
    return r;
}

__device__ __forceinline__ void sts128(uint32_t addr, float a, float b, float c, float d)
{
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

// The occupied slots of a table of at most 256 slots, in slot order, into list[0..nd); returns
// nd (every lane).
__device__ __forceinline__ int table_compact(const WarpTable& t, uint8_t* list, int lane)
{
    __syncwarp();
    int nd = 0;
    for (int base = 0; base < t.n; base += 32) {
        const int s = base + lane;
        const bool occ = t.keys[s] != kEmpty;
        const uint32_t m = __ballot_sync(0xffffffffu, occ);
        if (occ) list[nd + __popc(m & ((1u << lane) - 1u))] = (uint8_t)s;
        nd += __popc(m);
    }
    __syncwarp();
    return nd;
}

// The forward record pass of table_colours through the stage: per pass of up to 32 listed
// vertices, lane 0 announces the bytes of the pass's copies, each vertex's lane copies its
// record, the warp waits for the mbarrier's phase and forms the colours from shared memory in
// the same order as table_colours.  FP32 records (112 B at SH band 2) are 16-byte aligned and
// copied as they are; a 16-bit record of the mixed forms (56 B) starts on an 8-byte boundary,
// so the lane copies the 16-byte aligned window around it (64 B; the SH buffers carry 16
// spare bytes for the last record's window) and reads from the record's offset in it.
// Returns false (error word set) when a copy did not complete within the wait's limit; the
// warp then stops shading.
template <int NSH, int PREC>
__device__ __forceinline__ bool table_colours_bulk(const WarpTable& t, const GridView& g, const float* shs, int lane,
                                                   Stage& st)
{
    using RS = RecShape<NSH>;
    constexpr uint32_t kRecBytes = RS::REC * 4;  // the lane's stage slot
    constexpr uint32_t kSrcBytes = PREC == kPrecFP32 ? RS::REC * 4 : RS::REC * 2;
    constexpr uint32_t kCopyBytes = kSrcBytes % 16 == 0 ? kSrcBytes : ((kSrcBytes + 8 + 15) & ~15u);
    static_assert(kCopyBytes <= kRecBytes, "a copy window fits the lane's stage slot");
    const uint32_t mine = st.smem + (uint32_t)lane * kRecBytes;
    bulk_wait_read();  // the slot's last bulk reduction has read it
    proxy_fence_smem();
    const int nd = table_compact(t, st.list, lane);
    for (int p0 = 0; p0 < nd; p0 += 32) {  // passes of up to 32 listed vertices
        const int i = p0 + lane;
        const bool occ = i < nd;
        int s = 0;
        uint32_t key = 0u;
        uint32_t off = 0u;  // the record's offset in its copy window
        if (occ) {
            s = st.list[i];
            key = t.keys[s];
            const char* src = PREC == kPrecFP32
                                  ? reinterpret_cast<const char*>(g.params + (size_t)key * RS::REC)
                                  : reinterpret_cast<const char*>(sh16_records(g) + (size_t)key * RS::REC);
            off = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 15u);
            bulk_load(mine, src - off, kCopyBytes, st.mbar);
        }
        if (lane == 0) mbar_expect(st.mbar, (uint32_t)(nd - p0 < 32 ? nd - p0 : 32) * kCopyBytes);
        const bool done = __all_sync(0xffffffffu, mbar_wait_bounded(st.mbar, st.phase));
        if (!done) {
            if (lane == 0) atomicOr(st.err, 32);
            mbar_wait_bounded(st.mbar, st.phase);  // one more bounded wait for the copies in flight
            st.ok = false;
            return false;
        }
        st.phase ^= 1u;
        if (occ) {
            float col[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int v = 0; v < RS::NV4; v++) {
                float pv[4];
                if (PREC == kPrecFP32) {
                    const float4 p = lds128(mine + 16u * v);
                    pv[0] = p.x;
                    pv[1] = p.y;
                    pv[2] = p.z;
                    pv[3] = p.w;
                } else {
                    unpack4<PREC>(lds64(mine + off + 8u * v), pv);
                }
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int e = 4 * v + k;
                    if (e >= 1 && e < RS::NA) {
                        const int ch = (e - 1) / NSH;
                        const int kk = (e - 1) % NSH;
                        if (kk < g.n_sh_fwd) col[ch] = fmaf(pv[k], shs[kk], col[ch]);
                    }
                }
            }
            t.vb0[s] = col[0];
            t.vb1[s] = col[1];
            t.vb2[s] = col[2];
        }
        __syncwarp();
        proxy_fence_smem();  // the shared reads above before the next pass's copies overwrite the slots
    }
    __syncwarp();
    return true;
}

// The flush of table_flush through the stage: the lane of each listed vertex writes the
// vertex's gradient record into its stage slot and adds it to the grid's gradient record with
// one bulk reduction.
template <int NSH>
__device__ __forceinline__ void table_flush_bulk(const WarpTable& t, const GridView& g, const float* shs,
                                                 uint32_t* touched, int lane, const Stage& st)
{
    using RS = RecShape<NSH>;
    constexpr uint32_t kRecBytes = RS::REC * 4;
    const uint32_t mine = st.smem + (uint32_t)lane * kRecBytes;
    const int nd = table_compact(t, st.list, lane);
    for (int i = lane; i < nd; i += 32) {
        const int s = st.list[i];
        const uint32_t key = t.keys[s];
        const float va = t.va[s];
        const float bch[3] = {t.vb0[s], t.vb1[s], t.vb2[s]};
        bulk_wait_read();  // the slot's previous reduction has read it
#pragma unroll
        for (int q = 0; q < RS::NV4; q++) {
            float e4[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int e = 4 * q + k;
                float val = 0.f;
                if (e == 0) {
                    val = va;
                } else if (e < RS::NA) {
                    const int ch = (e - 1) / NSH;
                    const int kk = (e - 1) % NSH;
                    bool on = true;
                    if (g.hierarchy) on = kk >= g.band * g.band && kk < g.n_sh_fwd;
                    val = on ? bch[ch] * shs[kk] : 0.f;
                }
                e4[k] = val;
            }
            sts128(mine + 16u * q, e4[0], e4[1], e4[2], e4[3]);
        }
        proxy_fence_smem();  // the record's shared stores before the copy engine reads them
        bulk_reduce_add(g.grad + (size_t)key * RS::REC, mine, kRecBytes);
        atomicOr(touched + (key >> 5), 1u << (key & 31u));
        t.keys[s] = kEmpty;
        t.va[s] = 0.f;
        t.vb0[s] = 0.f;
        t.vb1[s] = 0.f;
        t.vb2[s] = 0.f;
    }
    __syncwarp();
}

// Shade one ray with a whole warp: forward colour (lane per sample, warp reduction), then
// the backward of renderRays_withGradients_RGBGPU (RenderUtils.cu:2145-2256) with warp prefix
// scans for the running weight/colour sums and the merged gradient scatter.
// SPL: samples a lane takes per chunk.  A chunk of 32 * SPL consecutive samples shares one
// table (of kHashSlots * SPL slots), so its distinct vertices are gathered and scattered once;
// the scans still run over 32 samples at a time, in sample order.
// BULK: the record passes go through the copy engine (table_colours_bulk, table_flush_bulk),
// staged in *stg.
template <int NSH, int MODE, int PREC, int SPL = 1, bool BULK = false>
__device__ __forceinline__ void shade_ray(const GridView& g, const RaysView& r, int b, int64_t ri,
                                          int cnt, const SampleRec* samples, float4* colours,
                                          int maxs, const double* acc_in, double* losses,
                                          double mask_coef, float huber, const WarpTable& tab,
                                          uint32_t* touched, int lane, Stage* stg = nullptr)
{
    const bool miss = cnt < 0;
    const int n = miss ? 0 : cnt;
    float shs[NSH];
    sh_basis<NSH>(r.dx[ri], r.dy[ri], r.dz[ri], shs);
    const SampleRec* S = samples + (size_t)b * maxs;
    float4* C = colours + (size_t)b * maxs;

    // ---- forward colour ----
    double s0 = 0., s1 = 0., s2 = 0.;
    for (int base = 0; base < n; base += 32 * SPL) {
        SampleRec s;
        Corners cr;
        int slot[8];
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int i = base + 32 * k + lane;
            if (i < n) {
                s = S[i];
                sample_corners(g, s, cr);
#pragma unroll
                for (int q = 0; q < 8; q++) slot[q] = table_slot(tab, cr.idx[q]);
            }
        }
        if constexpr (BULK) {
            if (!table_colours_bulk<NSH, PREC>(tab, g, shs, lane, *stg)) return;
        } else {
            table_colours<NSH, PREC>(tab, g, shs, lane);
        }
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int i = base + 32 * k + lane;
            if (i < n) {
                if (SPL > 1) {  // with more than one sample per lane, the corners are looked up again
                    s = S[i];
                    sample_corners(g, s, cr);
#pragma unroll
                    for (int q = 0; q < 8; q++) slot[q] = table_find(tab, cr.idx[q]);
                }
                float raw[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    raw[0] = fmaf(cr.w[q], tab.vb0[slot[q]], raw[0]);
                    raw[1] = fmaf(cr.w[q], tab.vb1[slot[q]], raw[1]);
                    raw[2] = fmaf(cr.w[q], tab.vb2[slot[q]], raw[2]);
                }
                const float col[3] = {colour_act(raw[0]), colour_act(raw[1]), colour_act(raw[2])};
                C[i] = make_float4(col[0], col[1], col[2], 0.f);
                const double w = (double)s.w;
                s0 += w * col[0];
                s1 += w * col[1];
                s2 += w * col[2];
            }
        }
        table_clear(tab, lane);
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    float pred[3];
    if (MODE & kForward) {
        if (miss) {
            pred[0] = pred[1] = pred[2] = 0.f;
        } else {
            // per-ray values the placement wrote are read from L2 (__ldcg): in the fused march a
            // neighbouring ray's placement on another SM may have written the same cache line
            const double bg = r.white_bg ? 1. - __ldcg(acc_in + b) : 0.;  // RenderUtils.cu:1709-1716
            pred[0] = (float)(s0 + bg);
            pred[1] = (float)(s1 + bg);
            pred[2] = (float)(s2 + bg);
        }
        if (lane == 0) {
            r.acc_r[ri] = pred[0];
            r.acc_g[ri] = pred[1];
            r.acc_b[ri] = pred[2];
        }
    } else {
        pred[0] = r.acc_r[ri];
        pred[1] = r.acc_g[ri];
        pred[2] = r.acc_b[ri];
    }
    if (!(MODE & kBackward)) return;

    // ---- backward ----
    if (miss) {
        if (lane == 0) losses[b] = 0.;
        return;
    }
    double res[3] = {
        pred[0] - r.r[ri] / 255.,
        pred[1] - r.g[ri] / 255.,
        pred[2] - r.b[ri] / 255.,
    };
    const double loss = (fabs(res[0]) + fabs(res[1]) + fabs(res[2])) * 255. / 3.;
    if (isnan(loss)) {
        if (lane == 0) losses[b] = 255.;
        return;
    }
    if (lane == 0) losses[b] = loss;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (res[i] > huber)
            res[i] = huber - 0.5 * huber * huber;
        else if (res[i] < -huber)
            res[i] = 0.5 * huber * huber - huber;
    }
    const float accw_f = __ldcg(r.acc_w + ri);
    float mask_loss = 0.f;
    const uint8_t gm = r.mask[ri];
    if (gm && accw_f < 1.) mask_loss = (gm / 255.0 - accw_f) * mask_coef;
    float wpre = fmax(1e-6, (double)accw_f);
    wpre = fmin(1 - 1e-6, (double)wpre);
    mask_loss += (logf(wpre) - log(1. - wpre)) * 1e-3;
    const float step = g.step;

    double carry_w = 0., carry_c0 = 0., carry_c1 = 0., carry_c2 = 0.;
    for (int base0 = 0; base0 < n; base0 += 32 * SPL) {
        for (int k = 0; k < SPL; k++) {
            const int base = base0 + 32 * k;
            if (base >= n) break;  // warp-uniform
            const int i = base + lane;
            const bool valid = i < n;
            SampleRec s;
            float4 col = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid) {
                s = S[i];
                col = C[i];
            } else {
                s.w = 0.f;
            }
            const double w = valid ? (double)s.w : 0.;
            const double aw = warp_inclusive_scan(w, lane);
            const double a0 = warp_inclusive_scan(w * col.x, lane);
            const double a1 = warp_inclusive_scan(w * col.y, lane);
            const double a2 = warp_inclusive_scan(w * col.z, lane);
            const double acc_i = carry_w + aw;
            const double acc_rgb0 = carry_c0 + a0;
            const double acc_rgb1 = carry_c1 + a1;
            const double acc_rgb2 = carry_c2 + a2;
            carry_w += __shfl_sync(0xffffffffu, aw, 31);
            carry_c0 += __shfl_sync(0xffffffffu, a0, 31);
            carry_c1 += __shfl_sync(0xffffffffu, a1, 31);
            carry_c2 += __shfl_sync(0xffffffffu, a2, 31);
            if (valid) {
                float grad[4];
                grad[1] = 0.6667f * w * res[0] * colour_deriv_from_act(col.x);
                grad[2] = 0.6667f * w * res[1] * colour_deriv_from_act(col.y);
                grad[3] = 0.6667f * w * res[2] * colour_deriv_from_act(col.z);
                const double Ti = (double)s.tn;
                grad[0] = res[0] * (Ti * col.x - (pred[0] - acc_rgb0));
                grad[0] += res[1] * (Ti * col.y - (pred[1] - acc_rgb1));
                grad[0] += res[2] * (Ti * col.z - (pred[2] - acc_rgb2));
                const float dd = 1.f / (1.f + expf(13.f - s.raw));  // density_derivation (RenderUtils.cu:497)
                grad[0] *= 0.6667 * step * dd;
                grad[0] += step * dd * (accw_f - acc_i - Ti) * mask_loss;
                // corner q receives grad[0]*w_q and grad[1+ch]*w_q*basis[k]: merge per vertex first
                Corners cr;
                sample_corners(g, s, cr);
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const float wq = cr.w[q];
                    const int sl = table_slot(tab, cr.idx[q]);
                    atomicAdd(&tab.va[sl], grad[0] * wq);
                    atomicAdd(&tab.vb0[sl], grad[1] * wq);
                    atomicAdd(&tab.vb1[sl], grad[2] * wq);
                    atomicAdd(&tab.vb2[sl], grad[3] * wq);
                }
            }
        }
        if constexpr (BULK)
            table_flush_bulk<NSH>(tab, g, shs, touched, lane, *stg);
        else
            table_flush<NSH>(tab, g, shs, touched, lane);
    }
}

// ---------------------------------------------------------------------------
// The two stages as kernels.  Placement is latency-bound per ray and needs only one thread
// per ray, all resident in one wave; shading is throughput-bound and takes a warp per ray.
// ---------------------------------------------------------------------------
// A placement block is one warp that marches `lanes` rays (lanes 0 .. lanes-1; the others exit
// at once).  Each ray is a dependent chain, and the lanes of a warp run in lock step: with 32
// rays a warp, nearly every iteration takes some lane into a new cell, so every lane pays for
// the cell's corner loads and waits on the slowest of them.  Fewer rays a warp spread the same
// chains over more warps, which the SM's schedulers interleave.
template <int MODE, typename Real, bool PROP>
__global__ void __launch_bounds__(32) k_place(GridView g, RaysView r, const int32_t* sidx, int start,
                                               int len, int64_t n_rays, SampleRec* samples, int maxs,
                                               int* counts, double* acc, int* err, const uint32_t* seg_masks,
                                               float* seg_w, Skip sk, int lanes)
{
    if ((int)threadIdx.x >= lanes) return;
    const int b = blockIdx.x * lanes + threadIdx.x;
    if (b >= len) return;
    const int64_t ri = sidx ? (int64_t)sidx[start + b] : (int64_t)start + b;
    if (ri < 0 || ri >= n_rays) {
        atomicOr(err, 2);
        counts[b] = -2;  // invalid ray index: nothing is read or written for it
        return;
    }
    const uint32_t mask = PROP && seg_masks ? seg_masks[b] : 0xffffffffu;
    float* sw = PROP && seg_w ? seg_w + (size_t)b * kProposalSegments : nullptr;
    place_ray<Real, PROP>(g, r, b, ri, samples, maxs, counts, acc, err, (MODE & kForward) != 0, mask, sw, sk);
}

// Rays a placement warp marches: the fewest (down to a floor, kPlaceLanesFloor or the
// CPX_PLACE_LANES environment variable) that still keep every warp of the batch resident at
// once, since a second wave would add a whole chain's length to the launch.
constexpr int kPlaceLanesFloor = 8;

static int place_lanes(const void* kernel, int len)
{
    struct Entry {
        const void* fn;
        int dev, resident;
    };
    static Entry cache[32];
    static int n_cache = 0;
    static std::mutex mu;
    static int floor_lanes = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    int resident = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (floor_lanes == 0) {
            const char* e = getenv("CPX_PLACE_LANES");
            const int v = e ? atoi(e) : kPlaceLanesFloor;
            floor_lanes = (v == 1 || v == 2 || v == 4 || v == 8 || v == 16 || v == 32) ? v : kPlaceLanesFloor;
        }
        for (int i = 0; i < n_cache; i++)
            if (cache[i].fn == kernel && cache[i].dev == dev) resident = cache[i].resident;
        if (resident == 0) {
            int sms = 0, per = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 32, 0);
            resident = sms * (per > 0 ? per : 1);
            if (n_cache < 32) cache[n_cache++] = Entry{kernel, dev, resident};
        }
    }
    int lanes = 32;
    while (lanes > floor_lanes && (len + lanes / 2 - 1) / (lanes / 2) <= resident) lanes /= 2;
    return lanes;
}

constexpr int kShadeWarps = 4;

static_assert(kHashSlots <= 256, "the stage's slot lists hold 8-bit slot indices");

// The stages of a block's shading warps: a record slot of RecShape<NSH>::REC floats (16-byte
// aligned) per lane, the warp's mbarrier and its list of occupied table slots.
template <int NSH, int W = kShadeWarps>
struct ShadeStage {
    float4 slots[W][32][RecShape<NSH>::NV4];
    unsigned long long mbar[W];
    uint8_t list[W][kHashSlots];
};

template <int NSH, int W = kShadeWarps>
__device__ __forceinline__ Stage stage_init(ShadeStage<NSH, W>& ss, int warp, int lane, int* err)
{
    Stage st;
    st.smem = (uint32_t)__cvta_generic_to_shared(&ss.slots[warp][0][0]);
    st.mbar = (uint32_t)__cvta_generic_to_shared(&ss.mbar[warp]);
    st.phase = 0u;
    st.err = err;
    st.list = ss.list[warp];
    st.ok = true;
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(st.mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    return st;
}

template <int NSH, int MODE, int PREC>
__global__ void __launch_bounds__(kShadeWarps * 32, 5) k_shade(GridView g, RaysView r,
                                                             const int32_t* sidx, int start,
                                                             int len, const SampleRec* samples,
                                                             float4* colours, int maxs,
                                                             const int* counts, const double* acc,
                                                             double* losses, double mask_coef,
                                                             float huber, uint32_t* touched, int* err)
{
    __shared__ uint32_t h_keys[kShadeWarps][kHashSlots];
    __shared__ float h_vals[kShadeWarps][4][kHashSlots];
    __shared__ ShadeStage<NSH> stage;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int s = lane; s < kHashSlots; s += 32) {
        h_keys[warp][s] = kEmpty;
        h_vals[warp][0][s] = h_vals[warp][1][s] = h_vals[warp][2][s] = h_vals[warp][3][s] = 0.f;
    }
    Stage stg = stage_init<NSH>(stage, warp, lane, err);
    const int b = blockIdx.x * kShadeWarps + warp;
    if (b >= len) return;  // warp-uniform
    const int cnt = counts[b];
    if (cnt == -2) {
        if ((MODE & kBackward) && lane == 0) losses[b] = 0.;
        return;
    }
    const int64_t ri = sidx ? (int64_t)sidx[start + b] : (int64_t)start + b;
    const WarpTable tab{h_keys[warp], h_vals[warp][0], h_vals[warp][1], h_vals[warp][2], h_vals[warp][3]};
    shade_ray<NSH, MODE, PREC, 1, true>(g, r, b, ri, cnt, samples, colours, maxs, acc, losses, mask_coef, huber,
                                        tab, touched, lane, &stg);
    bulk_wait_all();  // the bulk reductions are complete before the warp exits
}

// Shading with a work counter: the rays in order of decreasing sample count (k_order_by_count,
// a counting sort on count / 16 in one block), taken a ray per warp from the counter by
// persistent blocks -- the last rays the warps take are the short ones, so no SM waits on one
// long ray at the end of the launch.
constexpr int kOrderBuckets = 256;

__device__ __forceinline__ int order_bucket(int count)
{
    int k = count < 0 ? 0 : count >> 4;
    k = k < kOrderBuckets - 1 ? k : kOrderBuckets - 1;
    return kOrderBuckets - 1 - k;  // longest first
}

__global__ void __launch_bounds__(1024) k_order_by_count(const int* __restrict__ counts, int len, int* order,
                                                         int* ctr)
{
    __shared__ int hist[kOrderBuckets];
    for (int i = threadIdx.x; i < kOrderBuckets; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) *ctr = 0;  // the shading warps' work counter
    __syncthreads();
    for (int b = threadIdx.x; b < len; b += blockDim.x) atomicAdd(&hist[order_bucket(counts[b])], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < kOrderBuckets; k++) {
            const int h = hist[k];
            hist[k] = run;
            run += h;
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < len; b += blockDim.x) order[atomicAdd(&hist[order_bucket(counts[b])], 1)] = b;
}

template <int NSH, int MODE, int PREC>
__global__ void __launch_bounds__(kShadeWarps * 32, 5)
    k_shade_dyn(GridView g, RaysView r, const int32_t* sidx, int start, int len, const SampleRec* samples,
                float4* colours, int maxs, const int* counts, const double* acc, double* losses, double mask_coef,
                float huber, uint32_t* touched, const int* order, int* ctr, int* err)
{
    __shared__ uint32_t h_keys[kShadeWarps][kHashSlots];
    __shared__ float h_vals[kShadeWarps][4][kHashSlots];
    __shared__ ShadeStage<NSH> stage;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int s = lane; s < kHashSlots; s += 32) {
        h_keys[warp][s] = kEmpty;
        h_vals[warp][0][s] = h_vals[warp][1][s] = h_vals[warp][2][s] = h_vals[warp][3][s] = 0.f;
    }
    Stage stg = stage_init<NSH>(stage, warp, lane, err);
    const WarpTable tab{h_keys[warp], h_vals[warp][0], h_vals[warp][1], h_vals[warp][2], h_vals[warp][3]};
    while (true) {
        int k = 0;
        if (lane == 0) k = atomicAdd(ctr, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= len) break;  // warp-uniform
        const int b = order[k];
        const int cnt = counts[b];
        if (cnt == -2) {
            if ((MODE & kBackward) && lane == 0) losses[b] = 0.;
            continue;
        }
        const int64_t ri = sidx ? (int64_t)sidx[start + b] : (int64_t)start + b;
        shade_ray<NSH, MODE, PREC, 1, true>(g, r, b, ri, cnt, samples, colours, maxs, acc, losses, mask_coef, huber,
                                            tab, touched, lane, &stg);
        if (!stg.ok) break;  // a record copy timed out (error word set)
    }
    bulk_wait_all();  // the bulk reductions are complete before the warp exits
}

// ---------------------------------------------------------------------------
// The fused march: placement and shading in one launch, overlapped.  Placement is one
// dependent chain per ray and keeps only a warp or two per SM busy; shading is a warp per ray
// and wants the SM's throughput.  Warp 0 of every block runs placement lanes: a lane takes the
// next ray from a work counter, marches it, publishes it to a ready queue and takes another
// ray at once (the sample loop and the ray loop are one loop, so a lane never waits for the
// other lanes of its warp).  The other warps take ready rays in publication order and shade
// them, so shading runs while the long rays are still being placed.
//
// Progress: placement never waits on anything, and rays are handed out by the counter only
// to lanes that are running, so every ray is published whatever the scheduling of the
// blocks; a shading warp waits only for a slot that some running lane will fill.  The wait
// is still bounded (kSpinLimit polls); a warp that gives up sets error bit 8 and stops.
//
// queue[0]: next ray to place; queue[1]: next free ready slot; queue[2]: next slot to
// shade; queue[4 + s]: 1 + the ray published in slot s (0 = not yet).  Zeroed before every
// launch.  Per-ray values the placement writes (count, weight sum, accumulated weight) are
// read from L2; each ray's sample records start on a 128-byte line (maxs is a multiple of
// 4), so no SM holds a stale line of a ray it has not yet read.
// ---------------------------------------------------------------------------
constexpr int kFusedShadeWarps = 7;
constexpr int kFusedThreads = (1 + kFusedShadeWarps) * 32;
constexpr int kSpinLimit = 1 << 22;  // polls with 128-ns sleeps: well over a second

__device__ __forceinline__ int ld_acquire_gpu(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void publish_ray(int* queue, int b)
{
    __threadfence();  // the ray's samples, count and sums before its ready entry
    const int slot = atomicAdd(queue + 1, 1);
    atomicExch(queue + 4 + slot, b + 1);
}

template <int NSH, int MODE, int PREC, typename Real, bool PROP>
__global__ void __launch_bounds__(kFusedThreads, 2)
    k_march(GridView g, RaysView r, const int32_t* sidx, int start, int len, int64_t n_rays, SampleRec* samples,
            float4* colours, int maxs, int* counts, double* acc, int* err, const uint32_t* seg_masks,
            float* seg_w, Skip sk, double* losses, double mask_coef, float huber, uint32_t* touched, int* queue)
{
    __shared__ uint32_t h_keys[kFusedShadeWarps][kHashSlots];
    __shared__ float h_vals[kFusedShadeWarps][4][kHashSlots];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    constexpr bool kFwd = (MODE & kForward) != 0;
    if (warp == 0) {
        PlaceRay<Real> st;
        bool active = false;
        while (true) {
            if (!active) {
                const int b = atomicAdd(queue, 1);
                if (b >= len) break;
                const int64_t ri = sidx ? (int64_t)sidx[start + b] : (int64_t)start + b;
                if (ri < 0 || ri >= n_rays) {
                    atomicOr(err, 2);
                    counts[b] = -2;  // invalid ray index: nothing is read or written for it
                    publish_ray(queue, b);
                    continue;
                }
                const uint32_t mask = PROP && seg_masks ? seg_masks[b] : 0xffffffffu;
                float* sw = PROP && seg_w ? seg_w + (size_t)b * kProposalSegments : nullptr;
                if (!place_begin<Real, PROP>(st, g, r, b, ri, samples, maxs, counts, acc, kFwd, mask, sw)) {
                    publish_ray(queue, b);
                    continue;
                }
                active = true;
            }
            if (!(st.t < st.far_t) || place_iter<Real, PROP>(st, g, maxs, err, sk)) {
                place_end<Real>(st, r, counts, acc, kFwd);
                publish_ray(queue, st.b);
                active = false;
            }
        }
        return;
    }
    const int sw = warp - 1;
    for (int s = lane; s < kHashSlots; s += 32) {
        h_keys[sw][s] = kEmpty;
        h_vals[sw][0][s] = h_vals[sw][1][s] = h_vals[sw][2][s] = h_vals[sw][3][s] = 0.f;
    }
    __syncwarp();
    const WarpTable tab{h_keys[sw], h_vals[sw][0], h_vals[sw][1], h_vals[sw][2], h_vals[sw][3]};
    while (true) {
        int s = 0;
        if (lane == 0) s = atomicAdd(queue + 2, 1);
        s = __shfl_sync(0xffffffffu, s, 0);
        if (s >= len) break;  // warp-uniform
        int v = 0;
        if (lane == 0) {
            for (int spin = 0;; ++spin) {
                v = ld_acquire_gpu(queue + 4 + s);
                if (v != 0 || spin >= kSpinLimit) break;
                __nanosleep(128);
            }
        }
        v = __shfl_sync(0xffffffffu, v, 0);
        if (v == 0) {
            if (lane == 0) atomicOr(err, 8);
            break;
        }
        v = ld_acquire_gpu(queue + 4 + s);  // every lane acquires the published ray
        const int b = v - 1;
        const int cnt = __ldcg(counts + b);
        if (cnt == -2) {
            if ((MODE & kBackward) && lane == 0) losses[b] = 0.;
            continue;
        }
        const int64_t ri = sidx ? (int64_t)sidx[start + b] : (int64_t)start + b;
        shade_ray<NSH, MODE, PREC>(g, r, b, ri, cnt, samples, colours, maxs, acc, losses, mask_coef, huber, tab,
                                   touched, lane);
    }
}

// ---------------------------------------------------------------------------
// The touched map from the placed samples: a warp per ray, a lane per sample; a sample whose
// cell differs from the previous sample's sets its cell's 8 corner bits (the corners the
// shading will scatter gradients to, found the same way).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mark_touched(GridView g, const SampleRec* samples, const int* counts, int len,
                                                      int maxs, uint32_t* touched)
{
    const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= len) return;  // warp-uniform
    const int cnt = counts[b];
    const SampleRec* S = samples + (size_t)b * maxs;
    unsigned long long prev = ~0ull;  // the cell of the previous sample
    for (int base = 0; base < cnt; base += 32) {
        const int i = base + lane;
        SampleRec s;
        unsigned long long key = ~0ull - 1ull;
        if (i < cnt) {
            s = S[i];
            key = (unsigned long long)s.bx | ((unsigned long long)s.by << 16) | ((unsigned long long)s.bz << 32);
        }
        unsigned long long before = __shfl_up_sync(0xffffffffu, key, 1);
        if (lane == 0) before = prev;
        if (i < cnt && key != before) {
            unsigned idx[8];
            cell_corners(g, s.bx, s.by, s.bz, idx);
#pragma unroll
            for (int q = 0; q < 8; q++) atomicOr(touched + (idx[q] >> 5), 1u << (idx[q] & 31u));
        }
        prev = __shfl_sync(0xffffffffu, key, 31);
    }
}

cpx_status mark_touched(cpx_grid* g, int len, cudaStream_t st)
{
    if (len <= 0) return CPX_OK;
    const GridView gv = grid_view(g);
    k_mark_touched<<<(unsigned)((len + 7) / 8), 256, 0, st>>>(gv, g->scratch.samples, g->scratch.counts, len,
                                                             g->scratch.maxs, g->touched[g->tcur]);
    count_launch();
    return cuda_status(cudaGetLastError(), "touched map");
}

// ---------------------------------------------------------------------------
// Batch MSE of the per-ray losses (getMSEError, Utils.cu:311-320), one block.
// ---------------------------------------------------------------------------
__global__ void k_mse(const double* losses, int len, double* out)
{
    __shared__ double part[32];
    double s = 0.;
    for (int i = threadIdx.x; i < len; i += blockDim.x) s += losses[i] * losses[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.;
        v = warp_sum(v);
        if (threadIdx.x == 0) *out = len > 0 ? v / len : 0.;
    }
}

cpx_status mse_launch(const double* losses, int len, double* out, cudaStream_t s)
{
    k_mse<<<1, 1024, 0, s>>>(losses, len, out);
    count_launch();
    return cuda_status(cudaGetLastError(), "mse");
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
static int max_samples_per_ray(const cpx_grid* g)
{
    const double ex = (double)g->bbox[1] - g->bbox[0];
    const double ey = (double)g->bbox[3] - g->bbox[2];
    const double ez = (double)g->bbox[5] - g->bbox[4];
    const double diag = sqrt(ex * ex + ey * ey + ez * ez);
    // a multiple of 4, so every ray's sample records start on a 128-byte line (the fused march)
    return (((int)ceil((diag + 2.0) / g->step) + 8) + 3) & ~3;
}

// The grid's march scratch `which` (0: the march's own; 1: the look-ahead step's second one,
// which shares the error flags and the MSE word of the first) with room for len rays.
static cpx_status ensure_scratch(cpx_grid* g, int len, int which = 0)
{
    const int maxs = max_samples_per_ray(g);
    MarchScratch& s0 = g->scratch;
    if (s0.err == nullptr) {
        if (cudaMalloc((void**)&s0.err, sizeof(int) * 4) != cudaSuccess ||
            cudaMalloc((void**)&s0.mse, sizeof(double)) != cudaSuccess) {
            set_error("scratch allocation failed");
            return CPX_ERR_OUT_OF_MEMORY;
        }
        cudaMemset(s0.err, 0, sizeof(int) * 4);
    }
    MarchScratch& s = which ? g->scratch2 : g->scratch;
    s.err = s0.err;
    s.mse = s0.mse;
    if (s.cap_rays >= len && s.maxs == maxs) return CPX_OK;
    cudaFree(s.samples);
    cudaFree(s.colours);
    cudaFree(s.counts);
    cudaFree(s.acc);
    cudaFree(s.queue);
    s.samples = nullptr;
    s.colours = nullptr;
    s.counts = nullptr;
    s.acc = nullptr;
    s.queue = nullptr;
    s.cap_rays = 0;
    const int cap = len > 0 ? len : 1;
    const size_t ns = (size_t)cap * maxs;
    if (cudaMalloc((void**)&s.samples, ns * sizeof(SampleRec)) != cudaSuccess ||
        cudaMalloc((void**)&s.colours, ns * sizeof(float4)) != cudaSuccess ||
        cudaMalloc((void**)&s.counts, (size_t)cap * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&s.acc, (size_t)cap * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&s.queue, ((size_t)cap + 4) * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        set_error("march scratch of %zu samples could not be allocated", ns);
        return CPX_ERR_OUT_OF_MEMORY;
    }
    s.cap_rays = cap;
    s.maxs = maxs;
    return CPX_OK;
}

// Proposal inputs of a march: per-ray segment masks and/or segment-weight output.
struct Guide {
    const uint32_t* masks = nullptr;
    float* seg_w = nullptr;
    Skip skip;
    bool march32 = false;  // the FP32 march of the mixed forms (else the reference's sequence)
    bool two_stage = true;  // placement and shading as two launches (else the fused march, CPX_OPT_FUSED_MARCH)
    int stages = 3;         // bit 0: placement, bit 1: shading (a look-ahead step runs them apart)
    bool on() const { return masks != nullptr || seg_w != nullptr; }
};

// Blocks of the fused march: what the GPU holds at once, at most one block per 32 rays.
template <int NSH, int MODE, int PREC, typename Real, bool PROP>
static int fused_blocks(int len)
{
    static int resident = 0;  // per kernel instance
    if (resident == 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_march<NSH, MODE, PREC, Real, PROP>, kFusedThreads, 0);
        resident = sms * (per > 0 ? per : 1);
    }
    const int want = (len + 31) / 32;
    return want < resident ? want : resident;
}

template <int MODE, int NSH, int PREC, typename Real, bool PROP>
static void launch_fused(cudaStream_t st, const GridView& gv, const RaysView& rv, const int32_t* sidx, int start,
                         int len, int64_t n_rays, const MarchScratch& s, double* losses, double mask_coef,
                         float huber, uint32_t* touched, const Guide& guide)
{
    cudaMemsetAsync(s.queue, 0, ((size_t)len + 4) * sizeof(int), st);
    k_march<NSH, MODE, PREC, Real, PROP><<<fused_blocks<NSH, MODE, PREC, Real, PROP>(len), kFusedThreads, 0, st>>>(
        gv, rv, sidx, start, len, n_rays, s.samples, s.colours, s.maxs, s.counts, s.acc, s.err,
        PROP ? guide.masks : nullptr, PROP ? guide.seg_w : nullptr, guide.skip, losses, mask_coef, huber, touched,
        s.queue);
}

template <int MODE, int NSH, int PREC>
static void launch_mode(cudaStream_t st, const GridView& gv, const RaysView& rv, const int32_t* sidx,
                        int start, int len, int64_t n_rays, const MarchScratch& s, double* losses,
                        double mask_coef, float huber, uint32_t* touched, const Guide& guide)
{
    if (!guide.two_stage) {
        if (guide.march32 && guide.on())
            launch_fused<MODE, NSH, PREC, float, true>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef,
                                                       huber, touched, guide);
        else if (guide.march32)
            launch_fused<MODE, NSH, PREC, float, false>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef,
                                                        huber, touched, guide);
        else
            launch_fused<MODE, NSH, PREC, double, false>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef,
                                                         huber, touched, guide);
        return;
    }
    const dim3 sgrid((unsigned)((len + kShadeWarps - 1) / kShadeWarps));
    const dim3 sblock(kShadeWarps * 32);
    if (!(guide.stages & 1)) {
        // placement already done (a look-ahead step placed this batch under the last sweep)
    } else if (guide.march32 && guide.on()) {
        const int lanes = place_lanes((const void*)k_place<MODE, float, true>, len);
        k_place<MODE, float, true><<<(len + lanes - 1) / lanes, 32, 0, st>>>(
            gv, rv, sidx, start, len, n_rays, s.samples, s.maxs, s.counts, s.acc, s.err, guide.masks, guide.seg_w,
            guide.skip, lanes);
    } else if (guide.march32) {
        const int lanes = place_lanes((const void*)k_place<MODE, float, false>, len);
        k_place<MODE, float, false><<<(len + lanes - 1) / lanes, 32, 0, st>>>(
            gv, rv, sidx, start, len, n_rays, s.samples, s.maxs, s.counts, s.acc, s.err, nullptr, nullptr, guide.skip,
            lanes);
    } else {
        const int lanes = place_lanes((const void*)k_place<MODE, double, false>, len);
        k_place<MODE, double, false><<<(len + lanes - 1) / lanes, 32, 0, st>>>(
            gv, rv, sidx, start, len, n_rays, s.samples, s.maxs, s.counts, s.acc, s.err, nullptr, nullptr, guide.skip,
            lanes);
    }
    if (!(guide.stages & 2)) return;
    if (s.queue) {
        // longest rays first from a work counter (the queue's first word and its ray slots)
        static int resident = 0;  // per instance
        if (resident == 0) {
            int dev = 0, sms = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_shade_dyn<NSH, MODE, PREC>, kShadeWarps * 32, 0);
            resident = sms * (per > 0 ? per : 1);
        }
        const int blocks = (int)sgrid.x < resident ? (int)sgrid.x : resident;
        k_order_by_count<<<1, 1024, 0, st>>>(s.counts, len, s.queue + 4, s.queue);
        count_launch();
        k_shade_dyn<NSH, MODE, PREC><<<blocks, sblock, 0, st>>>(gv, rv, sidx, start, len, s.samples, s.colours,
                                                                 s.maxs, s.counts, s.acc, losses, mask_coef, huber,
                                                                 touched, s.queue + 4, s.queue, s.err);
        return;
    }
    k_shade<NSH, MODE, PREC><<<sgrid, sblock, 0, st>>>(gv, rv, sidx, start, len, s.samples, s.colours, s.maxs,
                                                       s.counts, s.acc, losses, mask_coef, huber, touched, s.err);
}

template <int NSH, int PREC>
static void launch_march(int mode, cudaStream_t st, const GridView& gv, const RaysView& rv,
                         const int32_t* sidx, int start, int len, int64_t n_rays,
                         const MarchScratch& s, double* losses, double mask_coef, float huber,
                         uint32_t* touched, const Guide& guide)
{
    if (mode == kForward)
        launch_mode<kForward, NSH, PREC>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef, huber,
                                         touched, guide);
    else if (mode == kBackward)
        launch_mode<kBackward, NSH, PREC>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef, huber,
                                          touched, guide);
    else
        launch_mode<kForwardBackward, NSH, PREC>(st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef,
                                                 huber, touched, guide);
}

template <int PREC>
static cpx_status launch_prec(int sh_dim, int mode, cudaStream_t st, const GridView& gv, const RaysView& rv,
                              const int32_t* sidx, int start, int len, int64_t n_rays, const MarchScratch& s,
                              double* losses, double mask_coef, float huber, uint32_t* touched, const Guide& guide)
{
    switch (sh_dim) {
    case 1: launch_march<1, PREC>(mode, st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef, huber, touched, guide); break;
    case 4: launch_march<4, PREC>(mode, st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef, huber, touched, guide); break;
    case 9: launch_march<9, PREC>(mode, st, gv, rv, sidx, start, len, n_rays, s, losses, mask_coef, huber, touched, guide); break;
    default:
        set_error("sh_dim %d unsupported", sh_dim);
        return CPX_ERR_UNSUPPORTED;
    }
    return CPX_OK;
}

static cpx_status march_check_args(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start,
                                   int len, int mode, double* losses)
{
    if (len < 0 || start < 0) {
        set_error("negative start/len");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!sidx && (int64_t)start + len > r->n) {
        set_error("batch [%d, %d) exceeds the %lld rays", start, start + len, (long long)r->n);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if ((mode & kBackward) && !losses && len > 0) {
        set_error("losses buffer is required for the backward");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse && !g->have_occupancy) {
        set_error("sparse grid without occupancy");
        return CPX_ERR_NOT_READY;
    }
    return CPX_OK;
}

int march_samples_per_ray(const cpx_grid* g) { return max_samples_per_ray(g); }

static cpx_status march_launch_guided_with(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                                           int mode, double* losses, double mask_coef, float huber,
                                           const MarchScratch& s, const Guide& guide, cudaStream_t st);

cpx_status march_launch_with(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                             int mode, double* losses, double mask_coef, float huber,
                             const MarchScratch& s, cudaStream_t st)
{
    return march_launch_guided_with(g, r, sidx, start, len, mode, losses, mask_coef, huber, s, Guide(), st);
}

static cpx_status march_launch_guided_with(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                                           int mode, double* losses, double mask_coef, float huber,
                                           const MarchScratch& s, const Guide& guide, cudaStream_t st)
{
    cpx_status rc = march_check_args(g, r, sidx, start, len, mode, losses);
    if (rc != CPX_OK || len == 0) return rc;
    Guide gd = guide;
    gd.march32 = g->prec != kPrecFP32 || (g->options & CPX_OPT_FP32_MARCH);
    gd.two_stage = !(g->options & CPX_OPT_FUSED_MARCH) || s.queue == nullptr || guide.stages != 3;
    if (guide.on() && !gd.march32) {
        set_error("the proposal-guided march runs on the FP32 march of the mixed forms only");
        return CPX_ERR_UNSUPPORTED;
    }
    if (g->sparse) gd.skip.dense = g->dense_mirror;
    // the FP32 march jumps over empty cells and bricks of a sparse grid
    if (gd.march32 && !(g->options & CPX_OPT_NO_EARLY_STOP)) gd.skip.t_stop = kStopTransmittance;
    if (dense_skip_on(g) && g->dense_cells) {
        gd.skip.cells = g->dense_cells;
        gd.skip.bits = g->dense_bricks;
        gd.skip.bx = (g->W - 1 + 7) / 8;
        gd.skip.by = (g->H - 1 + 7) / 8;
        gd.skip.bz = (g->D - 1 + 7) / 8;
    }
    if (gd.march32 && !(g->options & CPX_OPT_NO_EMPTY_SKIP) && g->sparse && g->brick_bits) {
        gd.skip.bits = g->brick_bits;
        gd.skip.bx = g->bricks[0];
        gd.skip.by = g->bricks[1];
        gd.skip.bz = g->bricks[2];
    }
    const GridView gv = grid_view(g);
    const RaysView rv = rays_view(r);
    uint32_t* touched = g->touched[g->tcur];
    if (g->prec == kPrecFP32)
        rc = launch_prec<kPrecFP32>(g->sh_dim, mode, st, gv, rv, sidx, start, len, r->n, s, losses, mask_coef, huber,
                                    touched, gd);
    else if (g->prec == kPrecBF16)
        rc = launch_prec<kPrecBF16>(g->sh_dim, mode, st, gv, rv, sidx, start, len, r->n, s, losses, mask_coef, huber,
                                    touched, gd);
    else
        rc = launch_prec<kPrecFP16>(g->sh_dim, mode, st, gv, rv, sidx, start, len, r->n, s, losses, mask_coef, huber,
                                    touched, gd);
    if (rc != CPX_OK) return rc;
    count_launch((gd.stages & 1) + ((gd.stages >> 1) & 1));
    return cuda_status(cudaGetLastError(), "march");
}

cpx_status march_launch_stages(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len, double* losses,
                               double mask_coef, float huber, int which, int stages, cudaStream_t st)
{
    cpx_status rc = march_check_args(g, r, sidx, start, len, kForwardBackward, losses);
    if (rc != CPX_OK) return rc;
    if (len == 0) return CPX_OK;
    rc = ensure_scratch(g, len, which);
    if (rc != CPX_OK) return rc;
    Guide guide;
    guide.stages = stages;
    return march_launch_guided_with(g, r, sidx, start, len, kForwardBackward, losses, mask_coef, huber,
                                    which ? g->scratch2 : g->scratch, guide, st);
}

cpx_status march_launch(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                        int mode, double* losses, double mask_coef, float huber,
                        cudaStream_t st)
{
    cpx_status rc = march_check_args(g, r, sidx, start, len, mode, losses);
    if (rc != CPX_OK) return rc;
    g->last_len = len;
    if (len == 0) return CPX_OK;
    rc = ensure_scratch(g, len);
    if (rc != CPX_OK) return rc;
    return march_launch_with(g, r, sidx, start, len, mode, losses, mask_coef, huber, g->scratch, st);
}

cpx_status march_launch_guided(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                               double* losses, double mask_coef, float huber, const uint32_t* masks,
                               float* seg_w, cudaStream_t st, int mode)
{
    cpx_status rc = march_check_args(g, r, sidx, start, len, mode, losses);
    if (rc != CPX_OK) return rc;
    g->last_len = len;
    if (len == 0) return CPX_OK;
    rc = ensure_scratch(g, len);
    if (rc != CPX_OK) return rc;
    if (seg_w) {
        cudaError_t e = cudaMemsetAsync(seg_w, 0, (size_t)len * kProposalSegments * sizeof(float), st);
        if (e != cudaSuccess) return cuda_status(e, "segment weights");
    }
    Guide guide;
    guide.masks = masks;
    guide.seg_w = seg_w;
    return march_launch_guided_with(g, r, sidx, start, len, mode, losses, mask_coef, huber, g->scratch, guide, st);
}

// ---------------------------------------------------------------------------
// Batched form: the batches of many scenes (grids of any size, any batch length) in one
// placement launch and one shading launch.  Both kernels are persistent: a warp takes the
// next rays from a global work counter, so scenes with long rays and scenes with short ones
// share the GPU without one launch per scene.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int batch_scene_of(const int* s_base, int n, int gray)
{
    int lo = 0, hi = n - 1;  // the last scene whose first ray is <= gray
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_base[mid] <= gray) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename Real>
__global__ void k_place_batched(BatchArgs a)
{
    __shared__ int s_base[kMaxBatchScenes];
    for (int i = threadIdx.x; i < a.n_scenes; i += blockDim.x) s_base[i] = a.scenes[i].ray_base;
    __syncthreads();
    const int iter = *a.iter;
    const int lane = threadIdx.x & 31;
    while (true) {
        int first = 0;
        if (lane == 0) first = atomicAdd(a.queue, 32);
        first = __shfl_sync(0xffffffffu, first, 0);
        if (first >= a.total_rays) break;  // warp-uniform
        const int gr = first + lane;
        if (gr >= a.total_rays) continue;
        const int si = batch_scene_of(s_base, a.n_scenes, gr);
        const BatchScene& sc = a.scenes[si];
        const int b = gr - sc.ray_base;
        const int64_t ri = (int64_t)(iter % sc.pool_batches) * sc.len + b;
        place_ray<Real, false>(sc.g, sc.r, b, ri, a.samples + sc.sample_base, sc.maxs, a.counts + sc.ray_base,
                               a.acc + sc.ray_base, a.err, true, 0xffffffffu, nullptr, sc.skip);
    }
}

// SPL: samples a lane takes per chunk (the autotuner's samples-per-step), tables of
// kHashSlots * SPL slots per warp.
template <int NSH, int PREC, int WARPS, int SPL>
__global__ void __launch_bounds__(WARPS * 32, 20 / WARPS) k_shade_batched(BatchArgs a)
{
    constexpr int kSlots = kHashSlots * SPL;
    // the bulk record passes where the stage fits beside the tables (one sample per lane, up to
    // four warps: the autotuner's usual shapes); the other shapes keep per-lane loads and atomics
    constexpr bool kBulk = SPL == 1 && WARPS <= 4;
    using StageMem = ShadeStage<NSH, kBulk ? WARPS : 1>;
    static_assert(WARPS * SPL * kHashSlots * 5 * 4 + sizeof(StageMem) + kMaxBatchScenes * 4 <= 48 * 1024,
                  "static shared memory of the tables and the stage");
    __shared__ uint32_t h_keys[WARPS][kSlots];
    __shared__ float h_vals[WARPS][4][kSlots];
    __shared__ StageMem stage;
    __shared__ int s_base[kMaxBatchScenes];
    for (int i = threadIdx.x; i < a.n_scenes; i += blockDim.x) s_base[i] = a.scenes[i].ray_base;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int s = lane; s < kSlots; s += 32) {
        h_keys[warp][s] = kEmpty;
        h_vals[warp][0][s] = h_vals[warp][1][s] = h_vals[warp][2][s] = h_vals[warp][3][s] = 0.f;
    }
    Stage stg;
    stg.ok = true;
    if constexpr (kBulk) stg = stage_init<NSH, WARPS>(stage, warp, lane, a.err);
    __syncthreads();
    WarpTable tab{h_keys[warp], h_vals[warp][0], h_vals[warp][1], h_vals[warp][2], h_vals[warp][3]};
    tab.n = kSlots;
    tab.shift = SPL == 1 ? 24u : (SPL == 2 ? 23u : 22u);
    const int iter = *a.iter;
    while (true) {
        int first = 0;
        if (lane == 0) first = atomicAdd(a.queue + 1, a.grab);
        first = __shfl_sync(0xffffffffu, first, 0);
        if (first >= a.total_rays) break;  // warp-uniform
        for (int q = 0; q < a.grab; q++) {
            const int gr = first + q;
            if (gr >= a.total_rays) break;
            const int si = batch_scene_of(s_base, a.n_scenes, gr);
            const BatchScene& sc = a.scenes[si];
            const int b = gr - sc.ray_base;
            const int cnt = a.counts[gr];
            if (cnt == -2) {
                if (lane == 0) a.losses[gr] = 0.;
                continue;
            }
            const int64_t ri = (int64_t)(iter % sc.pool_batches) * sc.len + b;
            shade_ray<NSH, kForwardBackward, PREC, SPL, kBulk>(sc.g, sc.r, b, ri, cnt, a.samples + sc.sample_base,
                                                          a.colours + sc.sample_base, sc.maxs, a.acc + sc.ray_base,
                                                          a.losses + sc.ray_base, a.mask_coef, a.huber, tab,
                                                          sc.touched, lane, kBulk ? &stg : nullptr);
            if (!stg.ok) break;  // a record copy timed out (error word set)
        }
        if (!stg.ok) break;
    }
    if constexpr (kBulk) bulk_wait_all();  // the bulk reductions are complete before the warp exits
}

static int batch_blocks(const void* fn, int threads, int smem)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
    return sms * (per > 0 ? per : 1);
}

template <int PREC>
static cpx_status batch_launch_prec(const BatchArgs& a, const BatchTuning& tn, cudaStream_t st)
{
    using Real = typename std::conditional<PREC == kPrecFP32, double, float>::type;
    const int pb = batch_blocks((const void*)k_place_batched<Real>, tn.place_block, 0);
    k_place_batched<Real><<<pb, tn.place_block, 0, st>>>(a);
#define CPX_SHADE_B(W, SPL)                                                                         \
    {                                                                                               \
        const int sb = batch_blocks((const void*)k_shade_batched<9, PREC, W, SPL>, W * 32, 0);      \
        k_shade_batched<9, PREC, W, SPL><<<sb, W * 32, 0, st>>>(a);                                 \
    }
    // shading warps per block x samples per lane: the combinations whose tables fit in a block
    if (tn.shade_warps == 2 && tn.spl == 4) CPX_SHADE_B(2, 4)
    else if (tn.shade_warps == 2 && tn.spl == 2) CPX_SHADE_B(2, 2)
    else if (tn.shade_warps == 2) CPX_SHADE_B(2, 1)
    else if (tn.shade_warps == 4 && tn.spl == 2) CPX_SHADE_B(4, 2)
    else if (tn.shade_warps == 8) CPX_SHADE_B(8, 1)
    else CPX_SHADE_B(4, 1)
#undef CPX_SHADE_B
    count_launch(2);
    return cuda_status(cudaGetLastError(), "batched march");
}

cpx_status batch_launch_march(int prec, const BatchArgs& a, const BatchTuning& tn, cudaStream_t st)
{
    if (prec == kPrecFP32) return batch_launch_prec<kPrecFP32>(a, tn, st);
    if (prec == kPrecBF16) return batch_launch_prec<kPrecBF16>(a, tn, st);
    return batch_launch_prec<kPrecFP16>(a, tn, st);
}

BatchScene batch_scene_view(cpx_grid* g, cpx_rays* r, int len, int pool_batches, int ray_base, int64_t sample_base)
{
    BatchScene sc;
    sc.g = grid_view(g);
    sc.r = rays_view(r);
    sc.skip = Skip();
    if (g->sparse) sc.skip.dense = g->dense_mirror;
    const bool march32 = g->prec != kPrecFP32 || (g->options & CPX_OPT_FP32_MARCH);
    if (march32 && !(g->options & CPX_OPT_NO_EARLY_STOP)) sc.skip.t_stop = kStopTransmittance;
    if (dense_skip_on(g) && g->dense_cells) {
        sc.skip.cells = g->dense_cells;
        sc.skip.bits = g->dense_bricks;
        sc.skip.bx = (g->W - 1 + 7) / 8;
        sc.skip.by = (g->H - 1 + 7) / 8;
        sc.skip.bz = (g->D - 1 + 7) / 8;
    }
    if (march32 && !(g->options & CPX_OPT_NO_EMPTY_SKIP) && g->sparse && g->brick_bits) {
        sc.skip.bits = g->brick_bits;
        sc.skip.bx = g->bricks[0];
        sc.skip.by = g->bricks[1];
        sc.skip.bz = g->bricks[2];
    }
    sc.touched = g->touched[g->tcur];
    sc.len = len;
    sc.pool_batches = pool_batches;
    sc.maxs = max_samples_per_ray(g);
    sc.ray_base = ray_base;
    sc.n_rays = r->n;
    sc.sample_base = sample_base;
    return sc;
}

}  // namespace cpx
