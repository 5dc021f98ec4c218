// upsample.cu -- coarse-to-fine grid refinement on the device.
//
// upsampleScene / upsample_trilinear (SparseVolumeRadianceField/SceneUtils.cu:262-485): every
// vertex of the finer grid takes the trilinear interpolation of the coarser grid at
// (col * srcW / dstW, row * srcH / dstH, depth * srcD / dstD) -- computed in float as the
// reference does -- with the fractions in double and the sums accumulated in float, corners
// in the reference's order; a density below the threshold becomes 0.  On a sparse source a
// position in an unoccupied cell gives zeros; a sparse target receives only its in-cage
// vertices.  With low_band_only only the first SH coefficient of each channel is
// interpolated and written (the reference's lowBoundOnly).
#include "cpx_internal.cuh"

namespace cpx {

struct UpsampleArgs {
    GridView src;
    float* dst_params;   // dst records (FP32 form)
    float* dst_density;  // dst density mirror
    const uint8_t* __restrict__ dst_in_cage;        // sparse target, else null
    const uint32_t* __restrict__ dst_index_offsets;  // sparse target, else null
    int dW, dH, dD, dst_rec, dst_sh;
    float threshold;
    int low_band;
};

// getIndex of SceneUtils.cu:250-260: coordinates clamped from above only.
__device__ __forceinline__ int up_index(int col, int row, int depth, int W, int H, int D)
{
    col = col < W ? col : W - 1;
    row = row < H ? row : H - 1;
    depth = depth < D ? depth : D - 1;
    return depth * W * H + row * W + col;
}

template <int NSH>
__global__ void __launch_bounds__(128) k_upsample(UpsampleArgs a)
{
    const GridView& s = a.src;
    const int64_t n = (int64_t)a.dW * a.dH * a.dD;
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int col = (int)(p % a.dW), row = (int)((p / a.dW) % a.dH), depth = (int)(p / ((int64_t)a.dW * a.dH));
    int64_t di = p;
    if (a.dst_in_cage) {
        if (!a.dst_in_cage[p]) return;
        di = a.dst_index_offsets[p];
    }
    const float bc[3] = {col * 1.f * s.W / a.dW, row * 1.f * s.H / a.dH, depth * 1.f * s.D / a.dD};
    const unsigned b0 = (unsigned)bc[0], b1 = (unsigned)bc[1], b2 = (unsigned)bc[2];
    constexpr int NA = 1 + 3 * NSH;
    float tri[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) tri[i] = 0.f;
    bool val = true;
    if (s.sparse) {
        const int ci = up_index((int)b0, (int)b1, (int)b2, s.W - 1, s.H - 1, s.D - 1);
        val = (s.occ_bits[ci >> 5] >> (ci & 31)) & 1u;
    }
    if (val) {
        const double x = bc[0] - b0;  // float - unsigned, then widened (SceneUtils.cu:281-283)
        const double y = bc[1] - b1;
        const double z = bc[2] - b2;
        const int nsh = a.low_band ? 1 : NSH;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const unsigned ox = (q >> 1) & 1, oy = q & 1, oz = (q >> 2) & 1;
            int idx = up_index((int)(b0 + ox), (int)(b1 + oy), (int)(b2 + oz), s.W, s.H, s.D);
            if (s.sparse) idx = (int)s.index_offsets[idx];
            double c;
            switch (q) {
            case 0: c = (1. - x) * (1. - y) * (1. - z); break;
            case 1: c = (1. - x) * y * (1. - z); break;
            case 2: c = x * (1. - y) * (1. - z); break;
            case 3: c = x * y * (1. - z); break;
            case 4: c = (1. - x) * (1. - y) * z; break;
            case 5: c = (1. - x) * y * z; break;
            case 6: c = x * (1. - y) * z; break;
            default: c = x * y * z; break;
            }
            const float* rec = s.params + (size_t)idx * s.rec;
            tri[0] += c * rec[0];
#pragma unroll
            for (int i = 0; i < NSH; i++) {
                if (i < nsh) {
                    tri[1 + i] += c * rec[1 + i];
                    tri[1 + NSH + i] += c * rec[1 + NSH + i];
                    tri[1 + 2 * NSH + i] += c * rec[1 + 2 * NSH + i];
                }
            }
        }
    }
    float* out = a.dst_params + (size_t)di * a.dst_rec;
    const float dens = !val || tri[0] < a.threshold ? 0.f : tri[0];
    out[0] = dens;
    a.dst_density[di] = dens;
    const int nw = a.low_band ? 1 : NSH;
#pragma unroll
    for (int i = 0; i < NSH; i++) {
        if (i < nw) {
            out[1 + i] = tri[1 + i];
            out[1 + a.dst_sh + i] = tri[1 + NSH + i];
            out[1 + 2 * a.dst_sh + i] = tri[1 + 2 * NSH + i];
        }
    }
}

}  // namespace cpx

using namespace cpx;

extern "C" cpx_status cpx_grid_upsample(const cpx_grid* src, cpx_grid* dst, float threshold, int low_band_only,
                                        cpx_stream stream)
{
    if (dst) ++dst->epoch;  // new densities: a placement done in advance is stale
    if (!src || !dst) {
        set_error("null grid handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (src->prec != kPrecFP32 || dst->prec != kPrecFP32) {
        set_error("upsampling runs on the FP32 form");
        return CPX_ERR_UNSUPPORTED;
    }
    if (low_band_only ? dst->sh_dim < 1 : dst->sh_dim != src->sh_dim) {
        set_error("target holds %d SH coefficients per channel, the source %d", dst->sh_dim, src->sh_dim);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (src->sparse && !src->have_occupancy) {
        set_error("sparse source without occupancy");
        return CPX_ERR_NOT_READY;
    }
    UpsampleArgs a;
    a.src = grid_view(const_cast<cpx_grid*>(src));
    a.dst_params = dst->params[dst->cur];
    a.dst_density = dst->density;
    a.dst_in_cage = dst->sparse ? dst->in_cage : nullptr;
    a.dst_index_offsets = dst->sparse ? dst->index_offsets : nullptr;
    a.dW = dst->W;
    a.dH = dst->H;
    a.dD = dst->D;
    a.dst_rec = dst->rec;
    a.dst_sh = dst->sh_dim;
    a.threshold = threshold;
    a.low_band = low_band_only ? 1 : 0;
    const int64_t n = dst->n_dense;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    cudaStream_t st = (cudaStream_t)stream;
    switch (src->sh_dim) {
    case 1: k_upsample<1><<<blocks, 128, 0, st>>>(a); break;
    case 4: k_upsample<4><<<blocks, 128, 0, st>>>(a); break;
    case 9: k_upsample<9><<<blocks, 128, 0, st>>>(a); break;
    default:
        set_error("sh_dim %d unsupported", src->sh_dim);
        return CPX_ERR_UNSUPPORTED;
    }
    count_launch();
    cpx_status s = cuda_status(cudaGetLastError(), "upsample");
    if (s != CPX_OK) return s;
    return refresh_dense_mirror(dst, st);
}
