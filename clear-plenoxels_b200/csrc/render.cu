// render.cu -- held-out view render and image error (evaluation path).
//
// renderImageGPU / volumeRender_RGB (SparseVolumeRadianceField/RenderUtils.cu:1720-1810,
// 1443-1580): one thread per pixel sets up its ray in double (getBound,
// RenderUtils.cu:34-97), marches with the training march's placement recurrence, and
// accumulates colour, expected depth and opacity.  Every operation follows the reference's
// types and order (trilinear SH accumulated in float with double weights, the colour dot
// product in float, sigmoid in double), so the image equals the reference's.
#include "cpx_internal.cuh"

namespace cpx {

struct ImageArgs {
    double alpha[2];
    double principle[2];
    double c2w[16];
    double centre[4];
    int bbox[6];
    int width, height, white_bg;
    int it_cap;      // iterations per ray: far - near never exceeds the box diagonal
    int* err;        // sticky error flags of the grid, or null
    float* rgb;      // [3][w*h] or null
    uint8_t* rgb8;   // [3][w*h] or null
    float* depth;    // [w*h] or null
    uint8_t* mask;   // [w*h] or null
};

__device__ __forceinline__ double dmin(double a, double b) { return a > b ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

__device__ __forceinline__ int clampi(int v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); }

template <int NSH, int PREC>
__global__ void __launch_bounds__(128) k_render_image(GridView g, ImageArgs a)
{
    constexpr int NA = 1 + 3 * NSH;
    constexpr int REC = (NA + 3) & ~3;
    const int64_t npix = (int64_t)a.width * a.height;
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= npix) return;
    const int pixelRow = (int)(p / a.width);
    const int pixelCol = (int)(p % a.height);  // the reference's column uses % height (RenderUtils.cu:1727)

    // getBound (RenderUtils.cu:34-97)
    double xInCamera[4] = {
        (pixelCol + 0.5 - a.principle[0]) / a.alpha[0],
        (pixelRow + 0.5 - a.principle[1]) / a.alpha[1],
        1.0,
        1.0,
    };
    double secondPoint[4];
    for (int row = 0; row < 4; row++) {
        secondPoint[row] = 0.;
        for (int col = 0; col < 4; col++) secondPoint[row] += a.c2w[row * 4 + col] * xInCamera[col];
        secondPoint[row] -= a.centre[row];
    }
    double sum = secondPoint[0] * secondPoint[0] + secondPoint[1] * secondPoint[1] + secondPoint[2] * secondPoint[2];
    sum = sqrt(sum);
    secondPoint[0] /= sum;
    secondPoint[1] /= sum;
    secondPoint[2] /= sum;
    double t6[6] = {
        (a.bbox[1] - a.centre[0]) / secondPoint[0], (a.bbox[0] - a.centre[0]) / secondPoint[0],
        (a.bbox[3] - a.centre[1]) / secondPoint[1], (a.bbox[2] - a.centre[1]) / secondPoint[1],
        (a.bbox[5] - a.centre[2]) / secondPoint[2], (a.bbox[4] - a.centre[2]) / secondPoint[2],
    };
    double t_min = dmin(t6[0], t6[1]);
    double t_max = dmax(t6[0], t6[1]);
    t_min = dmax(t_min, dmin(t6[2], t6[3]));
    t_max = dmin(t_max, dmax(t6[2], t6[3]));
    t_min = dmax(t_min, dmin(t6[4], t6[5]));
    t_max = dmin(t_max, dmax(t6[4], t6[5]));
    const double rayInfo[5] = {t_min, t_max, secondPoint[0], secondPoint[1], secondPoint[2]};

    float rgbf[3] = {0.f, 0.f, 0.f};
    float disparity = 0.f;
    uint8_t rgb8[3] = {0, 0, 0};
    uint8_t m = 0;
    if (rayInfo[0] > rayInfo[1]) {  // RenderUtils.cu:1745-1775
        rgb8[0] = rgb8[1] = rgb8[2] = 255;
        if (a.white_bg) rgbf[0] = rgbf[1] = rgbf[2] = 1.f;
    } else {
        // volumeRender_RGB (RenderUtils.cu:1443-1580)
        double t = rayInfo[0];
        double Ti = 1.0;
        double weights, acc = 0.;
        double accumulatedDensity = 0.;
        const float dir[3] = {(float)rayInfo[2], (float)rayInfo[3], (float)rayInfo[4]};
        float shs[9];
        shs[0] = 1.f;
        shs[1] = dir[1];
        shs[2] = dir[2];
        shs[3] = dir[0];
        shs[4] = dir[0] * dir[1];
        shs[5] = dir[1] * dir[2];
        shs[6] = (3.f * dir[2] * dir[2] - 1.f);
        shs[7] = dir[0] * dir[2];
        shs[8] = (dir[0] * dir[0] - dir[1] * dir[1]);
        const float step = g.step;
        // The weights sum to at most 1, so t advances by at least n * step - 1 over n
        // iterations; it_cap bounds that count for any near/far inside the box.
        int it = 0;
        while (t < rayInfo[1]) {
            if (++it > a.it_cap) {
                if (a.err) atomicOr(a.err, 1);
                break;
            }
            double baseCoords[3];
            for (int axisIndex = 0; axisIndex < 3; axisIndex++)
                baseCoords[axisIndex] = a.centre[axisIndex] + t * rayInfo[axisIndex + 2];
            // trilerpRGB_Render (RenderUtils.cu:645-824)
            const unsigned b0 = (unsigned int)baseCoords[0];
            const unsigned b1 = (unsigned int)baseCoords[1];
            const unsigned b2 = (unsigned int)baseCoords[2];
            if (g.sparse) {
                const int ci = clampi((int)b2, g.D - 1) * (g.W - 1) * (g.H - 1) +
                               clampi((int)b1, g.H - 1) * (g.W - 1) + clampi((int)b0, g.W - 1);
                if (!((g.occ_bits[ci >> 5] >> (ci & 31)) & 1u)) {
                    t += step;
                    continue;
                }
            }
            const double x = baseCoords[0] - b0;
            const double y = baseCoords[1] - b1;
            const double z = baseCoords[2] - b2;
            float tri0 = 0.f;
            float sh_tri[3 * NSH];
#pragma unroll
            for (int i = 0; i < 3 * NSH; i++) sh_tri[i] = 0.f;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const unsigned ox = (q >> 1) & 1, oy = q & 1, oz = (q >> 2) & 1;
                int idx = clampi((int)(b2 + oz), g.D) * g.W * g.H + clampi((int)(b1 + oy), g.H) * g.W +
                          clampi((int)(b0 + ox), g.W);
                if (g.sparse) idx = (int)g.index_offsets[idx];
                double contributes;
                switch (q) {
                case 0: contributes = (1. - x) * (1. - y) * (1. - z); break;
                case 1: contributes = (1. - x) * y * (1. - z); break;
                case 2: contributes = x * (1. - y) * (1. - z); break;
                case 3: contributes = x * y * (1. - z); break;
                case 4: contributes = (1. - x) * (1. - y) * z; break;
                case 5: contributes = (1. - x) * y * z; break;
                case 6: contributes = x * (1. - y) * z; break;
                default: contributes = x * y * z; break;
                }
                if (PREC == kPrecFP32) {
                    const float* rec = g.params + (size_t)idx * REC;
                    tri0 += contributes * rec[0];
#pragma unroll
                    for (int i = 0; i < NSH; i++) {
                        if (i < g.n_sh_fwd) {
                            sh_tri[i] += contributes * rec[1 + i];
                            sh_tri[NSH + i] += contributes * rec[1 + NSH + i];
                            sh_tri[2 * NSH + i] += contributes * rec[1 + 2 * NSH + i];
                        }
                    }
                } else {
                    // mixed forms: FP32 density, 16-bit SH record (slot e = parameter e)
                    const uint16_t* rec = sh16_records(g) + (size_t)idx * REC;
                    tri0 += contributes * g.density[idx];
#pragma unroll
                    for (int i = 0; i < NSH; i++) {
                        if (i < g.n_sh_fwd) {
                            sh_tri[i] += contributes * sh_to_f<PREC>(rec[1 + i]);
                            sh_tri[NSH + i] += contributes * sh_to_f<PREC>(rec[1 + NSH + i]);
                            sh_tri[2 * NSH + i] += contributes * sh_to_f<PREC>(rec[1 + 2 * NSH + i]);
                        }
                    }
                }
            }
            float triRes[4];
            triRes[0] = tri0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                triRes[c + 1] = 0.f;
#pragma unroll
                for (int k = 0; k < NSH; k++)
                    if (k < g.n_sh_fwd) triRes[c + 1] += sh_tri[c * NSH + k] * shs[k];
            }
            triRes[0] = logf(1.f + expf(triRes[0] - 13.f));
#pragma unroll
            for (int c = 1; c < 4; c++) triRes[c] = 1.f / (1.f + exp(-0.1 * triRes[c]));
            Ti = exp(-accumulatedDensity);
            weights = Ti * (1. - expf(-triRes[0] * step));
            acc += weights;
            disparity += weights * t;
            rgbf[0] += weights * triRes[1];
            rgbf[1] += weights * triRes[2];
            rgbf[2] += weights * triRes[3];
            accumulatedDensity += triRes[0] * step;
            t += fabs(step - weights);
        }
        for (int c = 0; c < 3; c++) rgb8[c] = (int)((rgbf[c] + 1. - acc) * 255 + 0.5);
        if (a.white_bg)
            for (int c = 0; c < 3; c++) rgbf[c] += 1. - acc;
        m = (uint8_t)(acc * 255);
    }
    if (a.rgb)
        for (int c = 0; c < 3; c++) a.rgb[c * npix + p] = rgbf[c];
    if (a.rgb8)
        for (int c = 0; c < 3; c++) a.rgb8[c * npix + p] = rgb8[c];
    if (a.depth) a.depth[p] = disparity;
    if (a.mask) a.mask[p] = m;
}

// Sum of squared differences in double, one block.
__global__ void k_sq_diff(const float* a, const float* b, int64_t n, double* out)
{
    __shared__ double part[32];
    double s = 0.;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = (double)a[i] - (double)b[i];
        s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) *out = v;
    }
}

}  // namespace cpx

using namespace cpx;

extern "C" cpx_status cpx_render_image(cpx_grid* g, const cpx_camera* cam, int width, int height,
                                       int white_bg, float* rgb_dev, uint8_t* rgb8_dev,
                                       float* depth_dev, uint8_t* mask_dev, cpx_stream stream)
{
    if (!g || !cam || width <= 0 || height <= 0) {
        set_error("invalid image render arguments");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse && !g->have_occupancy) {
        set_error("sparse grid without occupancy");
        return CPX_ERR_NOT_READY;
    }
    ImageArgs a;
    for (int i = 0; i < 2; i++) {
        a.alpha[i] = cam->alpha[i];
        a.principle[i] = cam->principle[i];
    }
    for (int i = 0; i < 16; i++) a.c2w[i] = cam->c2w[i];
    for (int i = 0; i < 4; i++) a.centre[i] = cam->centre[i];
    for (int i = 0; i < 6; i++) a.bbox[i] = g->bbox[i];
    a.width = width;
    a.height = height;
    a.white_bg = white_bg ? 1 : 0;
    a.it_cap = march_samples_per_ray(g);
    a.err = g->scratch.err;
    a.rgb = rgb_dev;
    a.rgb8 = rgb8_dev;
    a.depth = depth_dev;
    a.mask = mask_dev;
    const GridView gv = grid_view(g);
    const int64_t npix = (int64_t)width * height;
    const unsigned blocks = (unsigned)((npix + 127) / 128);
    cudaStream_t st = (cudaStream_t)stream;
    if (g->sh_dim != 1 && g->sh_dim != 4 && g->sh_dim != 9) {
        set_error("sh_dim %d unsupported", g->sh_dim);
        return CPX_ERR_UNSUPPORTED;
    }
#define CPX_IMAGE(PREC)                                                                \
    switch (g->sh_dim) {                                                               \
    case 1: k_render_image<1, PREC><<<blocks, 128, 0, st>>>(gv, a); break;             \
    case 4: k_render_image<4, PREC><<<blocks, 128, 0, st>>>(gv, a); break;             \
    default: k_render_image<9, PREC><<<blocks, 128, 0, st>>>(gv, a); break;            \
    }
    if (g->prec == kPrecFP32) {
        CPX_IMAGE(kPrecFP32)
    } else if (g->prec == kPrecBF16) {
        CPX_IMAGE(kPrecBF16)
    } else {
        CPX_IMAGE(kPrecFP16)
    }
#undef CPX_IMAGE
    count_launch();
    return cuda_status(cudaGetLastError(), "render image");
}

extern "C" cpx_status cpx_image_mse(const float* a_dev, const float* b_dev, int64_t n, double* mse_out,
                                    cpx_stream stream)
{
    if (!a_dev || !b_dev || n <= 0 || !mse_out) {
        set_error("invalid image error arguments");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    double* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(double));
    if (e != cudaSuccess) return cuda_status(e, "image mse");
    cudaStream_t st = (cudaStream_t)stream;
    k_sq_diff<<<1, 1024, 0, st>>>(a_dev, b_dev, n, d);
    count_launch();
    double sum = 0.;
    e = cudaMemcpyAsync(&sum, d, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_status(e, "image mse");
    *mse_out = sum / (double)n;
    return CPX_OK;
}
