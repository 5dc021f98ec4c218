// carve.cu -- silhouette carving and the bounding-box search of a dense grid.
//
// RenderUtils::bbox_silhouette (SVRF/RenderUtils.cu:323-478) runs silhouetteCarving
// (RenderUtils.cu:181-254) once per training camera, then getMaxRadius (:288-321) and
// getBoundingBoxZ (:256-286) with a host reduction.  Here carving is a thread per vertex
// (the reference walks a column per thread): the vertex's point (x + 0.5, y + 0.5, z) goes
// through the camera's 3x4 world-to-pixel matrix in double, as the reference's
// projectWorld2Image (:120-132) computes it, and when no pixel within `radius` of the
// truncated image position has a nonzero mask or colour byte, the vertex's density and
// density-LR multiplier become 0.  The box search is a thread per (x, y) column with the
// reduction in device atomics: the same bounds, independent of order.
#include <cstring>

#include "cpx_internal.cuh"

namespace cpx {

struct CarveArgs {
    double P[12];
    int W, H, D, img_w, img_h, radius;
    const uint8_t* __restrict__ red;
    const uint8_t* __restrict__ green;
    const uint8_t* __restrict__ blue;
    const uint8_t* __restrict__ mask;  // may be null (all zero)
    float* params;   // FP32 form: parameter records (slot 0 = density), else null
    int rec;
    float* density;  // the density array the march reads (FP32 mirror or the mixed form's)
    float* adaptive_lr;
};

__global__ void k_carve(CarveArgs a)
{
    const int64_t n = (int64_t)a.W * a.H * a.D;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int col = (int)(v % a.W), row = (int)((v / a.W) % a.H), depth = (int)(v / ((int64_t)a.W * a.H));
        const double world[4] = {col + 0.5, row + 0.5, (double)depth, 1.};
        double image[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            image[r] = 0.;
#pragma unroll
            for (int c = 0; c < 4; c++) image[r] += a.P[r * 4 + c] * world[c];
        }
        image[0] /= image[2];
        image[1] /= image[2];
        const int imageRow = (int)image[1];
        const int imageCol = (int)image[0];
        bool save = false;
        for (int nr = -a.radius; nr < a.radius + 1 && !save; nr++) {
            const double pr = imageRow + nr;
            for (int nc = -a.radius; nc < a.radius + 1; nc++) {
                const double pc = imageCol + nc;
                if (pc < 0 || pc >= a.img_w || pr < 0 || pr >= a.img_h) continue;
                const int p = (int)(pr * a.img_w + pc);
                if ((a.mask && a.mask[p]) || a.red[p] || a.green[p] || a.blue[p]) {
                    save = true;
                    break;
                }
            }
        }
        if (!save) {
            if (a.params) a.params[(size_t)v * a.rec] = 0.f;
            a.density[v] = 0.f;
            a.adaptive_lr[v] = 0.f;
        }
    }
}

// [0..5]: x min/max, y min/max, z min/max (ints); [6..7]: the largest radius (double bits)
struct BoxAcc {
    int b[6];
    unsigned long long max_radius;
};

__global__ void k_box_columns(const float* __restrict__ lr, int W, int H, int D, int want_radius, BoxAcc* acc)
{
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= (int64_t)W * H) return;
    const int row = (int)(p / W), col = (int)(p % W);
    const int64_t WH = (int64_t)W * H;
    // getBoundingBoxZ (RenderUtils.cu:256-286)
    int depth = 0;
    while (lr[depth * WH + p] < 1e-6 && depth + 1 < D) ++depth;
    int rmin = depth, rmax = depth;
    while (depth + 1 < D) {
        ++depth;
        if (lr[depth * WH + p] > 1e-6) rmax = depth;
    }
    if (rmin != depth) {
        atomicMin(&acc->b[0], col);
        atomicMax(&acc->b[1], col);
        atomicMin(&acc->b[2], row);
        atomicMax(&acc->b[3], row);
        atomicMin(&acc->b[4], rmin);
        atomicMax(&acc->b[5], rmax);
    }
    if (want_radius) {
        // getMaxRadius (RenderUtils.cu:288-321)
        double best = 0.;
        const double temp = (row - H / 2.) * (row - H / 2.) + (col - W / 2.) * (col - W / 2.);
        for (int d = 0; d < D; d++) {
            if (lr[d * WH + p] > 1e-6) {
                const double distance = sqrt(temp + (d - D / 2.) * (d - D / 2.));
                if (distance > best) best = distance;
            }
        }
        // non-negative doubles order as their bit patterns
        atomicMax(&acc->max_radius, (unsigned long long)__double_as_longlong(best));
    }
}

}  // namespace cpx

using namespace cpx;

extern "C" cpx_status cpx_carve_silhouette(cpx_grid* g, const double* projection, int img_w, int img_h,
                                           const uint8_t* red, const uint8_t* green, const uint8_t* blue,
                                           const uint8_t* mask, int radius, cpx_stream stream)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (!g || !projection || !red || !green || !blue || img_w < 1 || img_h < 1 || radius < 0) {
        set_error("carving needs a grid, a projection, three colour planes and a radius >= 0");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse) {
        set_error("carving runs on the dense grid (before sparsification)");
        return CPX_ERR_UNSUPPORTED;
    }
    const size_t plane = (size_t)img_w * img_h;
    uint8_t* planes = nullptr;
    cudaError_t e = cudaMalloc((void**)&planes, plane * 4);
    if (e != cudaSuccess) return cuda_status(e, "carving planes");
    cudaStream_t st = (cudaStream_t)stream;
    const uint8_t* src[4] = {red, green, blue, mask};
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
        if (src[i]) e = cudaMemcpyAsync(planes + i * plane, src[i], plane, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cudaFree(planes);
        return cuda_status(e, "carving planes");
    }
    CarveArgs a;
    std::memcpy(a.P, projection, sizeof(a.P));
    a.W = g->W;
    a.H = g->H;
    a.D = g->D;
    a.img_w = img_w;
    a.img_h = img_h;
    a.radius = radius;
    a.red = planes;
    a.green = planes + plane;
    a.blue = planes + 2 * plane;
    a.mask = mask ? planes + 3 * plane : nullptr;
    a.params = g->prec == kPrecFP32 ? g->params[g->cur] : nullptr;
    a.rec = g->rec;
    a.density = g->density;
    a.adaptive_lr = g->adaptive_lr;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_carve<<<sms * 8, 256, 0, st>>>(a);
    count_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(planes);
    if (e != cudaSuccess) return cuda_status(e, "carving");
    return refresh_dense_mirror(g, st);  // the density changed: the empty-space maps follow
}

extern "C" cpx_status cpx_grid_bbox(cpx_grid* g, int* bbox_out, double* scale_ratio_out)
{
    if (!g || !bbox_out) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse) {
        set_error("the bounding-box search runs on the dense grid");
        return CPX_ERR_UNSUPPORTED;
    }
    BoxAcc init;
    init.b[0] = g->W;
    init.b[1] = -1;
    init.b[2] = g->H;
    init.b[3] = -1;
    init.b[4] = g->D;
    init.b[5] = -1;
    init.max_radius = 0ull;
    BoxAcc* acc = nullptr;
    cudaError_t e = cudaMalloc((void**)&acc, sizeof(BoxAcc));
    if (e == cudaSuccess) e = cudaMemcpy(acc, &init, sizeof(BoxAcc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int64_t cols = (int64_t)g->W * g->H;
        k_box_columns<<<(unsigned)((cols + 255) / 256), 256>>>(g->adaptive_lr, g->W, g->H, g->D,
                                                              scale_ratio_out != nullptr, acc);
        count_launch();
        e = cudaGetLastError();
    }
    BoxAcc out;
    if (e == cudaSuccess) e = cudaMemcpy(&out, acc, sizeof(BoxAcc), cudaMemcpyDeviceToHost);
    cudaFree(acc);
    if (e != cudaSuccess) return cuda_status(e, "bounding box");
    // the box becomes the grid's ray box (the reference sets scene->bbox_*, RenderUtils.cu:457-464)
    for (int i = 0; i < 6; i++) {
        bbox_out[i] = out.b[i];
        g->bbox[i] = out.b[i];
    }
    if (scale_ratio_out) {
        double r;
        std::memcpy(&r, &out.max_radius, sizeof(r));
        *scale_ratio_out = r / g->W * 2.;
    }
    return CPX_OK;
}
