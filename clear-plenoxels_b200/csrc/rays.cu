// rays.cu -- training rays of a camera on the device (getBound + initialRays,
// SparseVolumeRadianceField/Rays.cu:22-144).
//
// One thread per listed pixel.  The arithmetic is the reference's, operation
// for operation (pixel centre in double, direction accumulated in float
// through double products, float sum of squares normalised by a double
// square root, slab test in double), so directions and near/far are the
// reference's bit for bit.
#include "cpx_internal.cuh"

namespace cpx {

struct CamArgs {
    double alpha[2];
    double principle[2];
    double c2w[16];
    double centre[4];
    int bbox[6];
};

__device__ __forceinline__ double minf_d(double x1, double x2) { return x1 > x2 ? x2 : x1; }
__device__ __forceinline__ double maxf_d(double x1, double x2) { return x1 > x2 ? x1 : x2; }

// normalizePoint (Rays.cu:13-20)
__device__ __forceinline__ void normalize_point(float* point)
{
    double sum = point[0] * point[0] + point[1] * point[1] + point[2] * point[2];
    sum = sqrt(sum);
    point[0] /= sum;
    point[1] /= sum;
    point[2] /= sum;
}

__global__ void k_rays_camera(CamArgs cam, int img_w, const uint8_t* __restrict__ red,
                              const uint8_t* __restrict__ green, const uint8_t* __restrict__ blue,
                              const uint8_t* __restrict__ mask, int has_mask,
                              const int32_t* __restrict__ pix, int64_t n_pix, int64_t offset,
                              RaysView rays_out_base, int white_bg)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_pix) return;
    const int pixelIndex = pix[i];
    const int pixelRow = pixelIndex / img_w;
    const int pixelCol = pixelIndex % img_w;
    // getBound (Rays.cu:22-75)
    float xInCamera[4] = {
        (float)((pixelCol + 0.5 - cam.principle[0]) / cam.alpha[0]),
        (float)((pixelRow + 0.5 - cam.principle[1]) / cam.alpha[1]),
        1.0f,
        1.0f,
    };
    float secondPoint[4];
    for (int row = 0; row < 4; row++) {
        secondPoint[row] = 0.;
        for (int col = 0; col < 4; col++) secondPoint[row] += cam.c2w[row * 4 + col] * xInCamera[col];
        secondPoint[row] -= cam.centre[row];
    }
    normalize_point(secondPoint);
    double t[6] = {
        (cam.bbox[1] - cam.centre[0]) / secondPoint[0],
        (cam.bbox[0] - cam.centre[0]) / secondPoint[0],
        (cam.bbox[3] - cam.centre[1]) / secondPoint[1],
        (cam.bbox[2] - cam.centre[1]) / secondPoint[1],
        (cam.bbox[5] - cam.centre[2]) / secondPoint[2],
        (cam.bbox[4] - cam.centre[2]) / secondPoint[2],
    };
    double t_min = minf_d(t[0], t[1]);
    double t_max = maxf_d(t[0], t[1]);
    t_min = maxf_d(t_min, minf_d(t[2], t[3]));
    t_max = minf_d(t_max, maxf_d(t[2], t[3]));
    t_min = maxf_d(t_min, minf_d(t[4], t[5]));
    t_max = minf_d(t_max, maxf_d(t[4], t[5]));
    float rayInfo[5];
    rayInfo[0] = t_min;
    rayInfo[1] = t_max;
    rayInfo[2] = secondPoint[0];
    rayInfo[3] = secondPoint[1];
    rayInfo[4] = secondPoint[2];

    // initialRays (Rays.cu:106-138)
    const int64_t ri = offset + i;
    float* ox = const_cast<float*>(rays_out_base.ox);
    float* oy = const_cast<float*>(rays_out_base.oy);
    float* oz = const_cast<float*>(rays_out_base.oz);
    float* dx = const_cast<float*>(rays_out_base.dx);
    float* dy = const_cast<float*>(rays_out_base.dy);
    float* dz = const_cast<float*>(rays_out_base.dz);
    float* nt = const_cast<float*>(rays_out_base.near_t);
    float* ft = const_cast<float*>(rays_out_base.far_t);
    uint8_t* gm = const_cast<uint8_t*>(rays_out_base.mask);
    uint8_t* gr = const_cast<uint8_t*>(rays_out_base.r);
    uint8_t* gg = const_cast<uint8_t*>(rays_out_base.g);
    uint8_t* gb = const_cast<uint8_t*>(rays_out_base.b);
    ox[ri] = cam.centre[0];
    oy[ri] = cam.centre[1];
    oz[ri] = cam.centre[2];
    nt[ri] = rayInfo[0];
    ft[ri] = rayInfo[1];
    dx[ri] = rayInfo[2];
    dy[ri] = rayInfo[3];
    dz[ri] = rayInfo[4];
    const uint8_t m = has_mask ? mask[pixelIndex] : (uint8_t)255;
    gm[ri] = m;
    if (white_bg) {
        gr[ri] = red[pixelIndex] * m / 255.f + 255 - m;
        gg[ri] = green[pixelIndex] * m / 255.f + 255 - m;
        gb[ri] = blue[pixelIndex] * m / 255.f + 255 - m;
    } else {
        gr[ri] = red[pixelIndex];
        gg[ri] = green[pixelIndex];
        gb[ri] = blue[pixelIndex];
    }
}

cpx_status rays_camera_launch(cpx_rays* r, const cpx_grid* g, const cpx_camera* cam, int img_w,
                              int64_t plane_bytes, const uint8_t* planes_dev,
                              const int32_t* pix_dev, int64_t n_pix, int64_t offset, int has_mask,
                              cudaStream_t st)
{
    CamArgs a;
    for (int i = 0; i < 2; i++) {
        a.alpha[i] = cam->alpha[i];
        a.principle[i] = cam->principle[i];
    }
    for (int i = 0; i < 16; i++) a.c2w[i] = cam->c2w[i];
    for (int i = 0; i < 4; i++) a.centre[i] = cam->centre[i];
    for (int i = 0; i < 6; i++) a.bbox[i] = g->bbox[i];
    const RaysView rv = rays_view(r);
    // planes_dev holds [red | green | blue | mask], plane_bytes each
    k_rays_camera<<<(unsigned)((n_pix + 255) / 256), 256, 0, st>>>(
        a, img_w, planes_dev, planes_dev + plane_bytes, planes_dev + 2 * plane_bytes,
        planes_dev + 3 * plane_bytes, has_mask, pix_dev, n_pix, offset, rv, r->white_bg);
    count_launch();
    return cuda_status(cudaGetLastError(), "rays");
}

}  // namespace cpx
