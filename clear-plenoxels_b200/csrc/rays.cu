// rays.cu -- training rays of a camera on the device (getBound + initialRays,
// SparseVolumeRadianceField/Rays.cu:22-144).
//
// One thread per listed pixel.  The arithmetic is the reference's, operation
// for operation (pixel centre in double, direction accumulated in float
// through double products, float sum of squares normalised by a double
// square root, slab test in double), so directions and near/far are the
// reference's bit for bit.
#include <cstring>
#include <vector>

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

// One ray: pixel pixelIndex of camera `cam`, written at ray ri.
__device__ __forceinline__ void camera_ray(const CamArgs& cam, int img_w, const uint8_t* __restrict__ red,
                                           const uint8_t* __restrict__ green, const uint8_t* __restrict__ blue,
                                           const uint8_t* __restrict__ mask, int has_mask, int pixelIndex,
                                           int64_t ri, const RaysView& rays_out_base, int white_bg)
{
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

__global__ void k_rays_camera(CamArgs cam, int img_w, const uint8_t* __restrict__ red,
                              const uint8_t* __restrict__ green, const uint8_t* __restrict__ blue,
                              const uint8_t* __restrict__ mask, int has_mask,
                              const int32_t* __restrict__ pix, int64_t n_pix, int64_t offset,
                              RaysView rays_out_base, int white_bg)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_pix) return;
    camera_ray(cam, img_w, red, green, blue, mask, has_mask, pix[i], offset + i, rays_out_base, white_bg);
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

// ---------------------------------------------------------------------------
// Ray source: the training rays generated per batch on the device from (camera, pixel)
// samples, instead of read from a table of every ray.  The reference builds the whole table
// (_rays::initialSelf, Rays.cu:187-240), shuffles an index on the host (ShuffleRank,
// Utils.cu:488-506) and gathers the table into that order (shuffleTo, Rays.cu:242-287); here
// the images and pixel lists stay on the device and sample i of an epoch is
// permute(i), a keyed bijection of [0, n): a 4-round Feistel network on the next even power of
// two, cycle-walked until the image lands below n.  The rays of a sample are the reference's
// bit for bit (the same per-ray arithmetic as cpx_rays_init_camera); the order is a uniform
// shuffle, not the host rand() sequence.
// ---------------------------------------------------------------------------
struct SourceArgs {
    const CamArgs* cams;
    const int64_t* cam_off;  // [n_cams + 1]: first sample of each camera
    int n_cams;
    int img_w;
    int64_t plane;
    const uint8_t* planes;   // per camera: red | green | blue | mask, plane bytes each
    int has_mask;
    const int32_t* pix;      // concatenated pixel lists, or null: every pixel of every camera
    int64_t n;
    int half_bits;           // Feistel half width; the domain is 2^(2 half_bits) >= n
    uint32_t key[4];
    int shuffled;
    int bbox[6];
    int white_bg;
    int* err;
};

__host__ __device__ __forceinline__ uint64_t feistel4(uint64_t x, int half_bits, const uint32_t* key)
{
    const uint64_t mask = (half_bits >= 64) ? ~0ull : ((1ull << half_bits) - 1ull);
    uint64_t L = x >> half_bits, R = x & mask;
    for (int r = 0; r < 4; r++) {
        const uint64_t f = (uint64_t)fmix32((uint32_t)R ^ key[r]) & mask;
        const uint64_t nl = R;
        R = L ^ f;
        L = nl;
    }
    return (L << half_bits) | R;
}

__global__ void k_rays_source(SourceArgs a, int64_t start, int len, RaysView out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    uint64_t j = (uint64_t)(start + i);
    if (a.shuffled) {
        // cycle-walk: the Feistel network permutes the power-of-two domain, so iterating it
        // from a value below n comes back below n (expected steps < 4 as n > domain / 4)
        int steps = 0;
        do {
            j = feistel4(j, a.half_bits, a.key);
        } while (j >= (uint64_t)a.n && ++steps < 4096);
        if (j >= (uint64_t)a.n) {
            atomicOr(a.err, 16);
            j = (uint64_t)(start + i);
        }
    }
    int lo = 0, hi = a.n_cams - 1;  // the camera whose range holds sample j
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.cam_off[mid] <= (int64_t)j) lo = mid;
        else hi = mid - 1;
    }
    const int c = lo;
    const int pixel = a.pix ? a.pix[j] : (int)((int64_t)j - a.cam_off[c]);
    CamArgs cam = a.cams[c];
    for (int k = 0; k < 6; k++) cam.bbox[k] = a.bbox[k];
    const uint8_t* base = a.planes + (size_t)c * 4 * a.plane;
    camera_ray(cam, a.img_w, base, base + a.plane, base + 2 * a.plane, base + 3 * a.plane, a.has_mask, pixel, i, out,
               a.white_bg);
}

}  // namespace cpx

using namespace cpx;

struct cpx_ray_source {
    SourceArgs a;
    CamArgs* cams = nullptr;
    int64_t* cam_off = nullptr;
    uint8_t* planes = nullptr;
    int32_t* pix = nullptr;
    int* err = nullptr;
};

static void source_free(cpx_ray_source* s)
{
    cudaFree(s->cams);
    cudaFree(s->cam_off);
    cudaFree(s->planes);
    cudaFree(s->pix);
    cudaFree(s->err);
    delete s;
}

static uint64_t splitmix64(uint64_t& x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

extern "C" {

cpx_status cpx_ray_source_create(const cpx_camera* cams, int n_cams, int img_w, int img_h, const uint8_t* red,
                                 const uint8_t* green, const uint8_t* blue, const uint8_t* gt_mask,
                                 const int32_t* pixel_index, const int64_t* n_pix, int white_bg,
                                 cpx_ray_source** out)
{
    if (!cams || n_cams < 1 || img_w < 1 || img_h < 1 || !red || !green || !blue || !out ||
        (pixel_index && !n_pix)) {
        set_error("a ray source needs cameras, image planes and, with pixel lists, their lengths");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t plane = (int64_t)img_w * img_h;
    std::vector<int64_t> off(n_cams + 1, 0);
    for (int c = 0; c < n_cams; c++) {
        const int64_t k = pixel_index ? n_pix[c] : plane;
        if (k < 0) {
            set_error("negative pixel count");
            return CPX_ERR_INVALID_ARGUMENT;
        }
        off[c + 1] = off[c] + k;
    }
    const int64_t n = off[n_cams];
    if (pixel_index) {
        for (int64_t i = 0; i < n; i++)
            if (pixel_index[i] < 0 || pixel_index[i] >= plane) {
                set_error("pixel index %d outside the %dx%d image", pixel_index[i], img_w, img_h);
                return CPX_ERR_INVALID_ARGUMENT;
            }
    }
    cpx_ray_source* s = new cpx_ray_source();
    std::vector<CamArgs> ca(n_cams);
    for (int c = 0; c < n_cams; c++) {
        std::memset(&ca[c], 0, sizeof(CamArgs));
        for (int i = 0; i < 2; i++) {
            ca[c].alpha[i] = cams[c].alpha[i];
            ca[c].principle[i] = cams[c].principle[i];
        }
        for (int i = 0; i < 16; i++) ca[c].c2w[i] = cams[c].c2w[i];
        for (int i = 0; i < 4; i++) ca[c].centre[i] = cams[c].centre[i];
    }
    cudaError_t e = cudaMalloc((void**)&s->cams, sizeof(CamArgs) * n_cams);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->cam_off, sizeof(int64_t) * (n_cams + 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->planes, (size_t)n_cams * 4 * plane);
    if (e == cudaSuccess && pixel_index) e = cudaMalloc((void**)&s->pix, sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->err, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMemset(s->err, 0, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMemcpy(s->cams, ca.data(), sizeof(CamArgs) * n_cams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->cam_off, off.data(), sizeof(int64_t) * (n_cams + 1), cudaMemcpyHostToDevice);
    const uint8_t* src[4] = {red, green, blue, gt_mask};
    for (int c = 0; c < n_cams && e == cudaSuccess; c++)
        for (int q = 0; q < 4 && e == cudaSuccess; q++)
            if (src[q])
                e = cudaMemcpy(s->planes + ((size_t)c * 4 + q) * plane, src[q] + (size_t)c * plane, plane,
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess && pixel_index && n > 0)
        e = cudaMemcpy(s->pix, pixel_index, sizeof(int32_t) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        source_free(s);
        set_error("ray source of %lld samples could not be set up", (long long)n);
        return CPX_ERR_OUT_OF_MEMORY;
    }
    SourceArgs& a = s->a;
    std::memset(&a, 0, sizeof(a));
    a.cams = s->cams;
    a.cam_off = s->cam_off;
    a.n_cams = n_cams;
    a.img_w = img_w;
    a.plane = plane;
    a.planes = s->planes;
    a.has_mask = gt_mask != nullptr;
    a.pix = s->pix;
    a.n = n;
    int bits = 2;
    while (bits < 64 && ((uint64_t)1 << bits) < (uint64_t)n) bits += 2;
    a.half_bits = bits / 2;
    a.shuffled = 0;
    a.white_bg = white_bg ? 1 : 0;
    a.err = s->err;
    *out = s;
    return CPX_OK;
}

cpx_status cpx_ray_source_destroy(cpx_ray_source* s)
{
    if (!s) return CPX_OK;
    cudaDeviceSynchronize();
    source_free(s);
    return CPX_OK;
}

cpx_status cpx_ray_source_count(const cpx_ray_source* s, int64_t* n)
{
    if (!s || !n) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    *n = s->a.n;
    return CPX_OK;
}

cpx_status cpx_ray_source_shuffle(cpx_ray_source* s, uint64_t seed, int shuffled)
{
    if (!s) {
        set_error("null ray source");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    uint64_t x = seed;
    for (int r = 0; r < 4; r++) s->a.key[r] = (uint32_t)splitmix64(x);
    s->a.shuffled = shuffled ? 1 : 0;
    return CPX_OK;
}

cpx_status cpx_ray_source_keys(const cpx_ray_source* s, uint32_t* keys, int* half_bits)
{
    if (!s || !keys || !half_bits) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    for (int r = 0; r < 4; r++) keys[r] = s->a.key[r];
    *half_bits = s->a.half_bits;
    return CPX_OK;
}

cpx_status cpx_ray_source_generate(cpx_ray_source* s, const cpx_grid* g, int64_t start, int len, cpx_rays* batch,
                                   cpx_stream stream)
{
    if (batch) ++batch->epoch;  // new ray fields: a placement done in advance is stale
    if (!s || !g || !batch || len < 0 || start < 0 || start + len > s->a.n || len > batch->n) {
        set_error("batch [%lld, +%d) outside the source's %lld samples or the ray buffer", (long long)start, len,
                  s ? (long long)s->a.n : 0ll);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (batch->white_bg != s->a.white_bg) {
        set_error("the ray buffer's background differs from the source's");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (len == 0) return CPX_OK;
    SourceArgs a = s->a;
    for (int i = 0; i < 6; i++) a.bbox[i] = g->bbox[i];
    k_rays_source<<<(unsigned)((len + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, start, len, rays_view(batch));
    count_launch();
    return cuda_status(cudaGetLastError(), "ray source");
}

cpx_status cpx_ray_source_check(cpx_ray_source* s)
{
    if (!s) {
        set_error("null ray source");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    int flags[4] = {0, 0, 0, 0};
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(flags, s->err, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "ray source check");
    cudaMemset(s->err, 0, sizeof(flags));
    if (flags[0] & 16) {
        set_error("the shuffle's cycle walk ran out of steps");
        return CPX_ERR_CUDA;
    }
    return CPX_OK;
}

}  // extern "C"
