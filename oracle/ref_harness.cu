// ref_harness.cu -- C-ABI shim around the reference's own entry points.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the
// reference's unmodified sources (Utils, ImageUtils, CameraUtils, SceneUtils,
// Rays, Optimizer, RenderUtils .cu) into oracle/_ref/libcpxref.so.  It fills the
// reference's plain structs (ObjectScene, Rays, Optimizer, Camera, Image) from
// caller buffers and calls the reference's public methods exactly as the
// reference's batch loop does (SVRF/Render.cu:407-500):
//   RenderUtils::renderRays, RenderUtils::renderRays_withGradients_RGB,
//   RenderUtils::addVarianceLoss, Optimizer::updateRGBScene,
//   objectScene::pruneSelf / getCagedNums, _rays::initialSelf.
// It is the parity pin for the CUDA product path and the reference arm of the
// benchmark; nothing in the product links it.
//
// One guard keeps the reference's kernels inside their buffers: the per-sample
// jitter arrays are re-allocated zero-padded beyond maxSamplePoint, because the
// march index can pass it (the loop count is bounded by (far - near + 1) / step
// + 2, RenderUtils.cu:1674-1705).

#include "RenderUtils.cuh"
#include "Optimizer.cuh"
#include "Rays.cuh"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct RefCtx {
    ObjectScene scene;
    Optimizer opt;
    Rays rays;
    bool have_opt = false;
    bool have_rays = false;
    double lr = 0., sh_lr = 0.;
    int* sample_index_dev = nullptr;  // identity table over all rays
    double* losses_dev = nullptr;
    int losses_cap = 0;
    int n_arrays = 0;
    float** param_ptrs_host = nullptr;  // host copy of scene.totalVariableGPUPtrs
    std::vector<float*> grad_ptrs, m_ptrs, v_ptrs;
};

int fail(cudaError_t e) { return e == cudaSuccess ? 0 : 100 + (int)e; }

// Pull the per-array device pointers of an Optimizer table to the host.
std::vector<float*> table_to_host(float** dev_table, int n)
{
    std::vector<float*> out(n, nullptr);
    cudaMemcpy(out.data(), dev_table, sizeof(float*) * n, cudaMemcpyDeviceToHost);
    return out;
}

// Replace the scene's jitter arrays with zeroed arrays long enough for every sample index.
int pad_offsets(ObjectScene& s)
{
    const int pad = (int)(2.0 / s.stepSize) + 64;
    const int n = s.maxSamplePoint + pad;
    double* bufs[3];
    for (int i = 0; i < 3; i++) {
        if (cudaMalloc((void**)&bufs[i], sizeof(double) * n) != cudaSuccess) return 2;
        cudaMemset(bufs[i], 0, sizeof(double) * n);
    }
    cudaFree(s.offsetXDevice);
    cudaFree(s.offsetYDevice);
    cudaFree(s.offsetZDevice);
    s.offsetXDevice = bufs[0];
    s.offsetYDevice = bufs[1];
    s.offsetZDevice = bufs[2];
    return 0;
}

}  // namespace

extern "C" {

int ref_device_sync(void) { return fail(cudaDeviceSynchronize()); }

// Dense scene (objectScene::initSelf with solid=true, SVRF/SceneUtils.cu:60-175),
// parameters overwritten from planar host arrays [(1+3 sh_dim)][W*H*D].
int ref_scene_create_dense(int W, int H, int D, int sh_dim, int band, float step,
                           const float* planar, const float* adaptive_lr, void** out)
{
    RefCtx* c = new RefCtx();
    c->scene.initSelf(W, H, D, false, true, 0.f, 0.f, step, sh_dim);
    c->scene.optimizingBand = band;
    c->n_arrays = 1 + 3 * sh_dim;
    c->param_ptrs_host = c->scene.totalVariableGPUPtrs;
    const int64_t N = (int64_t)W * H * D;
    for (int a = 0; a < c->n_arrays; a++)
        cudaMemcpy(c->param_ptrs_host[a], planar + (int64_t)a * N, sizeof(float) * N,
                   cudaMemcpyHostToDevice);
    if (adaptive_lr)
        cudaMemcpy(c->scene.adaptiveLRDevice, adaptive_lr, sizeof(float) * N, cudaMemcpyHostToDevice);
    int rc = pad_offsets(c->scene);
    if (rc) return rc;
    *out = c;
    return fail(cudaDeviceSynchronize());
}

// Sparse scene the way initSelfByUpsample builds it (SVRF/SceneUtils.cu:520-600):
// a dense temporary is pruned (pruneSelf) and scanned (getCagedNums), the sparse
// scene takes its occupancy / in-cage / index tables and the compacted parameters.
int ref_scene_create_sparse(int W, int H, int D, int sh_dim, int band, float step,
                            const float* dense_planar, float threshold, void** out,
                            uint32_t* n_in_cage)
{
    const int64_t N = (int64_t)W * H * D;
    const int n_arrays = 1 + 3 * sh_dim;
    ObjectScene temp;
    temp.initSelf(W, H, D, false, true, 0.f, 0.f, step, 1);
    cudaMemcpy(temp.sceneOpacityDevice, dense_planar, sizeof(float) * N, cudaMemcpyHostToDevice);
    temp.pruneSelf(threshold);
    temp.getCagedNums();
    const uint32_t cnt = temp.inCageNums;

    RefCtx* c = new RefCtx();
    c->scene.initSelf(W, H, D, false, false, 0.f, 0.f, step, sh_dim, (int)cnt);
    c->scene.optimizingBand = band;
    c->scene.sparse = true;
    c->n_arrays = n_arrays;
    c->param_ptrs_host = c->scene.totalVariableGPUPtrs;
    const int64_t C = (int64_t)(W - 1) * (H - 1) * (D - 1);
    cudaMemcpy(c->scene.occupancyDevice, temp.occupancyDevice, C, cudaMemcpyDeviceToDevice);
    cudaMalloc((void**)&c->scene.inCageInfoDevice, N);
    cudaMemcpy(c->scene.inCageInfoDevice, temp.inCageInfoDevice, N, cudaMemcpyDeviceToDevice);
    cudaMalloc((void**)&c->scene.indexOffsetsDevice, sizeof(unsigned int) * N);
    cudaMemcpy(c->scene.indexOffsetsDevice, temp.indexOffsetsDevice, sizeof(unsigned int) * N,
               cudaMemcpyDeviceToDevice);
    c->scene.inCageNums = cnt;
    // compaction in z-y-x order of the in-cage flags (SVRF/SceneUtils.cu:585-602)
    std::vector<float> comp((size_t)cnt);
    for (int a = 0; a < n_arrays; a++) {
        const float* src = dense_planar + (int64_t)a * N;
        size_t k = 0;
        for (int64_t v = 0; v < N; v++)
            if (temp.inCageInfoHost[v]) comp[k++] = src[v];
        cudaMemcpy(c->param_ptrs_host[a], comp.data(), sizeof(float) * cnt, cudaMemcpyHostToDevice);
    }
    temp.freeSelf();
    int rc = pad_offsets(c->scene);
    if (rc) return rc;
    if (n_in_cage) *n_in_cage = cnt;
    *out = c;
    return fail(cudaDeviceSynchronize());
}

// Occupancy outputs of a sparse scene (for the bit-exact comparison).
int ref_download_occupancy(void* h, uint8_t* occ, uint8_t* in_cage, uint32_t* index_offsets)
{
    RefCtx* c = (RefCtx*)h;
    const ObjectScene& s = c->scene;
    const int64_t N = (int64_t)s.sceneWidth * s.sceneHeight * s.sceneDepth;
    const int64_t C = (int64_t)(s.sceneWidth - 1) * (s.sceneHeight - 1) * (s.sceneDepth - 1);
    if (occ) cudaMemcpy(occ, s.occupancyDevice, C, cudaMemcpyDeviceToHost);
    if (in_cage) cudaMemcpy(in_cage, s.inCageInfoDevice, N, cudaMemcpyDeviceToHost);
    if (index_offsets)
        cudaMemcpy(index_offsets, s.indexOffsetsDevice, sizeof(uint32_t) * N, cudaMemcpyDeviceToHost);
    return fail(cudaDeviceSynchronize());
}

int ref_set_offsets(void* h, const double* ox, const double* oy, const double* oz, int n)
{
    RefCtx* c = (RefCtx*)h;
    const int pad = (int)(2.0 / c->scene.stepSize) + 64;
    if (n > c->scene.maxSamplePoint + pad) return 1;
    cudaMemcpy(c->scene.offsetXDevice, ox, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(c->scene.offsetYDevice, oy, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(c->scene.offsetZDevice, oz, sizeof(double) * n, cudaMemcpyHostToDevice);
    return fail(cudaDeviceSynchronize());
}

// objectScene::setSelfSampleOffset(stepSize / 2) right after srand(seed), as the batch loop calls
// it under SolidStrategy 0 (SVRF/Render.cu:402-405, SceneUtils.cu:792-798): the three offset
// arrays (maxSamplePoint entries each, x then y then z) to host memory.
int ref_sample_offsets(void* h, unsigned seed, double* out, int* n_out)
{
    RefCtx* c = (RefCtx*)h;
    srand(seed);
    c->scene.setSelfSampleOffset(c->scene.stepSize / 2.);
    const int n = c->scene.maxSamplePoint;
    cudaMemcpy(out, c->scene.offsetXDevice, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + n, c->scene.offsetYDevice, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + 2 * n, c->scene.offsetZDevice, sizeof(double) * n, cudaMemcpyDeviceToHost);
    *n_out = n;
    return fail(cudaDeviceSynchronize());
}

// The values the host's rand() returns after srand(seed): the seeds randGPU's calls draw.
void ref_rand_values(unsigned seed, unsigned* out, int n)
{
    srand(seed);
    for (int i = 0; i < n; i++) out[i] = (unsigned)rand();
}

int ref_max_sample_point(void* h) { return ((RefCtx*)h)->scene.maxSamplePoint; }

// Optimizer over the scene's parameter table (Optimizer.cu:81-187, Render.cu:63, 300-305).
int ref_optimizer_init(void* h, int hierarchy)
{
    RefCtx* c = (RefCtx*)h;
    c->opt.initialSelf(c->scene.actualGridNums, Adam, c->scene.totalVariableGPUPtrsDevice,
                       c->n_arrays);
    c->opt.initialAll();
    c->opt.hierarchyStrategy = hierarchy != 0;
    c->opt.setLearningRate(&c->lr, &c->sh_lr);
    c->grad_ptrs = table_to_host(c->opt.gradientDevice, c->n_arrays);
    c->m_ptrs = table_to_host(c->opt.momentumDevice, c->n_arrays);
    c->v_ptrs = table_to_host(c->opt.varianceDevice, c->n_arrays);
    c->have_opt = true;
    return fail(cudaDeviceSynchronize());
}

static int ensure_losses(RefCtx* c, int n)
{
    if (c->losses_cap >= n) return 0;
    cudaFree(c->losses_dev);
    c->losses_cap = n;
    return fail(cudaMalloc((void**)&c->losses_dev, sizeof(double) * n));
}

static int make_identity_index(RefCtx* c, int n)
{
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    cudaFree(c->sample_index_dev);
    cudaMalloc((void**)&c->sample_index_dev, sizeof(int) * n);
    return fail(cudaMemcpy(c->sample_index_dev, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
}

// Ray table filled directly (all 17 SoA fields of Rays.cuh:8-57, RGB).
int ref_rays_create(void* h, int n, int white_bg, const float* ox, const float* oy,
                    const float* oz, const float* dx, const float* dy, const float* dz,
                    const float* near_t, const float* far_t, const uint8_t* mask,
                    const uint8_t* r, const uint8_t* g, const uint8_t* b)
{
    RefCtx* c = (RefCtx*)h;
    c->rays.totalRays = n;
    c->rays.graylized = false;
    c->rays.whiteBKGD = white_bg != 0;
    c->rays.maskRaysOnly = true;
    c->rays.allocateSelfMemory();
    Rays& R = c->rays;
    cudaMemcpy(R.cameraCenterX_Device, ox, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.cameraCenterY_Device, oy, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.cameraCenterZ_Device, oz, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.directionX_Device, dx, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.directionY_Device, dy, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.directionZ_Device, dz, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.near_t_Device, near_t, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.far_t_Device, far_t, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.gtMask_Device, mask, n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.gtRed_Device, r, n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.gtGreen_Device, g, n, cudaMemcpyHostToDevice);
    cudaMemcpy(R.gtBlue_Device, b, n, cudaMemcpyHostToDevice);
    cudaMemset(R.accumulatedDensity_Device, 0, sizeof(float) * n);
    cudaMemset(R.accumulatedWeights_Device, 0, sizeof(float) * n);
    cudaMemset(R.accumulatedRed_Device, 0, sizeof(float) * n);
    cudaMemset(R.accumulatedGreen_Device, 0, sizeof(float) * n);
    cudaMemset(R.accumulatedBlue_Device, 0, sizeof(float) * n);
    c->have_rays = true;
    int rc = make_identity_index(c, n);
    if (rc) return rc;
    return fail(cudaDeviceSynchronize());
}

// Rays from cameras and images through _rays::initialSelf (Rays.cu:187-240).
// Per camera: alpha[2], principle[2], c2w[16], centre[4] (the device fields
// getBound reads); images are 4 planes (r, g, b, mask) of img_w*img_h bytes;
// pix[i] lists camera i's pixels (its masksIndex), n_pix[i] their count.
int ref_rays_init(void* h, int ncam, const double* alpha, const double* principle,
                  const double* c2w, const double* centre, int img_w, int img_h,
                  const uint8_t* images, const int* pix_concat, const int* n_pix,
                  int white_bg)
{
    RefCtx* c = (RefCtx*)h;
    std::vector<Camera> cams(ncam);
    std::vector<Image> imgs(ncam);
    std::vector<int> order(ncam);
    std::vector<std::vector<int>> pix_lists(ncam);
    const size_t plane = (size_t)img_w * img_h;
    size_t off = 0;
    for (int i = 0; i < ncam; i++) {
        Camera& cam = cams[i];
        cudaMalloc((void**)&cam.alphaDevice, sizeof(double) * 2);
        cudaMemcpy(cam.alphaDevice, alpha + 2 * i, sizeof(double) * 2, cudaMemcpyHostToDevice);
        cudaMalloc((void**)&cam.principleDevice, sizeof(double) * 2);
        cudaMemcpy(cam.principleDevice, principle + 2 * i, sizeof(double) * 2, cudaMemcpyHostToDevice);
        cudaMalloc((void**)&cam.c2wExternalMatDevice, sizeof(double) * 16);
        cudaMemcpy(cam.c2wExternalMatDevice, c2w + 16 * i, sizeof(double) * 16, cudaMemcpyHostToDevice);
        cudaMalloc((void**)&cam.cameraCenterDevice, sizeof(double) * 4);
        cudaMemcpy(cam.cameraCenterDevice, centre + 4 * i, sizeof(double) * 4, cudaMemcpyHostToDevice);
        Image& im = imgs[i];
        im.width = img_w;
        im.height = img_h;
        im.grayImage = false;
        const uint8_t* base = images + (size_t)i * 4 * plane;
        uint8_t* planes[4];
        for (int p = 0; p < 4; p++) {
            cudaMalloc((void**)&planes[p], plane);
            cudaMemcpy(planes[p], base + p * plane, plane, cudaMemcpyHostToDevice);
        }
        im.redDevice = planes[0];
        im.greenDevice = planes[1];
        im.blueDevice = planes[2];
        im.maskDevice = planes[3];
        pix_lists[i].assign(pix_concat + off, pix_concat + off + n_pix[i]);
        off += n_pix[i];
        im.masksIndex = pix_lists[i].data();
        im.masksLen = n_pix[i];
        order[i] = i;
    }
    c->rays.initialSelf(cams.data(), imgs.data(), c->scene, ncam, true, false, white_bg != 0,
                        order.data());
    for (int i = 0; i < ncam; i++) {
        cudaFree(cams[i].alphaDevice);
        cudaFree(cams[i].principleDevice);
        cudaFree(cams[i].c2wExternalMatDevice);
        cudaFree(cams[i].cameraCenterDevice);
        cudaFree(imgs[i].redDevice);
        cudaFree(imgs[i].greenDevice);
        cudaFree(imgs[i].blueDevice);
        cudaFree(imgs[i].maskDevice);
    }
    cudaMemset(c->rays.accumulatedDensity_Device, 0, sizeof(float) * c->rays.totalRays);
    cudaMemset(c->rays.accumulatedWeights_Device, 0, sizeof(float) * c->rays.totalRays);
    cudaMemset(c->rays.accumulatedRed_Device, 0, sizeof(float) * c->rays.totalRays);
    cudaMemset(c->rays.accumulatedGreen_Device, 0, sizeof(float) * c->rays.totalRays);
    cudaMemset(c->rays.accumulatedBlue_Device, 0, sizeof(float) * c->rays.totalRays);
    c->have_rays = true;
    int rc = make_identity_index(c, c->rays.totalRays);
    if (rc) return rc;
    return fail(cudaDeviceSynchronize());
}

int ref_rays_count(void* h) { return ((RefCtx*)h)->rays.totalRays; }


// RenderUtils::renderImage (RenderUtils.cu:1802) of one camera into host buffers:
// rgb float [3][w*h], rgb8 u8 [3][w*h], depth float [w*h], mask u8 [w*h].
int ref_render_image(void* h, const double* alpha, const double* principle, const double* c2w,
                     const double* centre, int width, int height, int white_bg, float* rgb,
                     uint8_t* rgb8, float* depth, uint8_t* mask)
{
    RefCtx* c = (RefCtx*)h;
    const size_t n = (size_t)width * height;
    Camera cam;
    cudaMalloc((void**)&cam.alphaDevice, sizeof(double) * 2);
    cudaMemcpy(cam.alphaDevice, alpha, sizeof(double) * 2, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&cam.principleDevice, sizeof(double) * 2);
    cudaMemcpy(cam.principleDevice, principle, sizeof(double) * 2, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&cam.c2wExternalMatDevice, sizeof(double) * 16);
    cudaMemcpy(cam.c2wExternalMatDevice, c2w, sizeof(double) * 16, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&cam.cameraCenterDevice, sizeof(double) * 4);
    cudaMemcpy(cam.cameraCenterDevice, centre, sizeof(double) * 4, cudaMemcpyHostToDevice);
    Image im;
    im.width = width;
    im.height = height;
    im.grayImage = false;
    im.whiteBG = white_bg != 0;
    float* fl[4];
    uint8_t* by[4];
    for (int p = 0; p < 4; p++) {
        cudaMalloc((void**)&fl[p], sizeof(float) * n);
        cudaMalloc((void**)&by[p], n);
    }
    im.redFloatDevice = fl[0];
    im.greenFloatDevice = fl[1];
    im.blueFloatDevice = fl[2];
    im.disparityDevice = fl[3];
    im.redDevice = by[0];
    im.greenDevice = by[1];
    im.blueDevice = by[2];
    im.maskDevice = by[3];
    RenderUtils::renderImage(im, cam, c->scene);
    int rc = fail(cudaDeviceSynchronize());
    for (int p = 0; p < 3; p++) {
        if (!rc) rc = fail(cudaMemcpy(rgb + p * n, fl[p], sizeof(float) * n, cudaMemcpyDeviceToHost));
        if (!rc) rc = fail(cudaMemcpy(rgb8 + p * n, by[p], n, cudaMemcpyDeviceToHost));
    }
    if (!rc) rc = fail(cudaMemcpy(depth, fl[3], sizeof(float) * n, cudaMemcpyDeviceToHost));
    if (!rc) rc = fail(cudaMemcpy(mask, by[3], n, cudaMemcpyDeviceToHost));
    for (int p = 0; p < 4; p++) {
        cudaFree(fl[p]);
        cudaFree(by[p]);
    }
    cudaFree(cam.alphaDevice);
    cudaFree(cam.principleDevice);
    cudaFree(cam.c2wExternalMatDevice);
    cudaFree(cam.cameraCenterDevice);
    return rc;
}

// Download the ray table: 8 float inputs, 4 byte inputs, 5 float outputs.
int ref_rays_download(void* h, float* ox, float* oy, float* oz, float* dx, float* dy, float* dz,
                      float* near_t, float* far_t, uint8_t* mask, uint8_t* r, uint8_t* g,
                      uint8_t* b, float* acc_den, float* acc_w, float* acc_r, float* acc_g,
                      float* acc_b)
{
    RefCtx* c = (RefCtx*)h;
    Rays& R = c->rays;
    const int n = R.totalRays;
    struct { void* dst; const void* src; size_t sz; } cp[] = {
        {ox, R.cameraCenterX_Device, 4}, {oy, R.cameraCenterY_Device, 4},
        {oz, R.cameraCenterZ_Device, 4}, {dx, R.directionX_Device, 4},
        {dy, R.directionY_Device, 4}, {dz, R.directionZ_Device, 4},
        {near_t, R.near_t_Device, 4}, {far_t, R.far_t_Device, 4},
        {mask, R.gtMask_Device, 1}, {r, R.gtRed_Device, 1}, {g, R.gtGreen_Device, 1},
        {b, R.gtBlue_Device, 1}, {acc_den, R.accumulatedDensity_Device, 4},
        {acc_w, R.accumulatedWeights_Device, 4}, {acc_r, R.accumulatedRed_Device, 4},
        {acc_g, R.accumulatedGreen_Device, 4}, {acc_b, R.accumulatedBlue_Device, 4},
    };
    for (auto& e : cp)
        if (e.dst) cudaMemcpy(e.dst, e.src, e.sz * n, cudaMemcpyDeviceToHost);
    return fail(cudaDeviceSynchronize());
}

// RenderUtils::renderRays (RenderUtils.cu:1961-1971) over rays [start, start+len).
int ref_render_forward(void* h, int start, int len)
{
    RefCtx* c = (RefCtx*)h;
    RenderUtils::renderRays(c->rays, c->scene, c->sample_index_dev, start, len);
    return fail(cudaGetLastError());
}

// RenderUtils::renderRays_withGradients_RGB (RenderUtils.cu:2258-2278); losses copied to host.
int ref_render_backward(void* h, int start, int len, double mask_coef, float huber,
                        double* losses_host)
{
    RefCtx* c = (RefCtx*)h;
    int rc = ensure_losses(c, len);
    if (rc) return rc;
    RenderUtils::renderRays_withGradients_RGB(c->opt, c->rays, c->scene, c->losses_dev,
                                              c->sample_index_dev, start, len, mask_coef, huber);
    if (losses_host)
        cudaMemcpy(losses_host, c->losses_dev, sizeof(double) * len, cudaMemcpyDeviceToHost);
    return fail(cudaGetLastError());
}

// RenderUtils::addVarianceLoss (RenderUtils.cu:2815-2851).
int ref_tv(void* h, double lam_d, double lam_sh, int type, int nbrs, int optimize_step)
{
    RefCtx* c = (RefCtx*)h;
    c->scene.optimizeStep = optimize_step;
    RenderUtils::addVarianceLoss(c->scene, c->opt, lam_d, lam_sh, type, nbrs);
    return fail(cudaGetLastError());
}

// Optimizer::updateRGBScene (Optimizer.cu:451-479).
int ref_adam(void* h, double lr, double sh_lr, int timestep)
{
    RefCtx* c = (RefCtx*)h;
    c->lr = lr;
    c->sh_lr = sh_lr;
    Optimizer::updateRGBScene(c->opt, c->scene, timestep);
    return fail(cudaGetLastError());
}

// One batch of the reference's training loop (Render.cu:407-500), losses read back
// to the host and reduced with getMSEError as the reference does.
int ref_train_step(void* h, int start, int len, double mask_coef, float huber, double lam_d,
                   double lam_sh, int tv_type, int nbrs, int do_tv, double lr, double sh_lr,
                   int timestep, double* losses_host, double* mse_out)
{
    RefCtx* c = (RefCtx*)h;
    int rc = ensure_losses(c, len);
    if (rc) return rc;
    RenderUtils::renderRays(c->rays, c->scene, c->sample_index_dev, start, len);
    RenderUtils::renderRays_withGradients_RGB(c->opt, c->rays, c->scene, c->losses_dev,
                                              c->sample_index_dev, start, len, mask_coef, huber);
    cudaMemcpy(losses_host, c->losses_dev, sizeof(double) * len, cudaMemcpyDeviceToHost);
    double loss = getMSEError(losses_host, len);
    if (mse_out) *mse_out = loss;
    if (do_tv) RenderUtils::addVarianceLoss(c->scene, c->opt, lam_d, lam_sh, tv_type, nbrs);
    c->lr = lr;
    c->sh_lr = sh_lr;
    Optimizer::updateRGBScene(c->opt, c->scene, timestep);
    return fail(cudaGetLastError());
}

static int copy_table(const std::vector<float*>& ptrs, int n_arrays, int64_t n, float* host,
                      bool to_device)
{
    for (int a = 0; a < n_arrays; a++) {
        if (!ptrs[a]) continue;
        if (to_device)
            cudaMemcpy(ptrs[a], host + (int64_t)a * n, sizeof(float) * n, cudaMemcpyHostToDevice);
        else
            cudaMemcpy(host + (int64_t)a * n, ptrs[a], sizeof(float) * n, cudaMemcpyDeviceToHost);
    }
    return fail(cudaDeviceSynchronize());
}

int64_t ref_n_active(void* h) { return ((RefCtx*)h)->scene.actualGridNums; }

// objectScene::initSelfByUpsample of the handle's scene into a dense target (SceneUtils.cu:487-517):
// the target's planar parameters [1 + 3 * its sh_dim][its vertices] to host memory.
int ref_upsample(void* h, float threshold, int low_band_only, int target_sh, float* planar_out)
{
    RefCtx* c = (RefCtx*)h;
    // The dense path of initSelfByUpsample (SceneUtils.cu:498-512) sizes the target by
    // lowBandOnly but hands the kernel src.sh_dim != targetSH_dim as its low-band flag: with
    // lowBandOnly set and targetSH_dim == src.sh_dim > 1 the kernel writes every coefficient
    // into a one-coefficient target, past its arrays.  That combination is refused here; the
    // reference's consistent low-band call is lowBandOnly with targetSH_dim = 1.
    if (low_band_only && target_sh == c->scene.sh_dim && target_sh > 1) return 1;
    if (target_sh < 1 || target_sh > c->scene.sh_dim) return 1;
    ObjectScene dst;
    dst.initSelfByUpsample(c->scene, threshold, low_band_only != 0, false, target_sh);
    int rc = fail(cudaDeviceSynchronize());
    const int na = 1 + 3 * dst.sh_dim;
    std::vector<float*> p(dst.totalVariableGPUPtrs, dst.totalVariableGPUPtrs + na);
    if (!rc) rc = copy_table(p, na, dst.actualGridNums, planar_out, false);
    dst.freeSelf();
    return rc;
}

// RenderUtils::bbox_silhouette (RenderUtils.cu:323-478) over ncam cameras given by their 3x4
// world-to-pixel matrices (12 doubles each) and images of 4 planes (r, g, b, mask) of
// img_w*img_h bytes: carving, then the bounding box into bbox_out[6] (wmin, wmax, hmin, hmax,
// dmin, dmax) and the returned scale ratio into scale_out.  Dense scenes.
int ref_bbox_silhouette(void* h, int ncam, const double* proj, const uint8_t* images, int img_w, int img_h,
                        int radius, int get_scale, int* bbox_out, double* scale_out)
{
    RefCtx* c = (RefCtx*)h;
    std::vector<Camera> cams(ncam);
    std::vector<Image> imgs(ncam);
    const size_t plane = (size_t)img_w * img_h;
    for (int i = 0; i < ncam; i++) {
        cudaMalloc((void**)&cams[i].projectionMatDevice, sizeof(double) * 12);
        cudaMemcpy(cams[i].projectionMatDevice, proj + 12 * i, sizeof(double) * 12, cudaMemcpyHostToDevice);
        Image& im = imgs[i];
        im.width = img_w;
        im.height = img_h;
        im.grayImage = false;
        uint8_t* planes[4];
        for (int p = 0; p < 4; p++) {
            cudaMalloc((void**)&planes[p], plane);
            cudaMemcpy(planes[p], images + ((size_t)i * 4 + p) * plane, plane, cudaMemcpyHostToDevice);
        }
        im.redDevice = planes[0];
        im.greenDevice = planes[1];
        im.blueDevice = planes[2];
        im.maskDevice = planes[3];
    }
    *scale_out = RenderUtils::bbox_silhouette(cams.data(), imgs.data(), &c->scene, ncam, radius, get_scale != 0,
                                              nullptr, 0);
    bbox_out[0] = c->scene.bbox_width_min;
    bbox_out[1] = c->scene.bbox_width_max;
    bbox_out[2] = c->scene.bbox_height_min;
    bbox_out[3] = c->scene.bbox_height_max;
    bbox_out[4] = c->scene.bbox_depth_min;
    bbox_out[5] = c->scene.bbox_depth_max;
    for (int i = 0; i < ncam; i++) {
        cudaFree(cams[i].projectionMatDevice);
        cudaFree(imgs[i].redDevice);
        cudaFree(imgs[i].greenDevice);
        cudaFree(imgs[i].blueDevice);
        cudaFree(imgs[i].maskDevice);
    }
    return fail(cudaDeviceSynchronize());
}

// objectScene::saveSelf (SceneUtils.cu:1246-1300) of the harness scene into `dir`.
int ref_save_text(void* h, const char* dir, int density_only, int band, int hierarchy_mode)
{
    RefCtx* c = (RefCtx*)h;
    ObjectScene& s = c->scene;
    if (s.sparse) {
        // the host copies of the sparse tables that initSelfByUpsample allocates
        // (SceneUtils.cu:542, 548) and copy2HostMemory fills before saving
        const size_t N = (size_t)s.sceneWidth * s.sceneHeight * s.sceneDepth;
        if (!s.inCageInfoHost) s.inCageInfoHost = (uchar*)calloc(N, sizeof(uchar));
        if (!s.indexOffsetsHost) s.indexOffsetsHost = (unsigned int*)malloc(sizeof(unsigned int) * N);
    }
    s.saveSelf(dir, density_only != 0, band, hierarchy_mode != 0);
    return fail(cudaDeviceSynchronize());
}

// objectScene::initFromFile (SceneUtils.cu:703-790) of a dense checkpoint in `dir` into a
// fresh scene, its planar parameters [1 + 3 target_sh][W*H*D] to host memory.
int ref_load_text(const char* dir, int W, int H, int D, float step, int sh_dim, int target_sh, float* planar_out)
{
    ObjectScene sc;
    sc.initFromFile(dir, W, H, D, false, step, sh_dim, target_sh, false, false);
    int rc = fail(cudaDeviceSynchronize());
    const int na = 1 + 3 * sc.sh_dim;
    std::vector<float*> p(sc.totalVariableGPUPtrs, sc.totalVariableGPUPtrs + na);
    if (!rc) rc = copy_table(p, na, sc.actualGridNums, planar_out, false);
    sc.freeSelf();
    return rc;
}

// Image::initSelfFromFile (ImageUtils.cu:84-128) of the colour image at `prefix` with its mask:
// planes r, g, b, mask (w*h bytes each) into planes_out, bbox[4], and the mask-area pixel list
// (masksIndex, up to w*h entries) with its length.
int ref_image_load_text(const char* prefix, int w, int h, uint8_t* planes_out, int* bbox_out, int* index_out,
                        int* n_out)
{
    Image im;
    im.initSelfFromFile(prefix, w, h, false, true);
    const size_t n = (size_t)w * h;
    std::memcpy(planes_out, im.redHost, n);
    std::memcpy(planes_out + n, im.greenHost, n);
    std::memcpy(planes_out + 2 * n, im.blueHost, n);
    std::memcpy(planes_out + 3 * n, im.maskHost, n);
    for (int i = 0; i < 4; i++) bbox_out[i] = im.bbox[i];
    *n_out = im.masksLen;
    std::memcpy(index_out, im.masksIndex, sizeof(int) * (size_t)im.masksLen);
    return fail(cudaDeviceSynchronize());
}

// The scene's density-LR multipliers (dense) to host memory.
int ref_adaptive_lr(void* h, float* out)
{
    RefCtx* c = (RefCtx*)h;
    const size_t n = (size_t)c->scene.sceneWidth * c->scene.sceneHeight * c->scene.sceneDepth;
    return fail(cudaMemcpy(out, c->scene.adaptiveLRDevice, sizeof(float) * n, cudaMemcpyDeviceToHost));
}

int ref_params(void* h, float* planar, int upload)
{
    RefCtx* c = (RefCtx*)h;
    std::vector<float*> p(c->param_ptrs_host, c->param_ptrs_host + c->n_arrays);
    return copy_table(p, c->n_arrays, c->scene.actualGridNums, planar, upload != 0);
}

int ref_grads(void* h, float* planar, int upload)
{
    RefCtx* c = (RefCtx*)h;
    return copy_table(c->grad_ptrs, c->n_arrays, c->scene.actualGridNums, planar, upload != 0);
}

int ref_moments(void* h, float* m, float* v, int upload)
{
    RefCtx* c = (RefCtx*)h;
    int rc = copy_table(c->m_ptrs, c->n_arrays, c->scene.actualGridNums, m, upload != 0);
    if (rc) return rc;
    return copy_table(c->v_ptrs, c->n_arrays, c->scene.actualGridNums, v, upload != 0);
}

void ref_destroy(void* h)
{
    RefCtx* c = (RefCtx*)h;
    if (!c) return;
    cudaDeviceSynchronize();
    if (c->have_rays) c->rays.freeSelf();
    if (c->have_opt) {
        for (int a = 0; a < c->n_arrays; a++) {
            cudaFree(c->grad_ptrs[a]);
            cudaFree(c->m_ptrs[a]);
            cudaFree(c->v_ptrs[a]);
        }
        cudaFree(c->opt.gradientDevice);
        cudaFree(c->opt.momentumDevice);
        cudaFree(c->opt.varianceDevice);
    }
    c->scene.freeSelf();
    cudaFree(c->sample_index_dev);
    cudaFree(c->losses_dev);
    delete c;
}

}  // extern "C"
