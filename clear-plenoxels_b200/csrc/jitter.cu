// jitter.cu -- per-sample jitter offsets on the device (SolidStrategy 0).
//
// The reference draws the offsets of every batch with objectScene::setSelfSampleOffset
// (SceneUtils.cu:792-798): for each axis, randGPU(offset, maxSamplePoint, stepSize / 2, 1)
// (Utils.cu:1002-1044) fills offset[k] = N(0,1) / 4 * radius from cuRAND's scrambled Sobol
// generator, where state i (of at most 20000) is dimension i of the JOEKUO6 64-bit
// direction numbers with scramble constant i, started at point i + rand().  This file calls
// the same cuRAND device functions (curand_init, curand_normal_double) in its own kernel,
// with the same direction numbers and constants fetched at run time from cuRAND's host API,
// so the offsets are the reference's bit for bit.  Reproduced as the reference does them:
//
//   * the scramble constants are 64-bit, but randGPU copies them into a 32-bit device array
//     (Utils.cu:1020-1023): state i gets the i-th 32-bit word of the 64-bit table;
//   * randGPU launches a square grid of 32x32 blocks, ((round(sqrt(len)) + 31) / 32)^2
//     blocks, which can cover fewer than len entries (len = 1050 -> 1024); the entries past
//     the grid keep their previous values (zero on a fresh grid);
//   * offset k uses state k % 20000; beyond 20000 entries the reference's threads share
//     states concurrently, here each state draws its entries one after another.
#include "cpx_internal.cuh"

#include <curand.h>
#include <curand_kernel.h>

#include <cmath>

namespace cpx {

constexpr int kSobolStates = 20000;  // randGPU's cap on generator states (Utils.cu:1013)

__global__ void k_sobol_normal(const curandDirectionVectors64_t* __restrict__ dirs,
                               const uint32_t* __restrict__ scramble, int n_states, unsigned long long first,
                               int n_write, double radius, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_states || i >= n_write) return;
    curandStateScrambledSobol64_t st;
    // initialize_generator (Utils.cu:934-947): offset = state index + the host's rand()
    curand_init(const_cast<unsigned long long*>(dirs[i]), (unsigned long long)scramble[i],
                (unsigned long long)i + first, &st);
    // normalDistribution (Utils.cu:963-976) with center 0
    for (int k = i; k < n_write; k += kSobolStates) out[k] = curand_normal_double(&st) / 4. * radius + 0.;
}

// objectScene::maxSamplePoint (SceneUtils.cu:96)
static int reference_max_sample_point(const cpx_grid* g)
{
    const int ss = g->W * g->W + g->H * g->H + g->D * g->D;
    return (int)(sqrt((double)ss) / g->step + 1.5);
}

static cpx_status ensure_sobol_tables(cpx_grid* g, int n_states)
{
    if (g->sobol_dirs && g->sobol_n == n_states) return CPX_OK;
    cudaFree(g->sobol_dirs);
    cudaFree(g->sobol_scramble);
    g->sobol_dirs = nullptr;
    g->sobol_scramble = nullptr;
    g->sobol_n = 0;
    curandDirectionVectors64_t* host_dirs = nullptr;
    unsigned long long* host_scramble = nullptr;
    if (curandGetDirectionVectors64(&host_dirs, CURAND_SCRAMBLED_DIRECTION_VECTORS_64_JOEKUO6) !=
            CURAND_STATUS_SUCCESS ||
        curandGetScrambleConstants64(&host_scramble) != CURAND_STATUS_SUCCESS) {
        set_error("cuRAND direction numbers or scramble constants unavailable");
        return CPX_ERR_CUDA;
    }
    cudaError_t e = cudaMalloc((void**)&g->sobol_dirs, (size_t)n_states * sizeof(curandDirectionVectors64_t));
    static_assert(sizeof(curandDirectionVectors64_t) == 64 * sizeof(unsigned long long), "64 direction words");
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->sobol_scramble, (size_t)n_states * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(g->sobol_dirs, host_dirs, (size_t)n_states * sizeof(curandDirectionVectors64_t),
                       cudaMemcpyHostToDevice);
    // the first n_states 32-bit words of the 64-bit table, as randGPU copies them
    if (e == cudaSuccess)
        e = cudaMemcpy(g->sobol_scramble, host_scramble, (size_t)n_states * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "sobol tables");
    g->sobol_n = n_states;
    return CPX_OK;
}

}  // namespace cpx

using namespace cpx;

extern "C" cpx_status cpx_grid_fill_sample_offsets(cpx_grid* g, float radius, const uint32_t* seeds,
                                                   cpx_stream stream)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (!g || !seeds || !(radius >= 0.f)) {
        set_error("fill_sample_offsets: null grid or seeds, or negative radius");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int len = reference_max_sample_point(g);
    if (len <= 0) {
        set_error("grid of no samples");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->n_off != len) {
        // the offset arrays of objectScene::initSelf: maxSamplePoint entries, zero at first
        for (int i = 0; i < 3; i++) {
            cudaFree(g->off[i]);
            g->off[i] = nullptr;
        }
        g->n_off = 0;
        for (int i = 0; i < 3; i++) {
            cudaError_t e = cudaMalloc((void**)&g->off[i], (size_t)len * sizeof(double));
            if (e == cudaSuccess) e = cudaMemset(g->off[i], 0, (size_t)len * sizeof(double));
            if (e != cudaSuccess) return cuda_status(e, "sample offsets");
        }
        g->n_off = len;
    }
    const int n_states = len < kSobolStates ? len : kSobolStates;
    cpx_status rc = ensure_sobol_tables(g, n_states);
    if (rc != CPX_OK) return rc;
    // entries randGPU's square grid of 32x32 blocks reaches (Utils.cu:1025-1027)
    const int square = (int)(sqrt(len * 1.0) + 0.5);
    const int64_t side = (square + 31) / 32;
    const int64_t reach = side * side * 1024;
    const int n_write = reach < len ? (int)reach : len;
    cudaStream_t st = (cudaStream_t)stream;
    const int threads = 256;
    const int blocks = (n_states + threads - 1) / threads;
    for (int a = 0; a < 3; a++) {
        k_sobol_normal<<<blocks, threads, 0, st>>>(reinterpret_cast<const curandDirectionVectors64_t*>(g->sobol_dirs),
                                                   g->sobol_scramble, n_states,
                                                   (unsigned long long)seeds[a], n_write, (double)radius,
                                                   g->off[a]);
        count_launch();
    }
    return cuda_status(cudaGetLastError(), "sample offsets");
}

extern "C" cpx_status cpx_grid_download_sample_offsets(const cpx_grid* g, double* ox, double* oy, double* oz,
                                                       int n)
{
    if (!g || n < 0 || n > g->n_off || (n > 0 && (!ox || !oy || !oz))) {
        set_error("download of %d offsets, the grid holds %d", n, g ? g->n_off : 0);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    double* dst[3] = {ox, oy, oz};
    cudaError_t e = cudaDeviceSynchronize();
    for (int a = 0; a < 3 && e == cudaSuccess && n > 0; a++)
        e = cudaMemcpy(dst[a], g->off[a], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    return cuda_status(e, "download sample offsets");
}
