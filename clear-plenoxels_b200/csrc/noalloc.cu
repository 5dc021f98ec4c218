// noalloc.cu -- the forward+backward march without any device allocation.
//
// cpx_render_forward_backward keeps its sample scratch in buffers the grid
// handle allocates (and grows) with cudaMalloc on first use.  Some callers
// cannot allow that: a host that hands every byte of device memory to its own
// pool allocator before training starts, or a latency-critical loop that is
// not allowed to allocate once it runs.  For them,
// cpx_render_forward_backward_noalloc runs the same two kernels with their
// scratch in the fixed array below, which the CUDA runtime places in device
// memory when the module is loaded.  It costs kNoAllocBytes (about 48 MiB) on
// every GPU that loads the library, for the life of the process, and caps a
// batch at kNoAllocRays rays and kNoAllocSamples sample slots (rays times the
// grid's per-ray sample bound).
//
// The array's name in host code is only a host-side stand-in for the device
// symbol, so host code never passes it to a kernel: the device address is
// looked up with cudaGetSymbolAddress once per device (on that device's first
// call) and cached.
#include "cpx_internal.cuh"

#include <mutex>

namespace cpx {

constexpr int kNoAllocRays = 16384;
constexpr int64_t kNoAllocSamples = int64_t(1) << 20;
constexpr size_t kSamplesBytes = (size_t)kNoAllocSamples * sizeof(SampleRec);
constexpr size_t kColoursBytes = (size_t)kNoAllocSamples * sizeof(float4);
constexpr size_t kCountsBytes = (size_t)kNoAllocRays * sizeof(int);
constexpr size_t kAccBytes = (size_t)kNoAllocRays * sizeof(double);
constexpr size_t kErrBytes = 256;
constexpr size_t kQueueBytes = ((size_t)kNoAllocRays + 4) * sizeof(int);  // the fused march's work queue
constexpr size_t kNoAllocBytes = kSamplesBytes + kColoursBytes + kCountsBytes + kAccBytes + kErrBytes + kQueueBytes;

// Shared by every call on a device: it keeps the last call's contents, and two calls that
// overlap on the GPU (different streams, or different host threads) race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mutex;

// Device address of the array on the current device (looked up once per device).
static cpx_status scratch_address(unsigned char** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "noalloc device");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device %d beyond the %d devices the fixed scratch supports", dev, kMaxDevices);
        return CPX_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "noalloc symbol");
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return CPX_OK;
}

}  // namespace cpx

using namespace cpx;

extern "C" cpx_status cpx_render_forward_backward_noalloc(cpx_grid* g, cpx_rays* r, double* losses_dev,
                                                          const int32_t* sample_index_dev, int start,
                                                          int len, double mask_coef, float huber_delta,
                                                          cpx_stream stream)
{
    if (!g || !r) {
        set_error("null handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int maxs = march_samples_per_ray(g);
    if (len > kNoAllocRays || (int64_t)len * maxs > kNoAllocSamples) {
        set_error("batch of %d rays x %d samples exceeds the fixed scratch (%d rays, %lld sample slots)",
                  len, maxs, kNoAllocRays, (long long)kNoAllocSamples);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (len <= 0) return len == 0 ? CPX_OK : CPX_ERR_INVALID_ARGUMENT;
    unsigned char* base = nullptr;
    cpx_status rc = scratch_address(&base);
    if (rc != CPX_OK) return rc;
    MarchScratch s;
    s.maxs = maxs;
    s.cap_rays = len;
    s.samples = reinterpret_cast<SampleRec*>(base);
    s.colours = reinterpret_cast<float4*>(base + kSamplesBytes);
    s.counts = reinterpret_cast<int*>(base + kSamplesBytes + kColoursBytes);
    s.acc = reinterpret_cast<double*>(base + kSamplesBytes + kColoursBytes + kCountsBytes);
    s.err = reinterpret_cast<int*>(base + kSamplesBytes + kColoursBytes + kCountsBytes + kAccBytes);
    s.queue = reinterpret_cast<int*>(base + kSamplesBytes + kColoursBytes + kCountsBytes + kAccBytes + kErrBytes);
    s.mse = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    // the flags must start at zero (the march zeroes its own queue); samples, colours, counts and
    // sums are written before use
    cudaError_t e = cudaMemsetAsync(s.err, 0, kErrBytes, st);
    if (e != cudaSuccess) return cuda_status(e, "noalloc flags");
    rc = march_launch_with(g, r, sample_index_dev, start, len, kForwardBackward, losses_dev, mask_coef,
                           huber_delta, s, st);
    if (rc != CPX_OK) return rc;
    // report this call's device-side checks (the flags live in the shared array)
    int flags[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(flags, s.err, sizeof(flags), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "noalloc");
    if (flags[0] & 2) {
        set_error("a sample index pointed outside the ray table");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (flags[0] & 1) {
        set_error("a ray's march exceeded its sample bound (near/far beyond the grid box?)");
        return CPX_ERR_ITERATION_CAP;
    }
    if (flags[0] & 8) {
        set_error("a shading warp of the fused march gave up waiting for a ray's placement");
        return CPX_ERR_NOT_READY;
    }
    if (flags[0] & 32) {
        set_error("a shading warp gave up waiting for a vertex record copy");
        return CPX_ERR_NOT_READY;
    }
    return CPX_OK;
}
