// api.cu -- the extern "C" entry points of libcpx (see include/cpx.h).
//
// Host-side logic only: argument checks, handle lifecycle, conversion between
// the reference's planar host layout and the record layout on the device, and
// the order of launches of one training batch (SVRF/Render.cu:407-500).
#include "cpx_internal.cuh"

#include <utility>

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>

namespace cpx {

static thread_local char g_last_error[512] = "";
static std::atomic<long long> g_launches{0};

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

cpx_status cuda_status(cudaError_t e, const char* where)
{
    if (e == cudaSuccess) return CPX_OK;
    set_error("%s: %s", where, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CPX_ERR_OUT_OF_MEMORY : CPX_ERR_CUDA;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Column e of a record array <-> a packed float array.
__global__ void k_set_column(float* aos, const float* col, int64_t n, int rec, int e,
                             float* density_out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = col[i];
    aos[i * rec + e] = v;
    if (density_out) density_out[i] = v;
}

__global__ void k_get_column(float* col, const float* aos, int64_t n, int rec, int e)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    col[i] = aos[i * rec + e];
}

// Column e of 16-bit records <-> a packed float array (round to nearest on the way in).
template <int PREC>
__global__ void k_set_column16(uint16_t* recs, const float* col, int64_t n, int slots, int e)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    recs[i * slots + e] = f_to_sh_rn<PREC>(col[i]);
}

template <int PREC>
__global__ void k_get_column16(float* col, const uint16_t* recs, int64_t n, int slots, int e)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    col[i] = sh_to_f<PREC>(recs[i * slots + e]);
}

// Moment column e of the half-moment form: m as m * 2^8, v through its root (sqrt(v) * 2^8),
// rounded to nearest and saturating as the sweep's stores do.
__global__ void k_set_moment16h(uint16_t* recs, const float* col, int64_t n, int slots, int e, int second)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = col[i];
    if (second) x = sqrtf(x > 0.f ? x : 0.f);
    x *= kMomScale;
    x = x > 65504.f ? 65504.f : (x < -65504.f ? -65504.f : x);
    recs[i * slots + e] = f_to_h16_rn(x);
}

__global__ void k_get_moment16h(float* col, const uint16_t* recs, int64_t n, int slots, int e, int second)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = h16_to_f(recs[i * slots + e]) * (1.f / kMomScale);
    col[i] = second ? x * x : x;
}

// Number of set bits of a word array (block reduction, one atomic per block).
__global__ void k_popcount(const uint32_t* __restrict__ w, int64_t n, unsigned long long* out)
{
    __shared__ unsigned int part;
    if (threadIdx.x == 0) part = 0;
    __syncthreads();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&part, (unsigned)__popc(w[i]));
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(out, (unsigned long long)part);
}

__global__ void k_fill(float* p, int64_t n, float v)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Packed ray records (9 words: 8 floats + rgba bytes) into the SoA ray table.
__global__ void k_unpack_rays(const uint32_t* __restrict__ src, int64_t count, int64_t offset,
                              RaysView rv)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t* w = src + i * 9;
    const int64_t ri = offset + i;
    const_cast<float*>(rv.ox)[ri] = __uint_as_float(w[0]);
    const_cast<float*>(rv.oy)[ri] = __uint_as_float(w[1]);
    const_cast<float*>(rv.oz)[ri] = __uint_as_float(w[2]);
    const_cast<float*>(rv.dx)[ri] = __uint_as_float(w[3]);
    const_cast<float*>(rv.dy)[ri] = __uint_as_float(w[4]);
    const_cast<float*>(rv.dz)[ri] = __uint_as_float(w[5]);
    const_cast<float*>(rv.near_t)[ri] = __uint_as_float(w[6]);
    const_cast<float*>(rv.far_t)[ri] = __uint_as_float(w[7]);
    const uint32_t gt = w[8];
    const_cast<uint8_t*>(rv.r)[ri] = (uint8_t)(gt & 0xff);
    const_cast<uint8_t*>(rv.g)[ri] = (uint8_t)((gt >> 8) & 0xff);
    const_cast<uint8_t*>(rv.b)[ri] = (uint8_t)((gt >> 16) & 0xff);
    const_cast<uint8_t*>(rv.mask)[ri] = (uint8_t)(gt >> 24);
}

static unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Which per-vertex state a planar column belongs to.
enum Field { kParams = 0, kGrads = 1, kMoment1 = 2, kMoment2 = 3 };

// Device column a (n floats) -> the grid's storage of `f`.
static void set_column(cpx_grid* g, Field f, const float* col, int64_t n, int a)
{
    const unsigned nb = blocks_for(n);
    if (f == kGrads) {
        k_set_column<<<nb, 256>>>(g->grad, col, n, g->rec, a, nullptr);
    } else if (g->prec == kPrecFP32) {
        float* dst = f == kParams ? g->params[g->cur] : (f == kMoment1 ? g->m : g->v);
        k_set_column<<<nb, 256>>>(dst, col, n, g->rec, a, (f == kParams && a == 0) ? g->density : nullptr);
        if (f == kParams && a == 0) {
            count_launch();
            refresh_dense_mirror(g, 0);
            return;
        }
    } else if (f == kParams && a == 0) {
        k_set_column<<<nb, 256>>>(g->dens[g->cur], col, n, 1, 0, nullptr);
        count_launch();
        refresh_dense_mirror(g, 0);
        return;
    } else if (f == kParams && g->prec == kPrecFP16) {
        k_set_column16<kPrecFP16><<<nb, 256>>>(g->sh16[g->cur], col, n, g->slots, a);
    } else if (g->mom_h) {
        k_set_moment16h<<<nb, 256>>>(f == kMoment1 ? g->m16 : g->v16, col, n, g->slots, a, f == kMoment2);
    } else {
        uint16_t* dst = f == kParams ? g->sh16[g->cur] : (f == kMoment1 ? g->m16 : g->v16);
        k_set_column16<kPrecBF16><<<nb, 256>>>(dst, col, n, g->slots, a);
    }
    count_launch();
}

// The grid's storage of `f`, column a -> device column (n floats).
static void get_column(const cpx_grid* g, Field f, float* col, int64_t n, int a)
{
    const unsigned nb = blocks_for(n);
    if (f == kGrads) {
        k_get_column<<<nb, 256>>>(col, g->grad, n, g->rec, a);
    } else if (g->prec == kPrecFP32) {
        const float* src = f == kParams ? g->params[g->cur] : (f == kMoment1 ? g->m : g->v);
        k_get_column<<<nb, 256>>>(col, src, n, g->rec, a);
    } else if (f == kParams && a == 0) {
        k_get_column<<<nb, 256>>>(col, g->dens[g->cur], n, 1, 0);
    } else if (f == kParams && g->prec == kPrecFP16) {
        k_get_column16<kPrecFP16><<<nb, 256>>>(col, g->sh16[g->cur], n, g->slots, a);
    } else if (g->mom_h) {
        k_get_moment16h<<<nb, 256>>>(col, f == kMoment1 ? g->m16 : g->v16, n, g->slots, a, f == kMoment2);
    } else {
        const uint16_t* src = f == kParams ? g->sh16[g->cur] : (f == kMoment1 ? g->m16 : g->v16);
        k_get_column16<kPrecBF16><<<nb, 256>>>(col, src, n, g->slots, a);
    }
    count_launch();
}

// Host planar [n_arrays][n] <-> device storage, one array at a time through a staging column.
static cpx_status planar_to_records(cpx_grid* g, Field f, const float* planar, int64_t n)
{
    if (n == 0) return CPX_OK;
    float* col = nullptr;
    cudaError_t e = cudaMalloc((void**)&col, n * sizeof(float));
    if (e != cudaSuccess) return cuda_status(e, "upload staging");
    for (int a = 0; a < g->n_arrays && e == cudaSuccess; a++) {
        e = cudaMemcpy(col, planar + (int64_t)a * n, n * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) break;
        set_column(g, f, col, n, a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(col);
    return cuda_status(e, "upload");
}

static cpx_status records_to_planar(const cpx_grid* g, Field f, float* planar, int64_t n)
{
    if (n == 0) return CPX_OK;
    float* col = nullptr;
    cudaError_t e = cudaMalloc((void**)&col, n * sizeof(float));
    if (e != cudaSuccess) return cuda_status(e, "download staging");
    for (int a = 0; a < g->n_arrays && e == cudaSuccess; a++) {
        get_column(g, f, col, n, a);
        e = cudaMemcpy(planar + (int64_t)a * n, col, n * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaFree(col);
    return cuda_status(e, "download");
}

static cpx_status check_grid(const cpx_grid* g)
{
    if (!g) {
        set_error("null grid handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return CPX_OK;
}

static cpx_status check_n(const cpx_grid* g, int64_t n)
{
    if (n != g->n_act) {
        set_error("array length %lld does not match the grid's %lld active vertices", (long long)n,
                  (long long)g->n_act);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return CPX_OK;
}

// Frees the per-vertex state (parameters, gradients, moments, density) and clears the pointers.
void free_state(cpx_grid* g)
{
    if (g->prec == kPrecFP32) cudaFree(g->density);  // the mixed forms alias dens[cur]
    g->density = nullptr;
    void** bufs[13] = {(void**)&g->params[0], (void**)&g->params[1], (void**)&g->grad, (void**)&g->m,
                       (void**)&g->v, (void**)&g->sh16[0], (void**)&g->sh16[1], (void**)&g->m16,
                       (void**)&g->v16, (void**)&g->dens[0], (void**)&g->dens[1],
                       (void**)&g->touched[0], (void**)&g->touched[1]};
    for (auto b : bufs) {
        cudaFree(*b);
        *b = nullptr;
    }
}

static void free_grid(cpx_grid* g)
{
    free_state(g);
    cudaFree(g->adaptive_lr);
    cudaFree(g->occ_bytes);
    cudaFree(g->occ_bits);
    cudaFree(g->in_cage);
    cudaFree(g->index_offsets);
    cudaFree(g->compact_to_dense);
    cudaFree(g->brick_bits);
    cudaFree(g->dense_mirror);
    cudaFree(g->dense_cells);
    cudaFree(g->dense_vbits);
    cudaFree(g->dense_bricks);
    for (int i = 0; i < 3; i++) cudaFree(g->off[i]);
    cudaFree(g->sobol_dirs);
    cudaFree(g->sobol_scramble);
    cudaFree(g->scratch.samples);
    cudaFree(g->scratch.colours);
    cudaFree(g->scratch.counts);
    cudaFree(g->scratch.acc);
    cudaFree(g->scratch.queue);
    cudaFree(g->scratch.err);
    cudaFree(g->scratch.mse);
    cudaFree(g->scratch2.samples);  // its error flags and MSE word are the first scratch's
    cudaFree(g->scratch2.colours);
    cudaFree(g->scratch2.counts);
    cudaFree(g->scratch2.acc);
    cudaFree(g->scratch2.queue);
    if (g->aside) cudaStreamDestroy(g->aside);
    if (g->ev_fork) cudaEventDestroy(g->ev_fork);
    if (g->ev_join) cudaEventDestroy(g->ev_join);
}

// Zeroed per-vertex state of `n` active vertices in the grid's storage form.
cudaError_t alloc_state(cpx_grid* g, int64_t n)
{
    const int64_t nn = n > 0 ? n : 1;
    const size_t rb = (size_t)nn * g->rec * sizeof(float);
    cudaError_t e = cudaSuccess;
    auto get = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    get((void**)&g->grad, rb);
    const size_t tb = (size_t)((nn + 31) / 32) * sizeof(uint32_t);
    get((void**)&g->touched[0], tb);
    get((void**)&g->touched[1], tb);
    g->tcur = 0;
    g->all_touched = 0;
    if (g->prec == kPrecFP32) {
        get((void**)&g->params[0], rb);
        get((void**)&g->params[1], rb);
        get((void**)&g->m, rb);
        get((void**)&g->v, rb);
        get((void**)&g->density, (size_t)nn * sizeof(float));
    } else {
        const size_t hb = (size_t)nn * g->slots * sizeof(uint16_t);
        // SH records with 16 bytes to spare: the shading's bulk copies move a record's 16-byte
        // aligned window, which for the last record reaches up to 8 bytes past it
        get((void**)&g->sh16[0], hb + 16);
        get((void**)&g->sh16[1], hb + 16);
        get((void**)&g->m16, hb);
        get((void**)&g->v16, hb);
        get((void**)&g->dens[0], (size_t)nn * sizeof(float));
        get((void**)&g->dens[1], (size_t)nn * sizeof(float));
        g->density = g->dens[g->cur];
    }
    return e;
}

}  // namespace cpx

using namespace cpx;

extern "C" {

const char* cpx_status_string(cpx_status s)
{
    switch (s) {
    case CPX_OK: return "ok";
    case CPX_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CPX_ERR_OUT_OF_MEMORY: return "out of memory";
    case CPX_ERR_CUDA: return "CUDA error";
    case CPX_ERR_ITERATION_CAP: return "march exceeded its sample bound";
    case CPX_ERR_NAN: return "NaN detected";
    case CPX_ERR_NOT_READY: return "not ready";
    case CPX_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

const char* cpx_last_error(void) { return g_last_error; }
int cpx_version(void) { return 100; }
int64_t cpx_kernel_launches(void) { return g_launches.load(); }

cpx_status cpx_grid_create(const cpx_grid_desc* d, cpx_grid** out)
{
    if (!d || !out) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (d->width < 2 || d->height < 2 || d->depth < 2) {
        set_error("grid needs at least 2 vertices per axis");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = (int64_t)d->width * d->height * d->depth;
    if (n >= (int64_t)1 << 31) {
        set_error("grid of %lld vertices exceeds the 32-bit index space", (long long)n);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (d->width > 65535 || d->height > 65535 || d->depth > 65535) {
        set_error("axis longer than 65535 vertices");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (d->sh_dim != 1 && d->sh_dim != 4 && d->sh_dim != 9) {
        set_error("sh_dim must be 1, 4 or 9 (got %d)", d->sh_dim);
        return CPX_ERR_UNSUPPORTED;
    }
    if (d->optimizing_band < 0 || (d->optimizing_band + 1) * (d->optimizing_band + 1) > d->sh_dim) {
        set_error("optimizing_band %d needs more than %d coefficients", d->optimizing_band, d->sh_dim);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!(d->step_size > 0.f) || !std::isfinite(d->step_size)) {
        set_error("step_size must be positive and finite");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (d->precision != CPX_PRECISION_FP32 && d->precision != CPX_PRECISION_BF16 &&
        d->precision != CPX_PRECISION_FP16 && d->precision != CPX_PRECISION_FP16_FULL) {
        set_error("unknown precision %d", d->precision);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cpx_grid* g = new (std::nothrow) cpx_grid();
    if (!g) return CPX_ERR_OUT_OF_MEMORY;
    g->W = d->width;
    g->H = d->height;
    g->D = d->depth;
    g->sh_dim = d->sh_dim;
    g->band = d->optimizing_band;
    g->hierarchy = d->hierarchy_strategy ? 1 : 0;
    g->optimize_step = 0;
    g->n_arrays = 1 + 3 * d->sh_dim;
    g->rec = (g->n_arrays + 3) & ~3;
    g->step = d->step_size;
    for (int i = 0; i < 6; i++) g->bbox[i] = d->bbox[i];
    g->n_dense = n;
    g->n_act = n;
    g->prec = d->precision == CPX_PRECISION_FP16_FULL ? kPrecFP16 : d->precision;
    g->mom_h = d->precision == CPX_PRECISION_FP16_FULL ? 1 : 0;
    g->sr_seed = d->sr_seed;
    g->slots = lowp_slots(g->n_arrays);
    cudaError_t e = alloc_state(g, n);
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->adaptive_lr, n * sizeof(float));
    // device error flags of the marches and sweeps
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->scratch.err, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMemset(g->scratch.err, 0, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->scratch.mse, sizeof(double));
    if (e == cudaSuccess) {
        k_fill<<<blocks_for(n), 256>>>(g->adaptive_lr, n, 1.f);
        count_launch();
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess && g->prec != kPrecFP32) lowp_prepare();
    if (e == cudaSuccess && refresh_dense_skip(g, 0) != CPX_OK) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_grid(g);
        delete g;
        set_error("grid of %lld vertices could not be allocated: %s", (long long)n,
                  cudaGetErrorString(e));
        return CPX_ERR_OUT_OF_MEMORY;
    }
    *out = g;
    return CPX_OK;
}

cpx_status cpx_grid_destroy(cpx_grid* g)
{
    if (!g) return CPX_OK;
    cudaDeviceSynchronize();
    free_grid(g);
    delete g;
    return CPX_OK;
}

cpx_status cpx_grid_info(const cpx_grid* g, int64_t* n_active, int* n_arrays, int* sparse)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    if (n_active) *n_active = g->n_act;
    if (n_arrays) *n_arrays = g->n_arrays;
    if (sparse) *sparse = g->sparse;
    return CPX_OK;
}

cpx_status cpx_grid_upload_params(cpx_grid* g, const float* planar, int64_t n)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g) || !planar) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    return planar_to_records(g, kParams, planar, n);
}

cpx_status cpx_grid_upload_params_device(cpx_grid* g, const float* planar_dev, int64_t n)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g) || !planar_dev) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    for (int a = 0; a < g->n_arrays; a++) set_column(g, kParams, planar_dev + (int64_t)a * n, n, a);
    return cuda_status(cudaDeviceSynchronize(), "device upload");
}

cpx_status cpx_grid_download_params(const cpx_grid* g, float* planar, int64_t n)
{
    if (check_grid(g) || !planar) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    cudaDeviceSynchronize();
    return records_to_planar(g, kParams, planar, n);
}

cpx_status cpx_grid_upload_grads(cpx_grid* g, const float* planar, int64_t n)
{
    if (check_grid(g) || !planar) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    g->all_touched = 1;  // gradients may be non-zero anywhere
    return planar_to_records(g, kGrads, planar, n);
}

cpx_status cpx_grid_download_grads(const cpx_grid* g, float* planar, int64_t n)
{
    if (check_grid(g) || !planar) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    cudaDeviceSynchronize();
    return records_to_planar(g, kGrads, planar, n);
}

cpx_status cpx_grid_upload_moments(cpx_grid* g, const float* m, const float* v, int64_t n)
{
    if (check_grid(g) || !m || !v) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    cpx_status s = planar_to_records(g, kMoment1, m, n);
    if (s != CPX_OK) return s;
    return planar_to_records(g, kMoment2, v, n);
}

cpx_status cpx_grid_download_moments(const cpx_grid* g, float* m, float* v, int64_t n)
{
    if (check_grid(g) || !m || !v) return CPX_ERR_INVALID_ARGUMENT;
    if (check_n(g, n)) return CPX_ERR_INVALID_ARGUMENT;
    cudaDeviceSynchronize();
    cpx_status s = records_to_planar(g, kMoment1, m, n);
    if (s != CPX_OK) return s;
    return records_to_planar(g, kMoment2, v, n);
}

cpx_status cpx_grid_set_adaptive_lr(cpx_grid* g, const float* lr_mult, int64_t n_dense)
{
    if (check_grid(g) || !lr_mult) return CPX_ERR_INVALID_ARGUMENT;
    if (n_dense != g->n_dense) {
        set_error("adaptive LR needs %lld entries", (long long)g->n_dense);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return cuda_status(cudaMemcpy(g->adaptive_lr, lr_mult, n_dense * sizeof(float),
                                  cudaMemcpyHostToDevice),
                       "adaptive lr");
}

cpx_status cpx_grid_set_sample_offsets(cpx_grid* g, const double* ox, const double* oy,
                                       const double* oz, int n)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g) || n < 0 || (n > 0 && (!ox || !oy || !oz))) return CPX_ERR_INVALID_ARGUMENT;
    cudaDeviceSynchronize();
    for (int i = 0; i < 3; i++) {
        cudaFree(g->off[i]);
        g->off[i] = nullptr;
    }
    g->n_off = 0;
    if (n == 0) return CPX_OK;
    const double* src[3] = {ox, oy, oz};
    for (int i = 0; i < 3; i++) {
        cudaError_t e = cudaMalloc((void**)&g->off[i], n * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(g->off[i], src[i], n * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_status(e, "sample offsets");
    }
    g->n_off = n;
    return CPX_OK;
}

cpx_status cpx_grid_set_options(cpx_grid* g, int options)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g) || (options & ~(CPX_OPT_NO_EMPTY_SKIP | CPX_OPT_FP32_MARCH | CPX_OPT_NO_EARLY_STOP | CPX_OPT_FUSED_MARCH |
                                   CPX_OPT_PLANE_SWEEP | CPX_OPT_SPLIT_SWEEP | CPX_OPT_SPARSE_ADAM)))
        return CPX_ERR_INVALID_ARGUMENT;
    g->options = options;
    cpx_status rc = refresh_dense_skip(g, 0);  // the maps of a grid now marched with jumps
    if (rc != CPX_OK) return rc;
    return cuda_status(cudaDeviceSynchronize(), "options");
}

cpx_status cpx_grid_set_optimize_step(cpx_grid* g, int optimize_step)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    g->optimize_step = optimize_step;
    return CPX_OK;
}

cpx_status cpx_occupancy_build(cpx_grid* g, float threshold, uint8_t* occupancy_out,
                               uint8_t* in_cage_out, uint32_t* index_offsets_out,
                               uint32_t* in_cage_count_out)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    if (g->sparse) {
        set_error("occupancy is built from a dense grid");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cudaDeviceSynchronize();
    cpx_status s = occupancy_launch(g, threshold);
    if (s != CPX_OK) return s;
    const int64_t C = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    cudaError_t e = cudaSuccess;
    if (occupancy_out) e = cudaMemcpy(occupancy_out, g->occ_bytes, C, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && in_cage_out)
        e = cudaMemcpy(in_cage_out, g->in_cage, g->n_dense, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && index_offsets_out)
        e = cudaMemcpy(index_offsets_out, g->index_offsets, g->n_dense * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost);
    if (in_cage_count_out) *in_cage_count_out = g->in_cage_count;
    return cuda_status(e, "occupancy download");
}

cpx_status cpx_grid_make_sparse(cpx_grid* g)
{
    if (g) ++g->epoch;  // what placement reads changes: a placement done in advance is stale
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    return make_sparse_launch(g);
}

cpx_status cpx_rays_create(int64_t n, int white_bg, cpx_rays** out)
{
    if (!out || n < 0) {
        set_error("invalid ray count");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    cpx_rays* r = new (std::nothrow) cpx_rays();
    if (!r) return CPX_ERR_OUT_OF_MEMORY;
    r->n = n;
    r->white_bg = white_bg ? 1 : 0;
    const int64_t nn = n > 0 ? n : 1;
    const size_t fbytes = (size_t)nn * sizeof(float);
    const size_t total = 13 * fbytes + 4 * (size_t)nn + 64;
    char* base = nullptr;
    cudaError_t e = cudaMalloc((void**)&base, total);
    if (e != cudaSuccess) {
        delete r;
        return cuda_status(e, "rays allocation");
    }
    cudaMemset(base, 0, total);
    r->block = base;
    float* f = reinterpret_cast<float*>(base);
    float** fields[13] = {&r->ox, &r->oy, &r->oz, &r->dx, &r->dy, &r->dz, &r->near_t, &r->far_t,
                          &r->acc_den, &r->acc_w, &r->acc_r, &r->acc_g, &r->acc_b};
    for (int i = 0; i < 13; i++) *fields[i] = f + (size_t)i * nn;
    uint8_t* u = reinterpret_cast<uint8_t*>(base + 13 * fbytes);
    r->mask = u;
    r->r = u + nn;
    r->g = u + 2 * nn;
    r->b = u + 3 * nn;
    *out = r;
    return CPX_OK;
}

cpx_status cpx_rays_destroy(cpx_rays* r)
{
    if (!r) return CPX_OK;
    cudaDeviceSynchronize();
    cudaFree(r->block);
    cudaFree(r->staging);
    delete r;
    return CPX_OK;
}

static bool range_ok(const cpx_rays* r, int64_t offset, int64_t count)
{
    if (!r || offset < 0 || count < 0 || offset + count > r->n) {
        set_error("ray range [%lld, %lld) outside the table", (long long)offset,
                  (long long)(offset + count));
        return false;
    }
    return true;
}

cpx_status cpx_rays_upload(cpx_rays* r, int64_t offset, int64_t count, const float* ox,
                           const float* oy, const float* oz, const float* dx, const float* dy,
                           const float* dz, const float* near_t, const float* far_t,
                           const uint8_t* gt_mask, const uint8_t* gt_r, const uint8_t* gt_g,
                           const uint8_t* gt_b, cpx_stream stream)
{
    if (r) ++r->epoch;  // the ray fields change: a placement done in advance is stale
    if (!range_ok(r, offset, count)) return CPX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    const float* fs[8] = {ox, oy, oz, dx, dy, dz, near_t, far_t};
    float* fd[8] = {r->ox, r->oy, r->oz, r->dx, r->dy, r->dz, r->near_t, r->far_t};
    const uint8_t* bs[4] = {gt_mask, gt_r, gt_g, gt_b};
    uint8_t* bd[4] = {r->mask, r->r, r->g, r->b};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 8 && e == cudaSuccess; i++)
        if (fs[i]) e = cudaMemcpyAsync(fd[i] + offset, fs[i], count * sizeof(float), cudaMemcpyHostToDevice, st);
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
        if (bs[i]) e = cudaMemcpyAsync(bd[i] + offset, bs[i], count, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return cuda_status(e, "rays upload");
}

cpx_status cpx_rays_upload_packed(cpx_rays* r, int64_t offset, int64_t count,
                                  const uint32_t* packed, cpx_stream stream)
{
    if (r) ++r->epoch;  // the ray fields change: a placement done in advance is stale
    if (!range_ok(r, offset, count) || (!packed && count > 0)) return CPX_ERR_INVALID_ARGUMENT;
    if (count == 0) return CPX_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (r->staging_cap < count) {
        cudaStreamSynchronize(st);
        cudaFree(r->staging);
        r->staging = nullptr;
        r->staging_cap = 0;
        cudaError_t e = cudaMalloc((void**)&r->staging, (size_t)count * 9 * sizeof(uint32_t));
        if (e != cudaSuccess) return cuda_status(e, "ray staging");
        r->staging_cap = count;
    }
    cudaError_t e = cudaMemcpyAsync(r->staging, packed, (size_t)count * 9 * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "packed upload");
    k_unpack_rays<<<blocks_for(count), 256, 0, st>>>(r->staging, count, offset, rays_view(r));
    count_launch();
    return cuda_status(cudaGetLastError(), "packed upload");
}

cpx_status cpx_rays_download(const cpx_rays* r, int64_t offset, int64_t count, float* ox,
                             float* oy, float* oz, float* dx, float* dy, float* dz,
                             float* near_t, float* far_t, uint8_t* gt_mask, uint8_t* gt_r,
                             uint8_t* gt_g, uint8_t* gt_b, float* acc_density,
                             float* acc_weights, float* acc_r, float* acc_g, float* acc_b)
{
    if (!range_ok(r, offset, count)) return CPX_ERR_INVALID_ARGUMENT;
    cudaDeviceSynchronize();
    float* fd[13] = {ox, oy, oz, dx, dy, dz, near_t, far_t, acc_density, acc_weights, acc_r, acc_g, acc_b};
    const float* fs[13] = {r->ox, r->oy, r->oz, r->dx, r->dy, r->dz, r->near_t, r->far_t,
                           r->acc_den, r->acc_w, r->acc_r, r->acc_g, r->acc_b};
    uint8_t* bd[4] = {gt_mask, gt_r, gt_g, gt_b};
    const uint8_t* bs[4] = {r->mask, r->r, r->g, r->b};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 13 && e == cudaSuccess; i++)
        if (fd[i]) e = cudaMemcpy(fd[i], fs[i] + offset, count * sizeof(float), cudaMemcpyDeviceToHost);
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
        if (bd[i]) e = cudaMemcpy(bd[i], bs[i] + offset, count, cudaMemcpyDeviceToHost);
    return cuda_status(e, "rays download");
}

cpx_status cpx_rays_init_camera(cpx_rays* r, const cpx_grid* g, const cpx_camera* cam,
                                int img_w, int img_h, const uint8_t* red, const uint8_t* green,
                                const uint8_t* blue, const uint8_t* gt_mask,
                                const int32_t* pixel_index, int64_t n_pix, int64_t offset)
{
    if (r) ++r->epoch;  // the ray fields change: a placement done in advance is stale
    if (check_grid(g) || !cam || !red || !green || !blue || (!pixel_index && n_pix > 0) ||
        img_w <= 0 || img_h <= 0)
        return CPX_ERR_INVALID_ARGUMENT;
    if (!range_ok(r, offset, n_pix)) return CPX_ERR_INVALID_ARGUMENT;
    const int64_t plane = (int64_t)img_w * img_h;
    for (int64_t i = 0; i < n_pix; i++) {
        if (pixel_index[i] < 0 || pixel_index[i] >= plane) {
            set_error("pixel index %d outside the %dx%d image", pixel_index[i], img_w, img_h);
            return CPX_ERR_INVALID_ARGUMENT;
        }
    }
    if (n_pix == 0) return CPX_OK;
    uint8_t* planes = nullptr;
    int32_t* pix = nullptr;
    cudaError_t e = cudaMalloc((void**)&planes, 4 * plane);
    if (e == cudaSuccess) e = cudaMalloc((void**)&pix, n_pix * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpy(planes, red, plane, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(planes + plane, green, plane, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(planes + 2 * plane, blue, plane, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && gt_mask) e = cudaMemcpy(planes + 3 * plane, gt_mask, plane, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pix, pixel_index, n_pix * sizeof(int32_t), cudaMemcpyHostToDevice);
    cpx_status s = cuda_status(e, "camera upload");
    if (s == CPX_OK)
        s = rays_camera_launch(r, g, cam, img_w, plane, planes, pix, n_pix, offset, gt_mask != nullptr,
                               nullptr);
    if (s == CPX_OK) s = cuda_status(cudaDeviceSynchronize(), "rays");
    cudaFree(planes);
    cudaFree(pix);
    return s;
}

cpx_status cpx_render_forward(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                              cpx_stream stream)
{
    if (check_grid(g) || !r) return CPX_ERR_INVALID_ARGUMENT;
    return march_launch(g, r, sidx, start, len, kForward, nullptr, 0., 0.f, (cudaStream_t)stream);
}

cpx_status cpx_render_backward(cpx_grid* g, cpx_rays* r, double* losses, const int32_t* sidx,
                               int start, int len, double mask_coef, float huber,
                               cpx_stream stream)
{
    if (check_grid(g) || !r) return CPX_ERR_INVALID_ARGUMENT;
    return march_launch(g, r, sidx, start, len, kBackward, losses, mask_coef, huber,
                        (cudaStream_t)stream);
}

cpx_status cpx_render_forward_backward(cpx_grid* g, cpx_rays* r, double* losses,
                                       const int32_t* sidx, int start, int len,
                                       double mask_coef, float huber, cpx_stream stream)
{
    if (check_grid(g) || !r) return CPX_ERR_INVALID_ARGUMENT;
    return march_launch(g, r, sidx, start, len, kForwardBackward, losses, mask_coef, huber,
                        (cudaStream_t)stream);
}

cpx_status cpx_tv_grad(cpx_grid* g, double lam_d, double lam_sh, int type, int nbrs,
                       cpx_stream stream)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    return tv_launch(g, lam_d, lam_sh, type, nbrs, (cudaStream_t)stream);
}

cpx_status cpx_adam_step(cpx_grid* g, double lr, double sh_lr, int timestep, cpx_stream stream)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    if (timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return sweep_adam(g, false, 0., 0., lr, sh_lr, timestep, (cudaStream_t)stream);
}

cpx_status cpx_tv_adam_step(cpx_grid* g, double lam_d, double lam_sh, double lr, double sh_lr,
                            int timestep, cpx_stream stream)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    if (timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse && !g->have_occupancy) {
        set_error("sparse grid without occupancy");
        return CPX_ERR_NOT_READY;
    }
    return sweep_adam(g, true, lam_d, lam_sh, lr, sh_lr, timestep, (cudaStream_t)stream);
}

// The step of CPX_OPT_SPLIT_SWEEP: placement; then, on the grid's second stream, the touched
// map from the placed samples and the sweep of the untouched vertices, beside the shading on
// the caller's stream; then the sweep of the touched vertices once both are done.  The
// untouched vertices' update reads nothing the shading writes (their gradients are zero and
// not read) and writes nothing it reads (the other parameter buffer, the moments, the density
// mirror that only placement reads), so the two run side by side.
static cpx_status train_step_split(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                                   const cpx_step_args* a, double* losses, double* mse_out, cudaStream_t st)
{
    g->last_len = len;
    cpx_status s = march_launch_stages(g, r, sidx, start, len, losses, a->mask_coef, a->huber_delta, 0, 1, st);
    if (s != CPX_OK) return s;
    cudaError_t e = cudaSuccess;
    if (!g->aside) e = cudaStreamCreateWithFlags(&g->aside, cudaStreamNonBlocking);
    if (e == cudaSuccess && !g->ev_fork) e = cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess && !g->ev_join) e = cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(g->ev_fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->aside, g->ev_fork, 0);
    if (e != cudaSuccess) return cuda_status(e, "split sweep stream");
    s = mark_touched(g, len, g->aside);
    if (s == CPX_OK)
        s = sweep_adam_pass(g, true, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, 1, g->aside);
    e = cudaEventRecord(g->ev_join, g->aside);  // recorded on every path: the caller's stream joins it
    if (s != CPX_OK) return s;
    if (e != cudaSuccess) return cuda_status(e, "split sweep join");
    s = march_launch_stages(g, r, sidx, start, len, losses, a->mask_coef, a->huber_delta, 0, 2, st);
    e = cudaStreamWaitEvent(st, g->ev_join, 0);
    if (s != CPX_OK) return s;
    if (e != cudaSuccess) return cuda_status(e, "split sweep join");
    s = sweep_adam_pass(g, true, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, 2, st);
    if (s != CPX_OK) return s;
    if (mse_out) {
        s = mse_launch(losses, len, g->scratch.mse, st);
        if (s != CPX_OK) return s;
        e = cudaMemcpyAsync(mse_out, g->scratch.mse, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e, "mse");
    }
    return CPX_OK;
}

cpx_status cpx_train_step(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                          const cpx_step_args* a, double* losses, double* mse_out,
                          cpx_stream stream)
{
    if (check_grid(g) || !r || !a) return CPX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    const bool fuse = a->do_tv && a->tv_type == 0 && a->tv_neighbours == 6;
    if (a->do_tv && !fuse && g->prec != kPrecFP32) {
        set_error("the mixed forms run TV type 0 / 6 neighbours fused into the optimizer sweep only");
        return CPX_ERR_UNSUPPORTED;
    }
    const bool split = (g->options & CPX_OPT_SPLIT_SWEEP) && fuse && g->prec == kPrecFP32 && !g->sparse &&
                       g->rec == 28 && !g->all_touched && len > 0 && a->timestep >= 1 &&
                       !(g->options & (CPX_OPT_FUSED_MARCH | CPX_OPT_FP32_MARCH | CPX_OPT_PLANE_SWEEP));
    if (split) return train_step_split(g, r, sidx, start, len, a, losses, mse_out, st);
    cpx_status s = march_launch(g, r, sidx, start, len, kForwardBackward, losses, a->mask_coef,
                                a->huber_delta, st);
    if (s != CPX_OK) return s;
    if (a->do_tv && !fuse) {
        s = tv_launch(g, a->lam_density, a->lam_sh, a->tv_type, a->tv_neighbours, st);
        if (s != CPX_OK) return s;
    }
    if (a->timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    s = sweep_adam(g, fuse, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, st);
    if (s != CPX_OK) return s;
    if (mse_out) {
        s = mse_launch(losses, len, g->scratch.mse, st);
        if (s != CPX_OK) return s;
        cudaError_t e = cudaMemcpyAsync(mse_out, g->scratch.mse, sizeof(double),
                                        cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e, "mse");
    }
    return CPX_OK;
}

cpx_status cpx_train_step_ahead(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                                cpx_rays* next_r, const int32_t* next_sidx, int next_start, int next_len,
                                const cpx_step_args* a, double* losses, double* mse_out, cpx_stream stream)
{
    if (check_grid(g) || !r || !a) return CPX_ERR_INVALID_ARGUMENT;
    if (a->timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const bool fuse = a->do_tv && a->tv_type == 0 && a->tv_neighbours == 6;
    const bool ahead_ok = g->prec == kPrecFP32 && !g->sparse && g->rec == 28 && (fuse || !a->do_tv) &&
                          !(g->options & (CPX_OPT_FUSED_MARCH | CPX_OPT_FP32_MARCH)) && next_r && next_len > 0 &&
                          len > 0;
    if (!ahead_ok) {  // the plain step: nothing is placed in advance
        g->ahead.valid = 0;
        return cpx_train_step(g, r, sidx, start, len, a, losses, mse_out, stream);
    }
    cudaStream_t st = (cudaStream_t)stream;
    // this batch: only its shading when the last step placed it on the current densities
    const bool placed = g->ahead.valid && g->ahead.r == r && g->ahead.rays_epoch == r->epoch && g->ahead.sidx == sidx &&
                        g->ahead.start == start && g->ahead.len == len && g->ahead.epoch == g->epoch;
    g->ahead.valid = 0;
    if (placed) std::swap(g->scratch, g->scratch2);  // the placed batch becomes the grid's own scratch
    g->last_len = len;
    cpx_status s = march_launch_stages(g, r, sidx, start, len, losses, a->mask_coef, a->huber_delta, 0,
                                       placed ? 2 : 3, st);
    if (s != CPX_OK) return s;
    // the densities the sweep will write, then the next batch's placement on them beside the sweep
    s = density_preview(g, fuse, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, st);
    if (s != CPX_OK) return s;
    cudaError_t e = cudaSuccess;
    if (!g->aside) e = cudaStreamCreateWithFlags(&g->aside, cudaStreamNonBlocking);
    if (e == cudaSuccess && !g->ev_fork) e = cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess && !g->ev_join) e = cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(g->ev_fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->aside, g->ev_fork, 0);
    if (e != cudaSuccess) return cuda_status(e, "look-ahead stream");
    s = march_launch_stages(g, next_r, next_sidx, next_start, next_len, losses, a->mask_coef, a->huber_delta, 1, 1,
                            g->aside);
    if (s != CPX_OK) return s;
    e = cudaEventRecord(g->ev_join, g->aside);
    if (e != cudaSuccess) return cuda_status(e, "look-ahead join");
    s = sweep_adam(g, fuse, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, st);
    if (s != CPX_OK) return s;
    e = cudaStreamWaitEvent(st, g->ev_join, 0);  // work after this step sees the placement done
    if (e != cudaSuccess) return cuda_status(e, "look-ahead join");
    g->ahead.valid = 1;
    g->ahead.r = next_r;
    g->ahead.rays_epoch = next_r->epoch;
    g->ahead.sidx = next_sidx;
    g->ahead.start = next_start;
    g->ahead.len = next_len;
    g->ahead.epoch = g->epoch;
    if (mse_out) {
        s = mse_launch(losses, len, g->scratch.mse, st);
        if (s != CPX_OK) return s;
        e = cudaMemcpyAsync(mse_out, g->scratch.mse, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e, "mse");
    }
    return CPX_OK;
}

cpx_status cpx_render_forward_guided(cpx_grid* g, cpx_rays* r, const int32_t* sidx, int start, int len,
                                     const uint32_t* masks, cpx_stream stream)
{
    if (check_grid(g) || !r) return CPX_ERR_INVALID_ARGUMENT;
    return march_launch_guided(g, r, sidx, start, len, nullptr, 0., 0.f, masks, nullptr, (cudaStream_t)stream,
                               kForward);
}

cpx_status cpx_render_forward_backward_guided(cpx_grid* g, cpx_rays* r, double* losses, const int32_t* sidx,
                                              int start, int len, double mask_coef, float huber,
                                              const uint32_t* masks, float* seg_w, cpx_stream stream)
{
    if (check_grid(g) || !r) return CPX_ERR_INVALID_ARGUMENT;
    return march_launch_guided(g, r, sidx, start, len, losses, mask_coef, huber, masks, seg_w, (cudaStream_t)stream);
}

// Finishes a batch after its march: TV + Adam sweep and the optional batch MSE.
static cpx_status finish_step(cpx_grid* g, const cpx_step_args* a, double* losses, int len, double* mse_out,
                              cudaStream_t st)
{
    if (a->timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const bool fuse = a->do_tv && a->tv_type == 0 && a->tv_neighbours == 6;
    cpx_status s = sweep_adam(g, fuse, a->lam_density, a->lam_sh, a->lr, a->sh_lr, a->timestep, st);
    if (s != CPX_OK || !mse_out) return s;
    s = mse_launch(losses, len, g->scratch.mse, st);
    if (s != CPX_OK) return s;
    cudaError_t e = cudaMemcpyAsync(mse_out, g->scratch.mse, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return cuda_status(e, "mse");
}

cpx_status cpx_train_step_proposal(cpx_grid* g, cpx_rays* r, cpx_proposal* p, const int32_t* sidx, int start,
                                   int len, const cpx_step_args* a, const cpx_proposal_schedule* sch, int iteration,
                                   double* losses, double* mse_out, cpx_stream stream)
{
    if (check_grid(g) || !r || !p || !a || !sch) return CPX_ERR_INVALID_ARGUMENT;
    if (g->prec == kPrecFP32) {
        set_error("the proposal form runs on the mixed-precision grid forms");
        return CPX_ERR_UNSUPPORTED;
    }
    if (a->do_tv && !(a->tv_type == 0 && a->tv_neighbours == 6)) {
        set_error("the mixed forms run TV type 0 / 6 neighbours fused into the optimizer sweep only");
        return CPX_ERR_UNSUPPORTED;
    }
    if (sch->train_every < 1 || sch->train_steps < 0 || iteration < 0) {
        set_error("invalid proposal schedule");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const bool label = iteration < sch->warmup || iteration % sch->train_every == 0;
    cpx_status s;
    if (label) {
        // full march recording the segment weights, then a training round on them
        float* seg_w = proposal_label_buffer(p, len);
        if (!seg_w) {
            set_error("proposal labels could not be allocated");
            return CPX_ERR_OUT_OF_MEMORY;
        }
        s = march_launch_guided(g, r, sidx, start, len, losses, a->mask_coef, a->huber_delta, nullptr, seg_w, st);
        if (s != CPX_OK) return s;
        const bool train = iteration % sch->train_every == 0 || iteration + 1 == sch->warmup;
        if (train && sch->train_steps > 0) {
            s = proposal_train(p, g, r, sidx, start, len, seg_w, sch->train_steps, sch->rays_per_step, true, st);
            if (s != CPX_OK) return s;
        }
    } else {
        uint32_t* masks = nullptr;
        s = proposal_masks(p, g, r, sidx, start, len, st, &masks);
        if (s != CPX_OK) return s;
        s = march_launch_guided(g, r, sidx, start, len, losses, a->mask_coef, a->huber_delta, masks, nullptr, st);
        if (s != CPX_OK) return s;
    }
    return finish_step(g, a, losses, len, mse_out, st);
}

cpx_status cpx_grid_touched_count(cpx_grid* g, int64_t* count)
{
    if (check_grid(g) || !count) return CPX_ERR_INVALID_ARGUMENT;
    if (g->all_touched) {
        *count = g->n_act;
        return CPX_OK;
    }
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_status(e, "touched count");
    cudaMemset(d, 0, sizeof(unsigned long long));
    const int64_t words = (g->n_act + 31) / 32;
    k_popcount<<<blocks_for(words), 256>>>(g->touched[g->tcur], words, d);
    count_launch();
    unsigned long long v = 0;
    e = cudaMemcpy(&v, d, sizeof(v), cudaMemcpyDeviceToHost);
    cudaFree(d);
    *count = (int64_t)v;
    return cuda_status(e, "touched count");
}

cpx_status cpx_grid_download_cell_map(cpx_grid* g, uint32_t* words, int64_t n_words)
{
    if (check_grid(g) || !words) return CPX_ERR_INVALID_ARGUMENT;
    if (!dense_skip_on(g)) {
        set_error("this grid's march keeps no dense empty-space map");
        return CPX_ERR_UNSUPPORTED;
    }
    const int64_t cells = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    const int64_t need = (cells + 31) / 32;
    if (n_words < need) {
        set_error("the map needs %lld words, %lld given", (long long)need, (long long)n_words);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!g->dense_cells) {
        set_error("no density uploaded yet");
        return CPX_ERR_NOT_READY;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(words, g->dense_cells, need * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    return cuda_status(e, "cell map download");
}

cpx_status cpx_grid_check(cpx_grid* g)
{
    if (check_grid(g)) return CPX_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "check");
    if (!g->scratch.err) return CPX_OK;
    int flags[4] = {0, 0, 0, 0};
    e = cudaMemcpy(flags, g->scratch.err, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "check");
    cudaMemset(g->scratch.err, 0, sizeof(flags));
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

cpx_status cpx_last_sample_counts(const cpx_grid* g, int32_t* counts_host, int len)
{
    if (check_grid(g) || !counts_host || len < 0 || len > g->last_len) {
        set_error("counts of %d rays requested, last batch had %d", len, g ? g->last_len : 0);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (len == 0) return CPX_OK;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(counts_host, g->scratch.counts, len * sizeof(int32_t), cudaMemcpyDeviceToHost);
    for (int i = 0; i < len; i++)
        if (counts_host[i] < 0) counts_host[i] = 0;
    return cuda_status(e, "counts");
}

}  // extern "C"
