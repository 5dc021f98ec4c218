// occupancy.cu -- occupancy, in-cage flags, compact index table and compaction.
//
// The reference builds these with a kernel per (x,y) column (pruneScene,
// SceneUtils.cu:831-881) followed by a host loop over every vertex for the
// compact index (getCagedNums, SceneUtils.cu:1081-1120) and a host compaction
// of the parameters (SceneUtils.cu:585-602).  Here all three run on the
// device: a thread per cell sets the occupancy byte/bit and the in-cage flags,
// a three-phase prefix scan turns the flags into the index table, and a
// thread per vertex moves in-cage records to their compact slots.  The index
// lists are identical to the reference's, including its quirks: the flag for
// the x = W-1 face is written at depth*W*H + H*W + col + 1 (SceneUtils.cu:872),
// i.e. at vertex (W-1, 0, depth+1) -- always inside the array since depth <= D-2
// -- and non-caged vertices get index 0.
#include "cpx_internal.cuh"

namespace cpx {

__device__ __forceinline__ int64_t grid_index_upper(int x, int y, int z, int W, int H, int D)
{
    x = x < W ? x : W - 1;
    y = y < H ? y : H - 1;
    z = z < D ? z : D - 1;
    return (int64_t)z * W * H + (int64_t)y * W + x;
}

// occupiedVoxel + pruneScene; one thread per cell, cells in z-y-x order.  With occ_in set the
// cells' occupancy is given (a loaded occupancy.txt) and only the in-cage rule runs.
__global__ void k_prune(const float* __restrict__ dens, const uint8_t* __restrict__ occ_in, int W, int H, int D,
                        float thr, uint8_t* occ, uint32_t* occ_bits, uint8_t* in_cage, int64_t n_cells,
                        unsigned long long* dropped)
{
    const int64_t ci = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int Wc = W - 1, Hc = H - 1;
    bool occupied = false;
    if (ci < n_cells) {
        const int x = (int)(ci % Wc);
        const int y = (int)((ci / Wc) % Hc);
        const int z = (int)(ci / ((int64_t)Wc * Hc));
        if (occ_in) {
            occupied = occ_in[ci] != 0;
        } else {
            for (int dz = 0; dz <= 1 && !occupied; dz++)
                for (int dy = 0; dy <= 1 && !occupied; dy++)
                    for (int dx = 0; dx <= 1 && !occupied; dx++)
                        if (dens[grid_index_upper(x + dx, y + dy, z + dz, W, H, D)] > thr) occupied = true;
        }
        occ[ci] = occupied ? 1 : 0;
        if (occupied) {
            const int64_t N = (int64_t)W * H * D;
            in_cage[(int64_t)z * W * H + (int64_t)y * W + x] = 1;
            if (z == D - 2) in_cage[(int64_t)(D - 1) * W * H + (int64_t)y * W + x] = 1;
            if (y == H - 2) in_cage[(int64_t)z * W * H + (int64_t)(H - 1) * W + x] = 1;
            if (x == W - 2) {
                const int64_t v = (int64_t)z * W * H + (int64_t)H * W + x + 1;
                if (v < N)
                    in_cage[v] = 1;
                else
                    atomicAdd(dropped, 1ull);
            }
        }
    }
    // one occupancy bit per cell: the warp covers 32 consecutive cells
    const unsigned bits = __ballot_sync(0xffffffffu, occupied);
    if ((threadIdx.x & 31) == 0) {
        const int64_t word = ci >> 5;
        if (word * 32 < n_cells) occ_bits[word] = bits;
    }
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
        uint32_t si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += u;
        }
        warp_sums[lane] = si - s;
        if (lane == 31) *total = si;
    }
    __syncthreads();
    return warp_sums[wid] + inc - v;
}

// Phase 1: in-cage count of each tile.
__global__ void __launch_bounds__(kScanThreads) k_scan_count(const uint8_t* flags, int64_t n,
                                                              uint32_t* tile_sums)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t total;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) c += flags[base + k] ? 1u : 0u;
    block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Phase 2: exclusive scan of the tile counts (single block, loops over chunks).
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(uint32_t* tile_sums, int n_tiles,
                                                              uint32_t* grand_total)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t total;
    uint32_t carry = 0;
    for (int base = 0; base < n_tiles; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < n_tiles ? tile_sums[i] : 0u;
        const uint32_t ex = block_exclusive_scan(v, ws, &total);
        if (i < n_tiles) tile_sums[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *grand_total = carry;
}

// Phase 3: index table (getCagedNums: running count for caged vertices, 0 otherwise).
__global__ void __launch_bounds__(kScanThreads) k_scan_write(const uint8_t* flags, int64_t n,
                                                              const uint32_t* tile_offsets,
                                                              uint32_t* index_offsets)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t total;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t f[kScanItems];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        f[k] = (base + k < n && flags[base + k]) ? 1u : 0u;
        c += f[k];
    }
    uint32_t run = tile_offsets[blockIdx.x] + block_exclusive_scan(c, ws, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) index_offsets[base + k] = f[k] ? run : 0u;
        run += f[k];
    }
}

// Brick occupancy: bit k of the brick map is set when any cell of 8x8x8 brick k is occupied.
// Thread per brick; a warp's 32 consecutive bricks form one word.
constexpr int kBrick = 8;

__global__ void k_bricks(const uint32_t* __restrict__ occ_bits, int cw, int ch, int cd, int bx, int by, int bz,
                         uint32_t* brick_bits)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nb = (int64_t)bx * by * bz;
    bool any = false;
    if (k < nb) {
        const int x0 = (int)(k % bx) * kBrick, y0 = (int)((k / bx) % by) * kBrick;
        const int z0 = (int)(k / ((int64_t)bx * by)) * kBrick;
        for (int z = z0; z < min(z0 + kBrick, cd) && !any; z++)
            for (int y = y0; y < min(y0 + kBrick, ch) && !any; y++)
                for (int x = x0; x < min(x0 + kBrick, cw) && !any; x++) {
                    const int64_t c = ((int64_t)z * ch + y) * cw + x;
                    any = (occ_bits[c >> 5] >> (c & 31)) & 1u;
                }
    }
    const unsigned word = __ballot_sync(0xffffffffu, any);
    if ((threadIdx.x & 31) == 0 && k < nb) brick_bits[k >> 5] = word;
}

cpx_status occupancy_launch(cpx_grid* g, float threshold) { return occupancy_build(g, threshold, nullptr); }

cpx_status occupancy_build(cpx_grid* g, float threshold, const uint8_t* occ_in_dev)
{
    const int64_t N = g->n_dense;
    const int64_t C = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    if (g->W < 2 || g->H < 2 || g->D < 2) {
        set_error("occupancy needs at least 2 vertices per axis");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!g->occ_bytes) {
        const int64_t words = (C + 31) / 32;
        if (cudaMalloc((void**)&g->occ_bytes, C) != cudaSuccess ||
            cudaMalloc((void**)&g->occ_bits, (words + 1) * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc((void**)&g->in_cage, N) != cudaSuccess ||
            cudaMalloc((void**)&g->index_offsets, N * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            set_error("occupancy tables could not be allocated");
            return CPX_ERR_OUT_OF_MEMORY;
        }
    }
    const int n_tiles = (int)((N + kScanTile - 1) / kScanTile);
    uint32_t* tile_sums = nullptr;
    unsigned long long* dropped = nullptr;
    uint32_t* total = nullptr;
    if (cudaMalloc((void**)&tile_sums, (size_t)n_tiles * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc((void**)&dropped, sizeof(unsigned long long) + sizeof(uint32_t) * 2) !=
            cudaSuccess) {
        cudaGetLastError();
        cudaFree(tile_sums);
        set_error("occupancy scratch could not be allocated");
        return CPX_ERR_OUT_OF_MEMORY;
    }
    total = reinterpret_cast<uint32_t*>(dropped + 1);
    cudaMemset(dropped, 0, sizeof(unsigned long long) + sizeof(uint32_t) * 2);
    cudaMemset(g->in_cage, 0, N);
    const int64_t words = (C + 31) / 32;
    cudaMemset(g->occ_bits, 0, (words + 1) * sizeof(uint32_t));
    const int64_t prune_threads = words * 32;
    k_prune<<<(unsigned)((prune_threads + 255) / 256), 256>>>(g->density, occ_in_dev, g->W, g->H, g->D,
                                                               threshold, g->occ_bytes,
                                                               g->occ_bits, g->in_cage, C,
                                                               dropped);
    {
        const int cw = g->W - 1, ch = g->H - 1, cd = g->D - 1;
        const int bx = (cw + kBrick - 1) / kBrick, by = (ch + kBrick - 1) / kBrick, bz = (cd + kBrick - 1) / kBrick;
        const int64_t nb = (int64_t)bx * by * bz;
        if (!g->brick_bits && cudaMalloc((void**)&g->brick_bits, ((nb + 31) / 32) * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(tile_sums);
            cudaFree(dropped);
            set_error("brick map could not be allocated");
            return CPX_ERR_OUT_OF_MEMORY;
        }
        g->bricks[0] = bx;
        g->bricks[1] = by;
        g->bricks[2] = bz;
        // whole warps: the warp that writes the last word has no brick in its tail threads
        k_bricks<<<(unsigned)((nb + 255) / 256), 256>>>(g->occ_bits, cw, ch, cd, bx, by, bz, g->brick_bits);
        count_launch();
    }
    k_scan_count<<<n_tiles, kScanThreads>>>(g->in_cage, N, tile_sums);
    k_scan_tiles<<<1, kScanThreads>>>(tile_sums, n_tiles, total);
    k_scan_write<<<n_tiles, kScanThreads>>>(g->in_cage, N, tile_sums, g->index_offsets);
    count_launch(4);
    uint32_t cnt = 0;
    cudaError_t e = cudaMemcpy(&cnt, total, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(tile_sums);
    cudaFree(dropped);
    if (e != cudaSuccess) return cuda_status(e, "occupancy");
    g->in_cage_count = cnt;
    g->have_occupancy = 1;
    return cuda_status(cudaGetLastError(), "occupancy");
}

// Move in-cage records to their compact slots (SceneUtils.cu:585-602).
__global__ void k_compact(const float4* __restrict__ src, float4* dst, float* dens_out,
                          const uint8_t* __restrict__ in_cage,
                          const uint32_t* __restrict__ index_offsets, uint32_t* c2d, int64_t N,
                          int S)
{
    const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= N || !in_cage[v]) return;
    const uint32_t c = index_offsets[v];
    for (int j = 0; j < S; j++) dst[(int64_t)c * S + j] = src[v * S + j];
    dens_out[c] = src[v * S].x;
    c2d[c] = (uint32_t)v;
}

// The same for the mixed forms: FP32 density and 16-bit SH records (S = 8-byte quads).
__global__ void k_compact16(const float* __restrict__ dens_in, const uint2* __restrict__ src, float* dens_out,
                            uint2* dst, const uint8_t* __restrict__ in_cage,
                            const uint32_t* __restrict__ index_offsets, uint32_t* c2d, int64_t N, int S)
{
    const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= N || !in_cage[v]) return;
    const uint32_t c = index_offsets[v];
    for (int j = 0; j < S; j++) dst[(int64_t)c * S + j] = src[v * S + j];
    dens_out[c] = dens_in[v];
    c2d[c] = (uint32_t)v;
}

__global__ void k_dense_mirror(float* mirror, const float* __restrict__ density, const uint8_t* __restrict__ in_cage,
                               const uint32_t* __restrict__ index_offsets, int64_t n)
{
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= n) return;
    mirror[d] = in_cage[d] ? density[index_offsets[d]] : __uint_as_float(kMirrorEmpty);
}

// Dense cell map, in two passes.  First a vertex map: bit x % 32 of word (z H + y) wpr + x / 32
// is set when vertex (x, y, z) has a density above kEmptyDensity (wpr = ceil(W / 32) words per
// row of vertices, padding bits clear).  Each density is read once, coalesced; a thread reads
// one column of kVertexRows rows, all loads in flight before the ballots.
constexpr int kVertexRows = 8;

__global__ void k_vertex_bits(const float* __restrict__ density, int W, int64_t rows, int wpr, uint32_t* vbits)
{
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * kVertexRows;
    const int lane = threadIdx.x & 31;
    float d[kVertexRows];
#pragma unroll
    for (int u = 0; u < kVertexRows; u++) d[u] = (r0 + u < rows && x < W) ? density[(r0 + u) * W + x] : 0.f;
#pragma unroll
    for (int u = 0; u < kVertexRows; u++) {
        const unsigned word = __ballot_sync(0xffffffffu, x < W && d[u] > kEmptyDensity);
        if (lane == 0 && r0 + u < rows && (x >> 5) < wpr) vbits[(r0 + u) * wpr + (x >> 5)] = word;
    }
}

// Then the cell map: bit c % 32 of word c / 32 is set unless all eight corner densities of cell
// c = (z (H-1) + y) (W-1) + x are at or below kEmptyDensity, i.e. when vertex column x or x+1 is
// open in any of the vertex rows (y, z), (y+1, z), (y, z+1), (y+1, z+1).  A thread per word; the
// word's cells fall in one or more cell rows, each segment taken from the four vertex rows
// with 64-bit funnel shifts (the segment and its x+1 column span at most 33 bits).
__global__ void k_cells_from_bits(const uint32_t* __restrict__ vbits, int W, int H, int wpr, int64_t n_cells,
                                  uint32_t* cells)
{
    const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (w >= (n_cells + 31) / 32) return;
    const int cw = W - 1, ch = H - 1;
    int64_t c = w * 32;
    const int64_t c_end = c + 32 < n_cells ? c + 32 : n_cells;
    uint32_t word = 0;
    int bit = 0;
    while (c < c_end) {
        const int64_t row = c / cw;
        const int x = (int)(c - row * cw);
        const int64_t y = row % ch, z = row / ch;
        const int len = (int)(cw - x < c_end - c ? cw - x : c_end - c);  // 1..32
        const int64_t r = z * H + y;
        const int64_t vrows[4] = {r, r + 1, r + H, r + H + 1};
        const int k = x >> 5, s = x & 31;
        uint64_t o = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t* rb = vbits + vrows[q] * wpr;
            const uint64_t lo = rb[k];
            const uint64_t hi = k + 1 < wpr ? rb[k + 1] : 0u;
            o |= ((hi << 32) | lo) >> s;
        }
        const uint32_t seg = (uint32_t)((o | (o >> 1)) & ((1ull << len) - 1));
        word |= seg << bit;  // bit + len <= 32
        bit += len;
        c += len;
    }
    cells[w] = word;
}

bool dense_skip_on(const cpx_grid* g)
{
    const bool march32 = g->prec != kPrecFP32 || (g->options & CPX_OPT_FP32_MARCH);
    return !g->sparse && march32 && !(g->options & CPX_OPT_NO_EMPTY_SKIP);
}

cpx_status refresh_dense_skip(cpx_grid* g, cudaStream_t st)
{
    if (!dense_skip_on(g)) return CPX_OK;
    const int cw = g->W - 1, ch = g->H - 1, cd = g->D - 1;
    const int64_t C = (int64_t)cw * ch * cd;
    const int bx = (cw + kBrick - 1) / kBrick, by = (ch + kBrick - 1) / kBrick, bz = (cd + kBrick - 1) / kBrick;
    const int64_t nb = (int64_t)bx * by * bz;
    const int64_t rows = (int64_t)g->H * g->D;
    const int wpr = (g->W + 31) / 32;
    if (!g->dense_cells) {
        if (cudaMalloc((void**)&g->dense_cells, ((C + 31) / 32) * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc((void**)&g->dense_vbits, rows * wpr * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc((void**)&g->dense_bricks, ((nb + 31) / 32) * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(g->dense_cells);
            cudaFree(g->dense_vbits);
            g->dense_cells = nullptr;
            g->dense_vbits = nullptr;
            set_error("empty-space maps could not be allocated");
            return CPX_ERR_OUT_OF_MEMORY;
        }
    }
    // whole warps in the vertex and brick launches: the warp that writes the last word has no
    // vertex (brick) in its tail threads
    const dim3 vgrid((unsigned)((rows + kVertexRows - 1) / kVertexRows), (unsigned)((g->W + 255) / 256));
    k_vertex_bits<<<vgrid, 256, 0, st>>>(g->density, g->W, rows, wpr, g->dense_vbits);
    const int64_t words = (C + 31) / 32;
    k_cells_from_bits<<<(unsigned)((words + 255) / 256), 256, 0, st>>>(g->dense_vbits, g->W, g->H, wpr, C,
                                                                        g->dense_cells);
    k_bricks<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(g->dense_cells, cw, ch, cd, bx, by, bz, g->dense_bricks);
    count_launch(3);
    return cuda_status(cudaGetLastError(), "empty-space maps");
}

cpx_status refresh_dense_mirror(cpx_grid* g, cudaStream_t st)
{
    if (!g->sparse) return refresh_dense_skip(g, st);
    if (!g->dense_mirror) return CPX_OK;
    k_dense_mirror<<<(unsigned)((g->n_dense + 255) / 256), 256, 0, st>>>(g->dense_mirror, g->density, g->in_cage,
                                                                          g->index_offsets, g->n_dense);
    count_launch();
    return cuda_status(cudaGetLastError(), "dense mirror");
}

cpx_status make_sparse_launch(cpx_grid* g)
{
    if (!g->have_occupancy) {
        set_error("cpx_occupancy_build must run before cpx_grid_make_sparse");
        return CPX_ERR_NOT_READY;
    }
    if (g->sparse) {
        set_error("grid is already sparse");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = g->in_cage_count;
    // the compact state is built in a holder of the same form, then replaces the dense one
    cpx_grid t;
    t.prec = g->prec;
    t.rec = g->rec;
    t.slots = g->slots;
    t.cur = 0;
    uint32_t* c2d = nullptr;
    cudaError_t e = alloc_state(&t, n);
    if (e == cudaSuccess) e = cudaMalloc((void**)&c2d, (n > 0 ? n : 1) * sizeof(uint32_t));
    if (e == cudaSuccess && !g->dense_mirror) e = cudaMalloc((void**)&g->dense_mirror, g->n_dense * sizeof(float));
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_state(&t);
        cudaFree(c2d);
        set_error("sparse buffers for %lld vertices could not be allocated", (long long)n);
        return CPX_ERR_OUT_OF_MEMORY;
    }
    const unsigned blocks = (unsigned)((g->n_dense + 255) / 256);
    if (g->prec == kPrecFP32) {
        k_compact<<<blocks, 256>>>(reinterpret_cast<const float4*>(g->params[g->cur]),
                                   reinterpret_cast<float4*>(t.params[0]), t.density, g->in_cage,
                                   g->index_offsets, c2d, g->n_dense, g->rec / 4);
    } else {
        k_compact16<<<blocks, 256>>>(g->dens[g->cur], reinterpret_cast<const uint2*>(g->sh16[g->cur]),
                                     t.dens[0], reinterpret_cast<uint2*>(t.sh16[0]), g->in_cage,
                                     g->index_offsets, c2d, g->n_dense, g->slots / 4);
    }
    count_launch();
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        free_state(&t);
        cudaFree(c2d);
        return cuda_status(e, "compaction");
    }
    free_state(g);
    cudaFree(g->compact_to_dense);
    g->params[0] = t.params[0];
    g->params[1] = t.params[1];
    g->grad = t.grad;
    g->m = t.m;
    g->v = t.v;
    g->sh16[0] = t.sh16[0];
    g->sh16[1] = t.sh16[1];
    g->m16 = t.m16;
    g->v16 = t.v16;
    g->dens[0] = t.dens[0];
    g->dens[1] = t.dens[1];
    g->touched[0] = t.touched[0];
    g->touched[1] = t.touched[1];
    g->tcur = 0;
    g->all_touched = 0;
    g->cur = 0;
    g->density = g->prec == kPrecFP32 ? t.density : g->dens[0];
    g->compact_to_dense = c2d;
    g->n_act = n;
    g->sparse = 1;
    cpx_status rc = refresh_dense_mirror(g, 0);
    if (rc != CPX_OK) return rc;
    return cuda_status(cudaDeviceSynchronize(), "dense mirror");
}

}  // namespace cpx
