// batch.cu -- batched multi-scene training: many scenes stepped by one placement launch and
// one shading launch (persistent kernels in march.cu), then each scene's TV + Adam sweep.
//
// The reference trains one scene per process (Experiment.cu); a batch lets small scenes share
// the GPU.  Iteration i of a scene reads batch i % pool of its ray table and steps Adam with
// timestep i + 1 read from a device counter, so one iteration captures as a CUDA graph and
// replays with no host work but the launch.  The grids' ping-pong buffers alternate every
// step, so there are two graphs, one per parity; a grid changed outside the batch (another
// buffer, another parity, gradients uploaded) no longer matches either and the step runs
// eagerly, after which the graphs are captured again on demand.
#include <cstring>
#include <vector>

#include "cpx_internal.cuh"

namespace cpx {

// What a captured graph depends on, per scene: the buffers the views and sweep arguments
// name and the flags that change which ones they name.
struct SceneSig {
    const void* grid;
    const void* params;
    const void* density;
    const void* touched;
    int cur, tcur, all_touched, options;
    int64_t n_act;
    bool operator==(const SceneSig& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

static SceneSig scene_sig(const cpx_grid* g)
{
    SceneSig s;
    std::memset(&s, 0, sizeof(s));
    s.grid = g;
    s.params = g->prec == kPrecFP32 ? (const void*)g->params[g->cur] : (const void*)g->sh16[g->cur];
    s.density = g->prec == kPrecFP32 ? (const void*)g->density : (const void*)g->dens[g->cur];
    s.touched = g->touched[g->tcur];
    s.cur = g->cur;
    s.tcur = g->tcur;
    s.all_touched = g->all_touched;
    s.options = g->options;
    s.n_act = g->n_act;
    return s;
}

__global__ void k_batch_advance(int* iter) { *iter += 1; }

__device__ __forceinline__ double batch_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// getMSEError (Utils.cu:311-320) of each scene's losses: one block per scene.
__global__ void k_batch_mse(const double* losses, const int* base, const int* len, double* out)
{
    __shared__ double part[32];
    const double* l = losses + base[blockIdx.x];
    const int n = len[blockIdx.x];
    double s = 0.;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += l[i] * l[i];
    s = batch_warp_sum(s);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.;
        v = batch_warp_sum(v);
        if (threadIdx.x == 0) out[blockIdx.x] = n > 0 ? v / n : 0.;
    }
}

}  // namespace cpx

using namespace cpx;

struct cpx_batch {
    std::vector<cpx_grid*> grids;
    std::vector<cpx_rays*> rays;
    std::vector<int> len, pool, ray_base;
    std::vector<int64_t> sample_base;
    int n = 0, total = 0, prec = 0;
    int64_t total_slots = 0;
    cpx_step_args args;
    bool fuse = false;
    BatchTuning tuning;
    // device buffers
    SampleRec* samples = nullptr;
    float4* colours = nullptr;
    int* counts = nullptr;
    double* acc = nullptr;
    double* losses = nullptr;
    int* err = nullptr;
    int* queue = nullptr;
    int* iter = nullptr;
    int* d_base = nullptr;
    int* d_len = nullptr;
    double* d_mse = nullptr;
    BatchScene* etab = nullptr;    // scene table of eager steps
    BatchScene* gtab[2] = {nullptr, nullptr};  // scene tables of the two graphs
    // the FP32 dense grids' sweeps run as one launch over a device table of their arguments:
    // the eager steps' table and the two graphs' tables
    void* stab_eager = nullptr;
    void* stab[2] = {nullptr, nullptr};
    std::vector<unsigned char> stab_host;
    int iteration = 0;             // host mirror of *iter
    // graphs
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    std::vector<SceneSig> sig[2];
    BatchTuning graph_tuning[2];
    int launches = 0;  // kernels per step
};

static void batch_free(cpx_batch* b)
{
    for (int p = 0; p < 2; p++) {
        if (b->graph[p]) cudaGraphExecDestroy(b->graph[p]);
        cudaFree(b->gtab[p]);
    }
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->samples);
    cudaFree(b->colours);
    cudaFree(b->counts);
    cudaFree(b->acc);
    cudaFree(b->losses);
    cudaFree(b->err);
    cudaFree(b->queue);
    cudaFree(b->iter);
    cudaFree(b->d_base);
    cudaFree(b->d_len);
    cudaFree(b->d_mse);
    cudaFree(b->etab);
    cudaFree(b->stab_eager);
    cudaFree(b->stab[0]);
    cudaFree(b->stab[1]);
    delete b;
}

// The grids whose sweeps run in the one batched launch, in batch order.
static std::vector<cpx_grid*> batch_sweep_grids(const cpx_batch* b)
{
    std::vector<cpx_grid*> out;
    for (cpx_grid* g : b->grids)
        if (sweep_batchable(g, b->fuse)) out.push_back(g);
    return out;
}

// The host image of the batched sweep's table for the grids' current buffers; returns its
// work items (0: no grid qualifies).
static int batch_sweep_table(cpx_batch* b, const std::vector<cpx_grid*>& sg)
{
    if (sg.empty()) return 0;
    b->stab_host.resize(sweep_table_bytes((int)sg.size()));
    const cpx_step_args& g = b->args;
    return sweep_table_fill(sg.data(), (int)sg.size(), g.lam_density, g.lam_sh, g.lr, g.sh_lr, b->iter,
                            b->stab_host.data());
}

static std::vector<BatchScene> batch_table(const cpx_batch* b)
{
    std::vector<BatchScene> t(b->n);
    for (int i = 0; i < b->n; i++)
        t[i] = batch_scene_view(b->grids[i], b->rays[i], b->len[i], b->pool[i], b->ray_base[i], b->sample_base[i]);
    return t;
}

static std::vector<SceneSig> batch_sig(const cpx_batch* b)
{
    std::vector<SceneSig> s(b->n);
    for (int i = 0; i < b->n; i++) s[i] = scene_sig(b->grids[i]);
    return s;
}

static bool valid_tuning(const BatchTuning& t)
{
    return t.place_block >= 32 && t.place_block <= 512 && t.place_block % 32 == 0 &&
           (t.shade_warps == 2 || t.shade_warps == 4 || t.shade_warps == 8) && t.grab >= 1 && t.grab <= 8 &&
           (t.spl == 1 || t.spl == 2 || t.spl == 4) && t.shade_warps * t.spl <= 8;
}

// Enqueue one iteration on st with the scene table at tab and the batched sweep's table at stab
// (items work items; both already on the device).
static cpx_status batch_enqueue(cpx_batch* b, const BatchScene* tab, const void* stab, int items,
                                const BatchTuning& tn, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(b->queue, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return cuda_status(e, "batch queue");
    BatchArgs a;
    a.scenes = tab;
    a.n_scenes = b->n;
    a.total_rays = b->total;
    a.samples = b->samples;
    a.colours = b->colours;
    a.counts = b->counts;
    a.acc = b->acc;
    a.losses = b->losses;
    a.err = b->err;
    a.queue = b->queue;
    a.iter = b->iter;
    a.mask_coef = b->args.mask_coef;
    a.huber = b->args.huber_delta;
    a.grab = tn.grab;
    cpx_status s = batch_launch_march(b->prec, a, tn, st);
    if (s != CPX_OK) return s;
    int launches = 2;
    const cpx_step_args& g = b->args;
    const std::vector<cpx_grid*> sg = batch_sweep_grids(b);
    for (int i = 0; i < b->n; i++) {
        cpx_grid* gr = b->grids[i];
        if (sweep_batchable(gr, b->fuse)) continue;  // in the batched sweep below
        if (g.do_tv && !b->fuse) {
            s = tv_launch(gr, g.lam_density, g.lam_sh, g.tv_type, g.tv_neighbours, st);
            if (s != CPX_OK) return s;
            launches++;
        }
        s = sweep_adam(gr, b->fuse, g.lam_density, g.lam_sh, g.lr, g.sh_lr, 1, st, b->iter);
        if (s != CPX_OK) return s;
        launches++;
    }
    if (!sg.empty()) {
        s = sweep_batched_launch(sg.data(), (int)sg.size(), stab, items, st);
        if (s != CPX_OK) return s;
        launches++;
    }
    k_batch_mse<<<b->n, 256, 0, st>>>(b->losses, b->d_base, b->d_len, b->d_mse);
    k_batch_advance<<<1, 1, 0, st>>>(b->iter);
    count_launch(2);
    b->launches = launches + 2;
    return cuda_status(cudaGetLastError(), "batch step");
}

static cpx_status batch_eager(cpx_batch* b, cudaStream_t st)
{
    const std::vector<BatchScene> t = batch_table(b);
    // the tables are copied from pageable memory: the call returns once the source is read
    cudaError_t e = cudaMemcpyAsync(b->etab, t.data(), sizeof(BatchScene) * b->n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "batch table");
    const std::vector<cpx_grid*> sg = batch_sweep_grids(b);
    const int items = batch_sweep_table(b, sg);
    if (items > 0) {
        e = cudaMemcpyAsync(b->stab_eager, b->stab_host.data(), b->stab_host.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_status(e, "batch sweep table");
    }
    return batch_enqueue(b, b->etab, b->stab_eager, items, b->tuning, st);
}

// Capture the iteration of the grids' current parity into graph p.  The capture runs the
// host side of a step (the grids' buffers flip) without executing it; the caller flips back.
static cpx_status batch_capture(cpx_batch* b, int p)
{
    if (b->graph[p]) {
        cudaGraphExecDestroy(b->graph[p]);
        b->graph[p] = nullptr;
    }
    const std::vector<BatchScene> t = batch_table(b);
    cudaError_t e = cudaMemcpy(b->gtab[p], t.data(), sizeof(BatchScene) * b->n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "batch table");
    const std::vector<cpx_grid*> sg = batch_sweep_grids(b);
    const int items = batch_sweep_table(b, sg);
    if (items > 0) {
        e = cudaMemcpy(b->stab[p], b->stab_host.data(), b->stab_host.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_status(e, "batch sweep table");
    }
    b->sig[p] = batch_sig(b);
    std::vector<int> cur(b->n), tcur(b->n), all(b->n);
    for (int i = 0; i < b->n; i++) {
        cur[i] = b->grids[i]->cur;
        tcur[i] = b->grids[i]->tcur;
        all[i] = b->grids[i]->all_touched;
    }
    e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "batch capture");
    cpx_status s = batch_enqueue(b, b->gtab[p], b->stab[p], items, b->tuning, b->cap);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(b->cap, &graph);
    for (int i = 0; i < b->n; i++) {  // nothing ran: the grids keep their buffers
        b->grids[i]->cur = cur[i];
        b->grids[i]->tcur = tcur[i];
        b->grids[i]->all_touched = all[i];
    }
    if (s != CPX_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    if (e != cudaSuccess) return cuda_status(e, "batch capture");
    e = cudaGraphInstantiate(&b->graph[p], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        b->graph[p] = nullptr;
        return cuda_status(e, "batch graph");
    }
    b->graph_tuning[p] = b->tuning;
    return CPX_OK;
}

static void flip_grids(cpx_batch* b)
{
    for (int i = 0; i < b->n; i++) {
        cpx_grid* g = b->grids[i];
        g->cur ^= 1;
        g->tcur ^= 1;
        g->all_touched = 0;
    }
}

static cpx_status batch_step(cpx_batch* b, bool graphs, cudaStream_t st)
{
    if (!graphs) {
        cpx_status s = batch_eager(b, st);
        if (s == CPX_OK) b->iteration++;
        return s;
    }
    const std::vector<SceneSig> now = batch_sig(b);
    bool any_all = false;
    for (const SceneSig& s : now) any_all |= s.all_touched != 0;
    if (any_all) {
        // gradients arrived by another route: this step reads every record, eagerly
        cpx_status s = batch_eager(b, st);
        if (s == CPX_OK) b->iteration++;
        return s;
    }
    int p = -1;
    for (int q = 0; q < 2; q++)
        if (b->graph[q] && b->sig[q] == now && b->graph_tuning[q].place_block == b->tuning.place_block &&
            b->graph_tuning[q].shade_warps == b->tuning.shade_warps && b->graph_tuning[q].grab == b->tuning.grab &&
            b->graph_tuning[q].spl == b->tuning.spl)
            p = q;
    if (p < 0) {
        // capture this parity into a free slot; with none free both graphs are stale (a grid
        // changed outside the batch, or the launch shapes did)
        p = !b->graph[0] ? 0 : !b->graph[1] ? 1 : -1;
        if (p < 0) {
            for (int q = 0; q < 2; q++) {
                cudaGraphExecDestroy(b->graph[q]);
                b->graph[q] = nullptr;
            }
            p = 0;
        }
        cpx_status s = batch_capture(b, p);
        if (s != CPX_OK) return s;
    }
    cudaError_t e = cudaGraphLaunch(b->graph[p], st);
    if (e != cudaSuccess) return cuda_status(e, "batch graph launch");
    count_launch(b->launches);
    flip_grids(b);
    b->iteration++;
    return CPX_OK;
}

extern "C" {

cpx_status cpx_batch_create(const cpx_batch_scene* scenes, int n_scenes, const cpx_step_args* args,
                            cpx_batch** out)
{
    if (!scenes || !args || !out || n_scenes < 1 || n_scenes > kMaxBatchScenes) {
        set_error("a batch holds 1..%d scenes", kMaxBatchScenes);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (args->timestep < 1) {
        set_error("timestep starts at 1");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const bool fuse = args->do_tv && args->tv_type == 0 && args->tv_neighbours == 6;
    cpx_batch* b = new cpx_batch();
    b->n = n_scenes;
    b->args = *args;
    b->fuse = fuse;
    int64_t rays = 0, slots = 0;
    for (int i = 0; i < n_scenes; i++) {
        cpx_grid* g = scenes[i].grid;
        cpx_rays* r = scenes[i].rays;
        const int len = scenes[i].rays_per_batch;
        const char* why = nullptr;
        if (!g || !r) why = "null grid or ray handle";
        else if (len < 1 || r->n < len) why = "rays_per_batch outside 1..n_rays";
        else if (g->sh_dim != 9) why = "batched scenes hold SH band 2 (9 coefficients per channel)";
        else if (i > 0 && g->prec != scenes[0].grid->prec) why = "the scenes of a batch share one precision form";
        else if (i > 0 && (g->options & CPX_OPT_FP32_MARCH) != (scenes[0].grid->options & CPX_OPT_FP32_MARCH))
            why = "the scenes of a batch share one march form";
        else if (g->prec == kPrecFP32 && (g->options & CPX_OPT_FP32_MARCH))
            why = "the batched FP32 form marches as the reference (no FP32-march option)";
        else if (g->sparse && !g->have_occupancy) why = "sparse grid without occupancy";
        else if (args->do_tv && !fuse && g->prec != kPrecFP32)
            why = "the mixed forms run TV type 0 / 6 neighbours fused into the optimizer sweep only";
        for (int j = 0; j < i && !why; j++)
            if (scenes[j].grid == g) why = "a grid appears twice in the batch";
        if (why) {
            set_error("scene %d: %s", i, why);
            delete b;
            return CPX_ERR_INVALID_ARGUMENT;
        }
        // the empty-space maps exist before any step is captured
        if (refresh_dense_skip(g, 0) != CPX_OK) {
            delete b;
            return CPX_ERR_OUT_OF_MEMORY;
        }
        b->grids.push_back(g);
        b->rays.push_back(r);
        b->len.push_back(len);
        b->pool.push_back((int)(r->n / len));
        b->ray_base.push_back((int)rays);
        b->sample_base.push_back(slots);
        rays += len;
        slots += (int64_t)len * march_samples_per_ray(g);
    }
    if (rays >= (1 << 30)) {
        set_error("a batch step holds fewer than 2^30 rays");
        delete b;
        return CPX_ERR_INVALID_ARGUMENT;
    }
    b->prec = scenes[0].grid->prec;
    b->total = (int)rays;
    b->total_slots = slots;
    b->iteration = args->timestep - 1;
    cudaError_t e = cudaSuccess;
    auto grab = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    grab((void**)&b->samples, sizeof(SampleRec) * (size_t)slots);
    grab((void**)&b->colours, sizeof(float4) * (size_t)slots);
    grab((void**)&b->counts, sizeof(int) * (size_t)rays);
    grab((void**)&b->acc, sizeof(double) * (size_t)rays);
    grab((void**)&b->losses, sizeof(double) * (size_t)rays);
    grab((void**)&b->err, sizeof(int) * 4);
    grab((void**)&b->queue, sizeof(int) * 2);
    grab((void**)&b->iter, sizeof(int));
    grab((void**)&b->d_base, sizeof(int) * n_scenes);
    grab((void**)&b->d_len, sizeof(int) * n_scenes);
    grab((void**)&b->d_mse, sizeof(double) * n_scenes);
    grab((void**)&b->etab, sizeof(BatchScene) * n_scenes);
    grab((void**)&b->gtab[0], sizeof(BatchScene) * n_scenes);
    grab((void**)&b->gtab[1], sizeof(BatchScene) * n_scenes);
    grab(&b->stab_eager, sweep_table_bytes(n_scenes));
    grab(&b->stab[0], sweep_table_bytes(n_scenes));
    grab(&b->stab[1], sweep_table_bytes(n_scenes));
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(b);
        set_error("batch buffers (%lld sample slots) could not be allocated", (long long)slots);
        return CPX_ERR_OUT_OF_MEMORY;
    }
    e = cudaMemset(b->err, 0, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMemset(b->d_mse, 0, sizeof(double) * n_scenes);
    if (e == cudaSuccess) e = cudaMemcpy(b->iter, &b->iteration, sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_base, b->ray_base.data(), sizeof(int) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_len, b->len.data(), sizeof(int) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_status(e, "batch create");
    }
    *out = b;
    return CPX_OK;
}

cpx_status cpx_batch_destroy(cpx_batch* b)
{
    if (!b) return CPX_OK;
    cudaDeviceSynchronize();
    batch_free(b);
    return CPX_OK;
}

cpx_status cpx_batch_step(cpx_batch* b, int use_graphs, cpx_stream stream)
{
    if (!b) {
        set_error("null batch handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    return batch_step(b, use_graphs != 0, (cudaStream_t)stream);
}

cpx_status cpx_batch_mse(cpx_batch* b, double* mse_host, cpx_stream stream)
{
    if (!b || !mse_host) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(mse_host, b->d_mse, sizeof(double) * b->n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return cuda_status(e, "batch mse");
}

cpx_status cpx_batch_check(cpx_batch* b)
{
    if (!b) {
        set_error("null batch handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "batch check");
    int flags[4] = {0, 0, 0, 0};
    e = cudaMemcpy(flags, b->err, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "batch check");
    cudaMemset(b->err, 0, sizeof(flags));
    if (flags[0] & 1) {
        set_error("a ray's march exceeded its sample bound (near/far beyond the grid box?)");
        return CPX_ERR_ITERATION_CAP;
    }
    if (flags[0] & 32) {
        set_error("a shading warp gave up waiting for a vertex record copy");
        return CPX_ERR_NOT_READY;
    }
    return CPX_OK;
}

cpx_status cpx_batch_info(const cpx_batch* b, int* iteration, int* total_rays, int* launches_per_step)
{
    if (!b) {
        set_error("null batch handle");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (iteration) *iteration = b->iteration;
    if (total_rays) *total_rays = b->total;
    if (launches_per_step) {
        int l = 4 + b->n;  // place, shade, per-scene sweeps, MSE, counter
        if (b->args.do_tv && !b->fuse) l += b->n;
        *launches_per_step = l;
    }
    return CPX_OK;
}

cpx_status cpx_batch_set_tuning(cpx_batch* b, const cpx_batch_tuning* t)
{
    if (!b || !t) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    BatchTuning n;
    n.place_block = t->place_block;
    n.shade_warps = t->shade_warps;
    n.grab = t->grab;
    n.spl = t->samples_per_step;
    if (!valid_tuning(n)) {
        set_error("tuning outside place_block 32..512 (multiple of 32), shade_warps 2/4/8, grab 1..8, "
                  "samples_per_step 1/2/4 with shade_warps * samples_per_step <= 8");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    b->tuning = n;
    return CPX_OK;
}

cpx_status cpx_batch_get_tuning(const cpx_batch* b, cpx_batch_tuning* t)
{
    if (!b || !t) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    t->place_block = b->tuning.place_block;
    t->shade_warps = b->tuning.shade_warps;
    t->grab = b->tuning.grab;
    t->samples_per_step = b->tuning.spl;
    return CPX_OK;
}

cpx_status cpx_batch_autotune(cpx_batch* b, int steps_per_trial, cpx_batch_tuning* best, cpx_stream stream)
{
    if (!b || steps_per_trial < 1) {
        set_error("autotune needs a batch and at least one step per trial");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        set_error("autotune events");
        return CPX_ERR_CUDA;
    }
    auto trial = [&](const BatchTuning& t, float* ms) -> cpx_status {
        b->tuning = t;
        cpx_status s = batch_step(b, false, st);  // one untimed step: first-use costs
        if (s != CPX_OK) return s;
        cudaEventRecord(e0, st);
        for (int i = 0; i < steps_per_trial && s == CPX_OK; i++) s = batch_step(b, false, st);
        cudaEventRecord(e1, st);
        if (s != CPX_OK) return s;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return cuda_status(e, "autotune");
        cudaEventElapsedTime(ms, e0, e1);
        return CPX_OK;
    };
    const int places[] = {64, 128, 256, 512};
    const int warps[] = {2, 4, 8};
    const int grabs[] = {1, 2, 4, 8};
    const int spls[] = {1, 2, 4};
    BatchTuning cur = b->tuning;
    float best_ms = 0.f;
    cpx_status s = trial(cur, &best_ms);
    for (int round = 0; round < 2 && s == CPX_OK; round++) {
        for (int dim = 0; dim < 4 && s == CPX_OK; dim++) {
            const int* vals = dim == 0 ? places : dim == 1 ? warps : dim == 2 ? grabs : spls;
            const int nv = dim == 1 || dim == 3 ? 3 : 4;
            for (int k = 0; k < nv && s == CPX_OK; k++) {
                BatchTuning t = cur;
                int& field = dim == 0 ? t.place_block : dim == 1 ? t.shade_warps : dim == 2 ? t.grab : t.spl;
                if (field == vals[k]) continue;
                field = vals[k];
                if (!valid_tuning(t)) continue;  // tables of shade_warps * samples_per_step > 8 warps
                float ms = 0.f;
                s = trial(t, &ms);
                if (s == CPX_OK && ms < best_ms) {
                    best_ms = ms;
                    cur = t;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tuning = cur;
    if (s != CPX_OK) return s;
    if (best) {
        best->place_block = cur.place_block;
        best->shade_warps = cur.shade_warps;
        best->grab = cur.grab;
        best->samples_per_step = cur.spl;
    }
    return CPX_OK;
}

}  // extern "C"
