/*
 * cpx_oracle.c -- CPU restatement of the Clear-plenoxels training hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path and the
 * timed CPU baseline.  See cpx_oracle.h for the contract.  Citations are
 * file:line in the reference project (SVRF = SparseVolumeRadianceField/).
 *
 * Parity pins: ray/AABB hits, occupancy and index lists are compared bit for
 * bit against the reference's own kernels run on a B200 (tests/golden/);
 * float results that pass through exp/log/pow agree to a few ulp.
 */
#include "cpx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static unsigned g_contract = ORC_CONTRACT_DEFAULT;
static int g_threads = 0;

void orc_set_contract_mode(unsigned mode) { g_contract = mode; }
unsigned orc_get_contract_mode(void) { return g_contract; }
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------- helpers */

/* (unsigned int)double as the GPU converts it (cvt.rzi.u32.f64 saturates;
 * NaN -> 0).  The reference relies on this at RenderUtils.cu:830-833. */
static inline uint32_t sat_u32(double v)
{
    if (!(v > 0.0)) return 0u;              /* negatives, -0, NaN */
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

/* getSceneIndex (RenderUtils.cu:3-13): clamp to the grid, z-y-x linear index. */
static inline int scene_index(int col, int row, int depth, int W, int H, int D)
{
    col = col < 0 ? 0 : (col > W - 1 ? W - 1 : col);
    row = row < 0 ? 0 : (row > H - 1 ? H - 1 : row);
    depth = depth < 0 ? 0 : (depth > D - 1 ? D - 1 : depth);
    return depth * W * H + row * W + col;
}

/* getIndex (SceneUtils.cu:250-260): upper clamp only. */
static inline int64_t grid_index_upper(int col, int row, int depth, int W, int H, int D)
{
    col = col < W ? col : W - 1;
    row = row < H ? row : H - 1;
    depth = depth < D ? depth : D - 1;
    return (int64_t)depth * W * H + (int64_t)row * W + col;
}

static inline double offset_at(const double* o, int n, int i)
{
    return (o && i >= 0 && i < n) ? o[i] : 0.0;
}

static inline double minf_d(double a, double b) { return a > b ? b : a; }
static inline double maxf_d(double a, double b) { return a > b ? a : b; }

/* ------------------------------------------------------ R4 activations */

/* density_activation: log(1 + exp(x - 13)) in float (RenderUtils.cu:491-495). */
float orc_density_activation(float x) { return logf(1.f + expf(x - 13.f)); }

/* density_derivation: 1 / (1 + exp(13 - x)) in float (RenderUtils.cu:497-501). */
float orc_density_derivation(float x) { return 1.f / (1.f + expf(13.f - x)); }

/* sigmoid: 1 / (1 + exp(-0.1 x)) evaluated in double (RenderUtils.cu:480-483). */
float orc_sigmoid(float x) { return (float)(1.0 / (1.0 + exp(-0.1 * (double)x))); }

/* sigmoid_derivative: 0.1 s (1 - s) (RenderUtils.cu:485-489). */
float orc_sigmoid_derivative(float x)
{
    float s = orc_sigmoid(x);
    return (float)(0.1 * (double)s * (double)(1.f - s));
}

/* ------------------------------------------------------ R5 SH basis */

/* The unnormalised basis the reference uses (RenderUtils.cu:1646-1670); entries
 * beyond band 2 are kept for completeness. */
void orc_sh_basis(const float d[3], float shs[25])
{
    const float x = d[0], y = d[1], z = d[2];
    shs[0] = 1.f;
    shs[1] = y;
    shs[2] = z;
    shs[3] = x;
    shs[4] = x * y;
    shs[5] = y * z;
    shs[6] = fmaf(3.f * z, z, -1.f);
    shs[7] = x * z;
    shs[8] = fmaf(x, x, -(y * y));
    shs[9] = y * (fmaf(3.f * x, x, -(y * y)));
    shs[10] = x * y * z;
    shs[11] = y * (fmaf(5.f * z, z, -1.f));
    shs[12] = fmaf(5.f * z * z, z, -(3.f * z));
    shs[13] = x * (fmaf(5.f * z, z, -1.f));
    shs[14] = (fmaf(x, x, -(y * y))) * z;
    shs[15] = x * (fmaf(x, x, -(3.f * y * y)));
    shs[16] = x * y * (fmaf(x, x, -(y * y)));
    shs[17] = y * (fmaf(3.f * x, x, -(y * y))) * z;
    shs[18] = x * y * (fmaf(7.f * z, z, -1.f));
    shs[19] = y * (fmaf(7.f * z * z, z, -(3.f * z)));
    shs[20] = fmaf(35.f * z * z * z, z, -(30.f * z * z)) + 3.f;
    shs[21] = x * (fmaf(7.f * z * z, z, -(3.f * z)));
    shs[22] = (float)((double)fmaf(x, x, -(y * y)) * ((double)(7.f * z * z) - 1.0));
    shs[23] = x * (fmaf(x, x, -(3.f * y * y))) * z;
    shs[24] = x * x * (fmaf(x, x, -(3.f * y * y))) - y * y * (fmaf(3.f * x, x, -(y * y)));
}

/* ------------------------------------------------------ R1 rays */

/* getBound (Rays.cu:22-75) + initialRays (Rays.cu:77-144) for one pixel list. */
void orc_rays_from_camera(const double* alpha, const double* principle,
                          const double* c2w, const double* centre, const int* bbox,
                          int img_w, const uint8_t* red, const uint8_t* green,
                          const uint8_t* blue, const uint8_t* mask, int white_bg,
                          const int* pix_index, int n_pix, orc_rays* out, int64_t out_start)
{
    for (int i = 0; i < n_pix; i++) {
        const int pixel = pix_index[i];
        const int row = pixel / img_w;
        const int col = pixel % img_w;

        float xin[4];
        xin[0] = (float)(((double)col + 0.5 - principle[0]) / alpha[0]);
        xin[1] = (float)(((double)row + 0.5 - principle[1]) / alpha[1]);
        xin[2] = 1.0f;
        xin[3] = 1.0f;

        float sp[4];
        for (int rr = 0; rr < 4; rr++) {
            sp[rr] = 0.f;
            for (int cc = 0; cc < 4; cc++) {
                if (g_contract & ORC_CONTRACT_RAYDIR)
                    sp[rr] = (float)fma(c2w[rr * 4 + cc], (double)xin[cc], (double)sp[rr]);
                else
                    sp[rr] = (float)((double)sp[rr] + c2w[rr * 4 + cc] * (double)xin[cc]);
            }
            sp[rr] = (float)((double)sp[rr] - centre[rr]);
        }

        /* normalizePoint (Rays.cu:13-20): float sum of squares, double sqrt. */
        float fs;
        if (g_contract & ORC_CONTRACT_NORM_P0)
            fs = fmaf(sp[2], sp[2], fmaf(sp[0], sp[0], sp[1] * sp[1]));
        else if (g_contract & ORC_CONTRACT_NORM_P1)
            fs = fmaf(sp[2], sp[2], fmaf(sp[1], sp[1], sp[0] * sp[0]));
        else
            fs = (sp[0] * sp[0] + sp[1] * sp[1]) + sp[2] * sp[2];
        double sum = sqrt((double)fs);
        sp[0] = (float)((double)sp[0] / sum);
        sp[1] = (float)((double)sp[1] / sum);
        sp[2] = (float)((double)sp[2] / sum);

        double t[6] = {
            ((double)bbox[1] - centre[0]) / (double)sp[0],
            ((double)bbox[0] - centre[0]) / (double)sp[0],
            ((double)bbox[3] - centre[1]) / (double)sp[1],
            ((double)bbox[2] - centre[1]) / (double)sp[1],
            ((double)bbox[5] - centre[2]) / (double)sp[2],
            ((double)bbox[4] - centre[2]) / (double)sp[2],
        };
        double t_min = minf_d(t[0], t[1]);
        double t_max = maxf_d(t[0], t[1]);
        t_min = maxf_d(t_min, minf_d(t[2], t[3]));
        t_max = minf_d(t_max, maxf_d(t[2], t[3]));
        t_min = maxf_d(t_min, minf_d(t[4], t[5]));
        t_max = minf_d(t_max, maxf_d(t[4], t[5]));

        const int64_t ri = out_start + i;
        out->ox[ri] = (float)centre[0];
        out->oy[ri] = (float)centre[1];
        out->oz[ri] = (float)centre[2];
        out->near_t[ri] = (float)t_min;
        out->far_t[ri] = (float)t_max;
        out->dx[ri] = sp[0];
        out->dy[ri] = sp[1];
        out->dz[ri] = sp[2];
        const uint8_t m = mask ? mask[pixel] : 255;
        out->mask[ri] = m;
        if (white_bg) {
            /* u8(r*m/255.f + 255 - m) (Rays.cu:128-133) */
            out->r[ri] = (uint8_t)((float)(red[pixel] * m) / 255.f + 255.f - (float)m);
            out->g[ri] = (uint8_t)((float)(green[pixel] * m) / 255.f + 255.f - (float)m);
            out->b[ri] = (uint8_t)((float)(blue[pixel] * m) / 255.f + 255.f - (float)m);
        } else {
            out->r[ri] = red[pixel];
            out->g[ri] = green[pixel];
            out->b[ri] = blue[pixel];
        }
    }
}

/* ------------------------------------------------------ R6 trilinear */

static inline int n_active_sh(const orc_scene* s) { return (s->band + 1) * (s->band + 1); }

/* Corner offsets in the reference's visiting order (RenderUtils.cu:855-990). */
static const int k_corner[8][3] = {
    {0, 0, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 0},
    {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1},
};

static inline double corner_weight(int q, double x, double y, double z)
{
    switch (q) {
    case 0: return (1. - x) * (1. - y) * (1. - z);
    case 1: return (1. - x) * y * (1. - z);
    case 2: return x * (1. - y) * (1. - z);
    case 3: return x * y * (1. - z);
    case 4: return (1. - x) * (1. - y) * z;
    case 5: return (1. - x) * y * z;
    case 6: return x * (1. - y) * z;
    default: return x * y * z;
    }
}

/* Sample position (RenderUtils.cu:1676-1678). */
static inline void sample_position(const orc_scene* s, const orc_rays* r, int ri, double t,
                                   int intT, double bc[3])
{
    const double o[3] = {(double)r->ox[ri], (double)r->oy[ri], (double)r->oz[ri]};
    const double d[3] = {(double)r->dx[ri], (double)r->dy[ri], (double)r->dz[ri]};
    const double off[3] = {offset_at(s->off_x, s->n_off, intT),
                           offset_at(s->off_y, s->n_off, intT),
                           offset_at(s->off_z, s->n_off, intT)};
    for (int a = 0; a < 3; a++) {
        if (g_contract & ORC_CONTRACT_POS)
            bc[a] = fma(t, d[a], o[a]) + off[a];
        else
            bc[a] = (o[a] + t * d[a]) + off[a];
    }
}

/* Cell index of a sample, -1 when the sparse occupancy says skip. */
static inline int occupied(const orc_scene* s, const uint32_t bi[3])
{
    if (!s->sparse) return 1;
    int ci = scene_index((int)bi[0], (int)bi[1], (int)bi[2], s->W - 1, s->H - 1, s->D - 1);
    return s->occ[ci] != 0;
}

static inline int64_t corner_index(const orc_scene* s, const uint32_t bi[3], int q)
{
    int idx = scene_index((int)(bi[0] + (uint32_t)k_corner[q][0]),
                          (int)(bi[1] + (uint32_t)k_corner[q][1]),
                          (int)(bi[2] + (uint32_t)k_corner[q][2]), s->W, s->H, s->D);
    if (s->sparse) return (int64_t)s->index_offsets[(uint32_t)idx];
    return (int64_t)(uint32_t)idx;
}

/* trilerpRGB (RenderUtils.cu:826-1004): raw density and raw colours. */
static int trilerp_rgb(const orc_scene* s, const double bc[3], const float* shs, float tri[4])
{
    uint32_t bi[3] = {sat_u32(bc[0]), sat_u32(bc[1]), sat_u32(bc[2])};
    if (!occupied(s, bi)) return 0;
    const double x = bc[0] - (double)bi[0];
    const double y = bc[1] - (double)bi[1];
    const double z = bc[2] - (double)bi[2];
    const int nsh = n_active_sh(s);
    const int64_t n = s->n_act;
    const float* rho = s->params;
    float sh_tri[75];
    for (int i = 0; i < s->sh_dim * 3; i++) sh_tri[i] = 0.f;
    tri[0] = tri[1] = tri[2] = tri[3] = 0.f;
    for (int q = 0; q < 8; q++) {
        const int64_t idx = corner_index(s, bi, q);
        const double c = corner_weight(q, x, y, z);
        tri[0] = (float)fma(c, (double)rho[idx], (double)tri[0]);
        for (int i = 0; i < nsh; i++) {
            for (int ch = 0; ch < 3; ch++) {
                const float* a = s->params + (int64_t)(1 + ch * s->sh_dim + i) * n;
                sh_tri[ch * s->sh_dim + i] =
                    (float)fma(c, (double)a[idx], (double)sh_tri[ch * s->sh_dim + i]);
            }
        }
    }
    for (int ch = 0; ch < 3; ch++) {
        float acc = 0.f;
        for (int i = 0; i < nsh; i++) acc = fmaf(sh_tri[ch * s->sh_dim + i], shs[i], acc);
        tri[1 + ch] = acc;
    }
    return 1;
}

/* accumulatedDensity += sigma * stepSize (RenderUtils.cu:1701). */
static inline double accd_add(double accd, float sigma, float step)
{
    if (g_contract & ORC_CONTRACT_ACCD) return fma((double)sigma, (double)step, accd);
    return accd + (double)(sigma * step);
}

/* ------------------------------------------------------ R7 forward */

static void forward_ray(const orc_scene* s, orc_rays* r, int ri, int* count)
{
    r->acc_den[ri] = 0.f;
    r->acc_w[ri] = 0.f;
    r->acc_r[ri] = 0.f;
    r->acc_g[ri] = 0.f;
    r->acc_b[ri] = 0.f;
    int n = 0;
    if (r->near_t[ri] > r->far_t[ri]) { /* RenderUtils.cu:1943-1946: no background */
        if (count) *count = 0;
        return;
    }
    const float dir[3] = {r->dx[ri], r->dy[ri], r->dz[ri]};
    float shs[25];
    orc_sh_basis(dir, shs);
    double t = (double)r->near_t[ri];
    const double far_t = (double)r->far_t[ri];
    double acc = 0., accd = 0.;
    float tri[4];
    int intT = 0;
    float acc_den = 0.f, acc_r = 0.f, acc_g = 0.f, acc_b = 0.f;
    while (t < far_t) {
        double bc[3];
        sample_position(s, r, ri, t, intT, bc);
        if (!trilerp_rgb(s, bc, shs, tri)) {
            t += (double)s->step;
            ++intT;
            continue;
        }
        const float sigma = orc_density_activation(tri[0]);
        const float c0 = orc_sigmoid(tri[1]);
        const float c1 = orc_sigmoid(tri[2]);
        const float c2 = orc_sigmoid(tri[3]);
        const double Ti = exp(-accd);
        const double w = Ti * (1. - (double)expf(-sigma * s->step));
        acc += w;
        acc_den += sigma;
        acc_r = (float)fma(w, (double)c0, (double)acc_r);
        acc_g = (float)fma(w, (double)c1, (double)acc_g);
        acc_b = (float)fma(w, (double)c2, (double)acc_b);
        accd = accd_add(accd, sigma, s->step);
        t += fabs((double)s->step - w);
        ++intT;
        ++n;
    }
    r->acc_den[ri] = acc_den;
    r->acc_w[ri] = (float)acc;
    if (r->white_bg) {
        acc_r = (float)((double)acc_r + (1. - acc));
        acc_g = (float)((double)acc_g + (1. - acc));
        acc_b = (float)((double)acc_b + (1. - acc));
    }
    r->acc_r[ri] = acc_r;
    r->acc_g[ri] = acc_g;
    r->acc_b[ri] = acc_b;
    if (count) *count = n;
}

void orc_render_forward(const orc_scene* s, orc_rays* r, const int* sample_index, int start,
                        int len, int* counts)
{
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int tid = 0; tid < len; tid++) {
        const int ri = sample_index ? sample_index[tid + start] : tid + start;
        forward_ray(s, r, ri, counts ? &counts[tid] : NULL);
    }
}

/* ------------------------------------------------------ R8 backward */

static inline void grad_add(double* p, double v)
{
#pragma omp atomic
    *p += v;
}

/* trilerpGradientsRGB (RenderUtils.cu:1074-1364): scatter one sample. */
static void scatter_sample(const orc_scene* s, const double bc[3], const float* shs,
                           const float g[4], double* grad)
{
    uint32_t bi[3] = {sat_u32(bc[0]), sat_u32(bc[1]), sat_u32(bc[2])};
    const double x = bc[0] - (double)bi[0];
    const double y = bc[1] - (double)bi[1];
    const double z = bc[2] - (double)bi[2];
    if (!occupied(s, bi)) return;
    const int64_t n = s->n_act;
    for (int q = 0; q < 8; q++) {
        const int64_t idx = corner_index(s, bi, q);
        const double c = corner_weight(q, x, y, z);
        grad_add(&grad[idx], (double)(float)((double)g[0] * c));
        for (int ch = 0; ch < 3; ch++) {
            int startk = ch * s->sh_dim + 1;
            int endk = startk + s->sh_dim;
            int shIdx = 0;
            if (s->hierarchy) {
                startk += s->band * s->band;
                endk -= (s->sh_dim - (s->band + 1) * (s->band + 1));
                shIdx += s->band * s->band;
            }
            for (int k = startk; k < endk; k++) {
                const float v = (float)((double)g[1 + ch] * c * (double)shs[shIdx]);
                grad_add(&grad[(int64_t)k * n + idx], (double)v);
                ++shIdx;
            }
        }
    }
}

static void backward_ray(const orc_scene* s, const orc_rays* r, int tid, int ri,
                         double mask_coef, float huber, double* losses, double* grad, int* count)
{
    const float dir[3] = {r->dx[ri], r->dy[ri], r->dz[ri]};
    float shs[25];
    orc_sh_basis(dir, shs);
    int n = 0;
    if (r->near_t[ri] > r->far_t[ri]) {
        losses[tid] = 0.;
        if (count) *count = 0;
        return;
    }
    double res[3] = {
        (double)r->acc_r[ri] - (double)r->r[ri] / 255.,
        (double)r->acc_g[ri] - (double)r->g[ri] / 255.,
        (double)r->acc_b[ri] - (double)r->b[ri] / 255.,
    };
    losses[tid] = (fabs(res[0]) + fabs(res[1]) + fabs(res[2])) * 255. / 3.;
    if (isnan(losses[tid])) {
        losses[tid] = 255.;
        if (count) *count = 0;
        return;
    }
    const double hd = (double)huber;
    for (int i = 0; i < 3; i++) {
        if (res[i] > hd)
            res[i] = fma(-(0.5 * hd), hd, hd);
        else if (res[i] < -hd)
            res[i] = fma(0.5 * hd, hd, -hd);
    }
    double t = (double)r->near_t[ri];
    const double far_t = (double)r->far_t[ri];
    double accd = 0., accw = 0.;
    double acc_rgb[3] = {0., 0., 0.};
    float tri[4], act[4], g[4];
    float mask_loss = 0.f;
    const float accw_f = r->acc_w[ri];
    if (r->mask[ri] && accw_f < 1.) {
        mask_loss = (float)(((double)r->mask[ri] / 255.0 - (double)accw_f) * mask_coef);
    }
    float wpre = (float)maxf_d(1e-6, (double)accw_f);
    wpre = (float)minf_d(1 - 1e-6, (double)wpre);
    mask_loss = (float)fma((double)logf(wpre) - log(1. - (double)wpre), 1e-3, (double)mask_loss);
    int intT = 0;
    const double pred[3] = {(double)r->acc_r[ri], (double)r->acc_g[ri], (double)r->acc_b[ri]};
    while (t < far_t) {
        double bc[3];
        sample_position(s, r, ri, t, intT, bc);
        if (!trilerp_rgb(s, bc, shs, tri)) {
            t += (double)s->step;
            ++intT;
            continue;
        }
        act[0] = orc_density_activation(tri[0]);
        act[1] = orc_sigmoid(tri[1]);
        act[2] = orc_sigmoid(tri[2]);
        act[3] = orc_sigmoid(tri[3]);
        double Ti = exp(-accd);
        const double w = Ti * (1. - (double)expf(-act[0] * s->step));
        accw += w;
        for (int c = 0; c < 3; c++) acc_rgb[c] = fma(w, (double)act[1 + c], acc_rgb[c]);
        for (int c = 0; c < 3; c++)
            g[1 + c] = (float)((double)0.6667f * w * res[c] * (double)orc_sigmoid_derivative(tri[1 + c]));
        accd = accd_add(accd, act[0], s->step);
        Ti = exp(-accd);
        g[0] = (float)(res[0] * fma(Ti, (double)act[1], -(pred[0] - acc_rgb[0])));
        g[0] = (float)fma(res[1], fma(Ti, (double)act[2], -(pred[1] - acc_rgb[1])), (double)g[0]);
        g[0] = (float)fma(res[2], fma(Ti, (double)act[3], -(pred[2] - acc_rgb[2])), (double)g[0]);
        const float dd = orc_density_derivation(tri[0]);
        g[0] = (float)((double)g[0] * (0.6667 * (double)s->step * (double)dd));
        g[0] = (float)fma((double)(s->step * dd) * (((double)accw_f - accw) - Ti), (double)mask_loss,
                          (double)g[0]);
        scatter_sample(s, bc, shs, g, grad);
        t += fabs((double)s->step - w);
        ++intT;
        ++n;
    }
    if (count) *count = n;
}

void orc_render_backward(const orc_scene* s, const orc_rays* r, const int* sample_index,
                         int start, int len, double mask_coef, float huber_delta,
                         double* losses, double* grad, int* counts)
{
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int tid = 0; tid < len; tid++) {
        const int ri = sample_index ? sample_index[tid + start] : tid + start;
        backward_ray(s, r, tid, ri, mask_coef, huber_delta, losses, grad,
                     counts ? &counts[tid] : NULL);
    }
}

/* ------------------------------------------------------ R9 TV */

/* getNeighboorGridIndexes (RenderUtils.cu:2549-2575). */
static void neighbour_indexes(const orc_scene* s, int cx, int cy, int cz, uint32_t res[27])
{
    for (int dz = -1; dz < 2; dz++)
        for (int dy = -1; dy < 2; dy++)
            for (int dx = -1; dx < 2; dx++) {
                uint32_t v = (uint32_t)scene_index(cx + dx, cy + dy, cz + dz, s->W, s->H, s->D);
                if (s->sparse) v = s->index_offsets[v];
                res[(dz + 1) * 9 + (dy + 1) * 3 + dx + 1] = v;
            }
}

/* One TV term (RenderUtils.cu:2755-2757): grad += coef / (sd + 1e-6) * disparity. */
static inline float tv_apply(float g, double coef, float sd, float disparity)
{
    return (float)fma(coef / ((double)sd + 1.e-6), (double)disparity, (double)g);
}

/* Six-neighbour term for one parameter array (RenderUtils.cu:2663-2757). */
static float tv6_value(const float* a, const uint32_t* ix, double coef, float g)
{
    static const int nb[6] = {4, 10, 12, 14, 16, 22};
    const float self = a[ix[13]];
    float sum = 0.f, disp = 0.f;
    for (int j = 0; j < 6; j++) {
        const float nv = ix[nb[j]] != 0 ? a[ix[nb[j]]] : self;
        const float d = self - nv;
        sum = fmaf(d, d, sum);
        disp = (j == 0) ? d : disp + d;
    }
    sum = sqrtf(sum) / 6.f;
    return tv_apply(g, coef, sum, disp);
}

static void tv_type0(const orc_scene* s, float* grad, double lam_d, double lam_sh, int nbrs)
{
    const int W = s->W, H = s->H, D = s->D;
    const int64_t n = s->n_act;
    const int startSH = s->hierarchy ? s->band * s->band : 0;
    const int endSH = (s->band + 1) * (s->band + 1);
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int pos = 0; pos < W * H; pos++) {
        const int row = pos / W, col = pos % W;
        if (row == 0 || row == H - 1 || col == 0 || col == W - 1) continue;
        uint32_t ix[27];
        if (nbrs == 3) {
            /* RenderUtils.cu:2606-2661 (depth from 0; disparity keeps the last term) */
            for (int depth = 0; depth < D - 1; depth++) {
                neighbour_indexes(s, col, row, depth, ix);
                if (s->sparse && !s->in_cage[ix[13]]) continue;
                {
                    const float* a = s->params;
                    const float self = a[ix[13]];
                    float sum = 0.f;
                    const float n14 = ix[14] != 0 ? a[ix[14]] : self;
                    sum = fmaf(self - n14, self - n14, sum);
                    const float n16 = ix[16] != 0 ? a[ix[16]] : self;
                    sum = fmaf(self - n16, self - n16, sum);
                    const float n22 = ix[22] != 0 ? a[ix[22]] : self;
                    const float disp = self - n22;
                    sum = fmaf(self - n22, self - n22, sum);
                    sum = sqrtf(sum) / 3.f;
                    grad[ix[13]] = tv_apply(grad[ix[13]], lam_d, sum, disp);
                }
                for (int ch = 0; ch < 3; ch++)
                    for (int k = ch * s->sh_dim + startSH; k < ch * s->sh_dim + endSH; k++) {
                        const float* a = s->params + (int64_t)(1 + k) * n;
                        float* gk = grad + (int64_t)(1 + k) * n;
                        const float self = a[ix[13]];
                        float sum = 0.f;
                        const float n14 = ix[14] != 0 ? a[ix[14]] : self;
                        sum = fmaf(self - n14, self - n14, sum);
                        const float n16 = ix[16] != 0 ? a[ix[16]] : self;
                        sum = fmaf(self - n16, self - n16, sum);
                        const float n22 = ix[4] != 0 ? a[ix[22]] : self;
                        const float disp = self - n22;
                        sum = fmaf(self - n22, self - n22, sum);
                        sum = sqrtf(sum) / 3.f;
                        gk[ix[13]] = tv_apply(gk[ix[13]], lam_sh, sum, disp);
                    }
            }
        } else if (nbrs == 6) {
            for (int depth = 1; depth < D - 1; depth++) {
                neighbour_indexes(s, col, row, depth, ix);
                if (s->sparse && !s->in_cage[ix[13]]) continue;
                grad[ix[13]] = tv6_value(s->params, ix, lam_d, grad[ix[13]]);
                for (int ch = 0; ch < 3; ch++)
                    for (int k = ch * s->sh_dim + startSH; k < ch * s->sh_dim + endSH; k++) {
                        const float* a = s->params + (int64_t)(1 + k) * n;
                        float* gk = grad + (int64_t)(1 + k) * n;
                        gk[ix[13]] = tv6_value(a, ix, lam_sh, gk[ix[13]]);
                    }
            }
        } else {
            /* 26 neighbours (RenderUtils.cu:2766-2812).  The SH disparity always reads
             * slot 4 of the neighbour array, which for the first four neighbours still
             * holds the previous array's value (density for the first SH array). */
            for (int depth = 1; depth < D - 1; depth++) {
                neighbour_indexes(s, col, row, depth, ix);
                if (s->sparse && !s->in_cage[ix[13]]) continue;
                float slot4 = 0.f;
                {
                    const float* a = s->params;
                    const float self = a[ix[13]];
                    float sum = 0.f, disp = 0.f;
                    for (int j = 0; j < 27; j++) {
                        if (j == 13) continue;
                        const float nv = ix[j] != 0 ? a[ix[j]] : self;
                        if (j == 4) slot4 = nv;
                        sum = fmaf(self - nv, self - nv, sum);
                        disp += self - nv;
                    }
                    sum = sqrtf(sum) / 26.f;
                    grad[ix[13]] = tv_apply(grad[ix[13]], lam_d, sum, disp);
                }
                for (int ch = 0; ch < 3; ch++)
                    for (int k = ch * s->sh_dim + startSH; k < ch * s->sh_dim + endSH; k++) {
                        const float* a = s->params + (int64_t)(1 + k) * n;
                        float* gk = grad + (int64_t)(1 + k) * n;
                        const float self = a[ix[13]];
                        float sum = 0.f, disp = 0.f;
                        for (int j = 0; j < 27; j++) {
                            if (j == 13) continue;
                            const float nv = ix[j] != 0 ? a[ix[j]] : self;
                            if (j == 4) slot4 = nv;
                            sum = fmaf(self - nv, self - nv, sum);
                            disp += self - slot4;
                        }
                        sum = sqrtf(sum) / 26.f;
                        gk[ix[13]] = tv_apply(gk[ix[13]], lam_sh, sum, disp);
                    }
            }
        }
    }
}

/* getVoxelGridIndexes (RenderUtils.cu:2442-2467). */
static void cell_corner_indexes(const orc_scene* s, int qx, int qy, int qz, uint32_t res[8])
{
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                uint32_t v = (uint32_t)scene_index(qx + dx, qy + dy, qz + dz, s->W, s->H, s->D);
                if (s->sparse) v = s->index_offsets[v];
                res[dz * 4 + dy * 2 + dx] = v;
            }
}

/* Voxel-disparity term, VarianceType 1 (RenderUtils.cu:2469-2547).  The reference
 * updates shared corners with unsynchronised += from neighbouring threads; the
 * oracle applies every update once, in column order (the race-free sum). */
static void tv_type1(const orc_scene* s, float* grad, double lam_d, double lam_sh)
{
    const int W = s->W, H = s->H, D = s->D;
    const int64_t n = s->n_act;
    const int startSH = s->hierarchy ? s->band * s->band : 0;
    const int endSH = (s->band + 1) * (s->band + 1);
    for (int pos = 0; pos < (W - 1) * (H - 1); pos++) {
        const int row = pos / (W - 1), col = pos % (W - 1);
        uint32_t ix[8];
        for (int depth = 0; depth < D - 1; depth++) {
            const int vi = scene_index(col, row, depth, W - 1, H - 1, D - 1);
            if (s->sparse && !s->occ[vi]) continue;
            cell_corner_indexes(s, col, row, depth, ix);
            if (s->optimize_step <= 1) {
                float mean[3][25];
                for (int k = startSH; k < endSH; k++) mean[0][k] = mean[1][k] = mean[2][k] = 0.f;
                for (int i = 0; i < 8; i++)
                    for (int k = startSH; k < endSH; k++)
                        for (int ch = 0; ch < 3; ch++) {
                            const float* a = s->params + (int64_t)(1 + ch * s->sh_dim + k) * n;
                            mean[ch][k] += a[ix[i]] / 8.f;
                        }
                for (int i = 0; i < 8; i++)
                    for (int k = startSH; k < endSH; k++)
                        for (int ch = 0; ch < 3; ch++) {
                            const int64_t arr = 1 + (int64_t)s->sh_dim * ch + k;
                            const float* a = s->params + arr * n;
                            float* gk = grad + arr * n;
                            gk[ix[i]] = (float)fma(lam_sh, (double)(a[ix[i]] - mean[ch][k]),
                                                   (double)gk[ix[i]]);
                        }
            }
            float sum = 0.f;
            for (int i = 0; i < 8; i++) sum += s->params[ix[i]];
            sum /= 8.f;
            for (int i = 0; i < 8; i++)
                grad[ix[i]] = (float)fma(lam_d, (double)(s->params[ix[i]] - sum), (double)grad[ix[i]]);
        }
    }
}

void orc_tv_grad(const orc_scene* s, float* grad, double lam_density, double lam_sh, int type,
                 int nbrs)
{
    if (type == 0) {
        tv_type0(s, grad, lam_density, lam_sh, nbrs);
    } else if (type == 1) {
        tv_type1(s, grad, lam_density, lam_sh);
    } else if (type == 2) {
        tv_type0(s, grad, lam_density, lam_sh, nbrs);
        tv_type1(s, grad, lam_density, lam_sh);
    }
}

/* ------------------------------------------------------ R10 Adam */

void orc_adam(orc_scene* s, float* grad, float* m, float* v, double lr, double sh_lr,
              int timestep)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1.e-6f;
    const int64_t n = s->n_act;
    const double bc1 = 1. - (double)powf(beta1, (float)timestep);
    const double bc2 = 1. - (double)powf(beta2, (float)timestep);
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int64_t p = 0; p < n; p++) {
        double lr_p = lr;
        if (!s->sparse && s->adaptive_lr) lr_p = lr * (double)s->adaptive_lr[p];
        {
            const float g = grad[p];
            m[p] = (float)fma(1. - (double)beta1, (double)g, (double)(beta1 * m[p]));
            v[p] = (float)fma((1. - (double)beta2) * (double)g, (double)g, (double)(beta2 * v[p]));
            const float cm = (float)((double)m[p] / bc1);
            const float cv = (float)((double)v[p] / bc2);
            const double temp = (double)s->params[p] - lr_p * (double)cm / (double)(sqrtf(cv) + eps);
            s->params[p] = temp < 0. ? 0.f : (float)temp;
            grad[p] = 0.f;
        }
        for (int ch = 0; ch < 3; ch++) {
            int startk = ch * s->sh_dim + 1;
            int endk = startk + s->sh_dim;
            if (s->hierarchy) {
                startk += s->band * s->band;
                endk -= (s->sh_dim - (s->band + 1) * (s->band + 1));
            }
            for (int k = startk; k < endk; k++) {
                const int64_t e = (int64_t)k * n + p;
                const float g = grad[e];
                m[e] = (float)fma(1. - (double)beta1, (double)g, (double)(beta1 * m[e]));
                v[e] = (float)fma((1. - (double)beta2) * (double)g, (double)g, (double)(beta2 * v[e]));
                const float cm = (float)((double)m[e] / bc1);
                const float cv = (float)((double)v[e] / bc2);
                s->params[e] = (float)((double)s->params[e] - sh_lr * (double)cm / (double)(sqrtf(cv) + eps));
                grad[e] = 0.f;
            }
        }
    }
}

/* ------------------------------------------------------ R3 occupancy */

/* occupiedVoxel (SceneUtils.cu:800-829): any corner density strictly above thresh. */
static int occupied_voxel(const float* dens, int W, int H, int D, int x, int y, int z, float thr)
{
    for (int dz = 0; dz <= 1; dz++)
        for (int dy = 0; dy <= 1; dy++)
            for (int dx = 0; dx <= 1; dx++)
                if (dens[grid_index_upper(x + dx, y + dy, z + dz, W, H, D)] > thr) return 1;
    return 0;
}

uint32_t orc_occupancy(const float* density, int W, int H, int D, float threshold,
                       uint8_t* occ, uint8_t* in_cage, uint32_t* index_offsets,
                       int64_t* dropped_writes)
{
    const int64_t N = (int64_t)W * H * D;
    int64_t dropped = 0;
    memset(in_cage, 0, (size_t)N);
    /* pruneScene (SceneUtils.cu:831-881) */
    for (int row = 0; row < H - 1; row++)
        for (int col = 0; col < W - 1; col++)
            for (int depth = 0; depth < D - 1; depth++) {
                const int64_t ci = (int64_t)depth * (W - 1) * (H - 1) + (int64_t)row * (W - 1) + col;
                if (!occupied_voxel(density, W, H, D, col, row, depth, threshold)) {
                    occ[ci] = 0;
                    continue;
                }
                occ[ci] = 1;
                in_cage[(int64_t)depth * W * H + (int64_t)row * W + col] = 1;
                if (depth == D - 2) in_cage[(int64_t)(D - 1) * W * H + (int64_t)row * W + col] = 1;
                if (row == H - 2) in_cage[(int64_t)depth * W * H + (int64_t)(H - 1) * W + col] = 1;
                if (col == W - 2) {
                    /* the reference writes depth*W*H + H*W + col + 1 here (SceneUtils.cu:872):
                     * vertex (W-1, 0, depth+1), at most (D-1)*W*H + W-1 < N */
                    const int64_t v = (int64_t)depth * W * H + (int64_t)H * W + col + 1;
                    if (v < N) in_cage[v] = 1;
                    else dropped++;
                }
            }
    /* getCagedNums (SceneUtils.cu:1081-1120) */
    uint32_t k = 0;
    for (int64_t v = 0; v < N; v++) index_offsets[v] = in_cage[v] ? k++ : 0u;
    if (dropped_writes) *dropped_writes = dropped;
    return k;
}

void orc_compact(const float* dense, int n_arrays, int64_t n_dense, const uint8_t* in_cage,
                 float* compact, int64_t n_compact)
{
    int64_t c = 0;
    for (int64_t v = 0; v < n_dense && c < n_compact; v++) {
        if (!in_cage[v]) continue;
        for (int a = 0; a < n_arrays; a++) compact[(int64_t)a * n_compact + c] = dense[(int64_t)a * n_dense + v];
        c++;
    }
}

/* ------------------------------------------------------ R13 image render */

/* getBound of the image path, all in double (RenderUtils.cu:34-97). */
static void image_ray(const double* alpha, const double* principle, const double* c2w,
                      const double* centre, const int* bbox, int row, int col, double info[5])
{
    const double xin[4] = {((double)col + 0.5 - principle[0]) / alpha[0],
                           ((double)row + 0.5 - principle[1]) / alpha[1], 1.0, 1.0};
    double sp[4];
    for (int r = 0; r < 4; r++) {
        sp[r] = 0.;
        for (int c = 0; c < 4; c++) sp[r] = fma(c2w[r * 4 + c], xin[c], sp[r]);
        sp[r] -= centre[r];
    }
    double sum = fma(sp[2], sp[2], fma(sp[0], sp[0], sp[1] * sp[1]));
    sum = sqrt(sum);
    sp[0] /= sum;
    sp[1] /= sum;
    sp[2] /= sum;
    double t[6] = {
        ((double)bbox[1] - centre[0]) / sp[0], ((double)bbox[0] - centre[0]) / sp[0],
        ((double)bbox[3] - centre[1]) / sp[1], ((double)bbox[2] - centre[1]) / sp[1],
        ((double)bbox[5] - centre[2]) / sp[2], ((double)bbox[4] - centre[2]) / sp[2],
    };
    double t_min = minf_d(t[0], t[1]);
    double t_max = maxf_d(t[0], t[1]);
    t_min = maxf_d(t_min, minf_d(t[2], t[3]));
    t_max = minf_d(t_max, maxf_d(t[2], t[3]));
    t_min = maxf_d(t_min, minf_d(t[4], t[5]));
    t_max = minf_d(t_max, maxf_d(t[4], t[5]));
    info[0] = t_min;
    info[1] = t_max;
    info[2] = sp[0];
    info[3] = sp[1];
    info[4] = sp[2];
}

void orc_render_image(const orc_scene* s, const double* alpha, const double* principle,
                      const double* c2w, const double* centre, const int* bbox, int width,
                      int height, int white_bg, float* rgb, uint8_t* rgb8, float* depth,
                      uint8_t* mask)
{
    const int64_t npix = (int64_t)width * height;
#pragma omp parallel for schedule(dynamic, 64) num_threads(orc_get_threads())
    for (int64_t p = 0; p < npix; p++) {
        const int row = (int)(p / width);
        const int col = (int)(p % height); /* the reference's column uses % height (RenderUtils.cu:1727) */
        float acc_rgb[3] = {0.f, 0.f, 0.f};
        float disp = 0.f;
        uint8_t px8[3] = {0, 0, 0};
        uint8_t m = 0;
        double info[5];
        image_ray(alpha, principle, c2w, centre, bbox, row, col, info);
        if (info[0] > info[1]) {
            px8[0] = px8[1] = px8[2] = 255;
            if (white_bg) acc_rgb[0] = acc_rgb[1] = acc_rgb[2] = 1.f;
        } else {
            const float dir[3] = {(float)info[2], (float)info[3], (float)info[4]};
            float shs[25];
            orc_sh_basis(dir, shs);
            double t = info[0], acc = 0., accd = 0.;
            float tri[4];
            while (t < info[1]) {
                double bc[3];
                for (int a = 0; a < 3; a++) bc[a] = fma(t, info[2 + a], centre[a]);
                if (!trilerp_rgb(s, bc, shs, tri)) {
                    t += (double)s->step;
                    continue;
                }
                const float sigma = orc_density_activation(tri[0]);
                const float c0 = orc_sigmoid(tri[1]), c1 = orc_sigmoid(tri[2]), c2 = orc_sigmoid(tri[3]);
                const double Ti = exp(-accd);
                const double w = Ti * (1. - (double)expf(-sigma * s->step));
                acc += w;
                disp = (float)fma(w, t, (double)disp);
                acc_rgb[0] = (float)fma(w, (double)c0, (double)acc_rgb[0]);
                acc_rgb[1] = (float)fma(w, (double)c1, (double)acc_rgb[1]);
                acc_rgb[2] = (float)fma(w, (double)c2, (double)acc_rgb[2]);
                accd = accd_add(accd, sigma, s->step);
                t += fabs((double)s->step - w);
            }
            /* (int)((c + 1. - acc) * 255 + 0.5) with the multiply-add fused (RenderUtils.cu:1565) */
            for (int c = 0; c < 3; c++) px8[c] = (uint8_t)(int)fma(((double)acc_rgb[c] + 1.) - acc, 255., 0.5);
            if (white_bg)
                for (int c = 0; c < 3; c++) acc_rgb[c] = (float)((double)acc_rgb[c] + (1. - acc));
            m = (uint8_t)(acc * 255);
        }
        if (rgb) for (int c = 0; c < 3; c++) rgb[(int64_t)c * npix + p] = acc_rgb[c];
        if (rgb8) for (int c = 0; c < 3; c++) rgb8[(int64_t)c * npix + p] = px8[c];
        if (depth) depth[p] = disp;
        if (mask) mask[p] = m;
    }
}

/* ------------------------------------------------------ R11 */

double orc_mse(const double* losses, int n)
{
    double res = 0.0;
    for (int i = 0; i < n; i++) res += losses[i] * losses[i];
    return res / n;
}

/* ------------------------------------------------------ testRender KAT */

void orc_composite_kat(const double* opacity, const double* colour, int n, const double* gt,
                       double* render_res, double* weights, double* opacity_grad,
                       double* colour_grad)
{
    double acc_op = 0., Ti;
    for (int c = 0; c < 3; c++) render_res[c] = 0.;
    for (int i = 0; i < n; i++) {
        Ti = exp(-acc_op);
        weights[i] = Ti * (1. - exp(-opacity[i] * 1.));
        acc_op += opacity[i] * 1.;
        for (int c = 0; c < 3; c++) render_res[c] += weights[i] * colour[c * n + i];
    }
    double acc_rr[3] = {0., 0., 0.};
    acc_op = 0.;
    for (int i = 0; i < n; i++) {
        opacity_grad[i] = 0.;
        for (int c = 0; c < 3; c++) colour_grad[c * n + i] = 0.;
    }
    for (int i = 0; i < n; i++) {
        Ti = exp(-acc_op);
        weights[i] = Ti * (1. - exp(-opacity[i] * 1.));
        acc_op += opacity[i] * 1.;
        for (int c = 0; c < 3; c++) {
            acc_rr[c] += weights[i] * colour[c * n + i];
            colour_grad[c * n + i] += 0.667 * (render_res[c] - gt[c]) * weights[i];
        }
        Ti = exp(-acc_op);
        for (int c = 0; c < 3; c++) {
            opacity_grad[i] += 0.667 * (render_res[c] - gt[c]) * 1. * Ti * colour[c * n + i];
            opacity_grad[i] -= 0.667 * (render_res[c] - gt[c]) * 1. * (render_res[c] - acc_rr[c]);
        }
    }
}

/* ------------------------------------------------------ FP64 oracle */

static void sh_basis64(const double d[3], double shs[9])
{
    shs[0] = 1.;
    shs[1] = d[1];
    shs[2] = d[2];
    shs[3] = d[0];
    shs[4] = d[0] * d[1];
    shs[5] = d[1] * d[2];
    shs[6] = 3. * d[2] * d[2] - 1.;
    shs[7] = d[0] * d[2];
    shs[8] = d[0] * d[0] - d[1] * d[1];
}

static inline double softplus64(double x) { return log(1. + exp(x - 13.)); }
static inline double softplus64_d(double x) { return 1. / (1. + exp(13. - x)); }
static inline double sigmoid64(double x) { return 1. / (1. + exp(-0.1 * x)); }

/* Raw density and raw colours at bc, all in double; 0 when the sparse occupancy skips. */
static int trilerp64(const orc_scene* s, const double bc[3], const double* shs, double tri[4],
                     double* wq, int64_t* iq)
{
    uint32_t bi[3] = {sat_u32(bc[0]), sat_u32(bc[1]), sat_u32(bc[2])};
    if (!occupied(s, bi)) return 0;
    const double x = bc[0] - (double)bi[0];
    const double y = bc[1] - (double)bi[1];
    const double z = bc[2] - (double)bi[2];
    const int nsh = n_active_sh(s);
    const int64_t n = s->n_act;
    tri[0] = tri[1] = tri[2] = tri[3] = 0.;
    for (int q = 0; q < 8; q++) {
        const int64_t idx = corner_index(s, bi, q);
        const double c = corner_weight(q, x, y, z);
        wq[q] = c;
        iq[q] = idx;
        tri[0] += c * (double)s->params[idx];
        for (int ch = 0; ch < 3; ch++)
            for (int i = 0; i < nsh; i++)
                tri[1 + ch] += c * (double)s->params[(int64_t)(1 + ch * s->sh_dim + i) * n + idx] * shs[i];
    }
    return 1;
}

/* FP32 march of the mixed forms on a sparse grid, at an empty cell: the whole steps that carry
 * the position bc out of that cell, or out of its 8x8x8 brick when the brick is empty
 * (bricks: one byte per brick). */
static int empty_steps64(const orc_bricks* bk, const double bc[3], const double d[3], double step)
{
    uint32_t bi[3] = {sat_u32(bc[0]), sat_u32(bc[1]), sat_u32(bc[2])};
    int kb[3];
    const int bn[3] = {bk->bx, bk->by, bk->bz};
    for (int a = 0; a < 3; a++) {
        kb[a] = (int)(bi[a] >> 3);
        if (kb[a] > bn[a] - 1) kb[a] = bn[a] - 1;
    }
    const int empty = !bk->bits[((int64_t)kb[2] * bk->by + kb[1]) * bk->bx + kb[0]];
    double ex = 3.0e38;
    for (int a = 0; a < 3; a++) {
        const double lo = empty ? 8.0 * kb[a] : (double)bi[a];
        const double hi = empty ? 8.0 * kb[a] + 8.0 : (double)bi[a] + 1.0;
        double e = ex;
        if (d[a] > 0.) e = (hi - bc[a]) / d[a];
        else if (d[a] < 0.) e = (lo - bc[a]) / d[a];
        if (e < ex) ex = e;
    }
    const double n = ceil(ex / step);
    return n < 1. ? 1 : (n > 1e6 ? 1000000 : (int)n);
}

/* The dense empty-cell map of the FP32 march: is the cell at bc open?  Cell coordinates as
 * the march truncates them, clamped to the cell range (getSceneIndex on cells). */
static int dense_open64(const orc_scene* s, const orc_bricks* bk, const double bc[3])
{
    if (!bk || !bk->cells || s->sparse) return 1;
    const int64_t cw = s->W - 1, ch = s->H - 1, cd = s->D - 1;
    int64_t c[3] = {(int64_t)sat_u32(bc[0]), (int64_t)sat_u32(bc[1]), (int64_t)sat_u32(bc[2])};
    const int64_t n[3] = {cw, ch, cd};
    for (int a = 0; a < 3; a++) c[a] = c[a] > n[a] - 1 ? n[a] - 1 : c[a];
    return bk->cells[(c[2] * ch + c[1]) * cw + c[0]] != 0;
}

static void ray64(const orc_scene* s, const orc_rays* r, const orc_bricks* bk, int tid, int ri, double mask_coef,
                  double huber, double* pred, double* accw_out, double* losses, double* grad)
{
    pred[3 * tid] = pred[3 * tid + 1] = pred[3 * tid + 2] = 0.;
    accw_out[tid] = 0.;
    losses[tid] = 0.;
    if (r->near_t[ri] > r->far_t[ri]) return;
    const double o[3] = {r->ox[ri], r->oy[ri], r->oz[ri]};
    const double d[3] = {r->dx[ri], r->dy[ri], r->dz[ri]};
    double shs[9];
    sh_basis64(d, shs);
    const double step = s->step;
    const double far_t = r->far_t[ri];
    /* forward */
    double t = r->near_t[ri], accd = 0., acc = 0., rgb[3] = {0., 0., 0.};
    double tri[4], wq[8];
    int64_t iq[8];
    while (t < far_t) {
        double bc[3];
        for (int a = 0; a < 3; a++) bc[a] = o[a] + t * d[a];
        if (!dense_open64(s, bk, bc) || !trilerp64(s, bc, shs, tri, wq, iq)) {
            t += bk && bk->bits ? empty_steps64(bk, bc, d, step) * step : step;
            continue;
        }
        const double sigma = softplus64(tri[0]);
        const double w = exp(-accd) * (1. - exp(-sigma * step));
        acc += w;
        for (int c = 0; c < 3; c++) rgb[c] += w * sigmoid64(tri[1 + c]);
        accd += sigma * step;
        t += fabs(step - w);
        if (bk && exp(-accd) < bk->t_stop) break;
    }
    const double bg = r->white_bg ? 1. - acc : 0.;
    for (int c = 0; c < 3; c++) pred[3 * tid + c] = rgb[c] + bg;
    accw_out[tid] = acc;
    /* backward (renderRays_withGradients_RGBGPU, RenderUtils.cu:2051-2256, in double) */
    const double gt[3] = {r->r[ri] / 255., r->g[ri] / 255., r->b[ri] / 255.};
    double res[3];
    for (int c = 0; c < 3; c++) res[c] = pred[3 * tid + c] - gt[c];
    losses[tid] = (fabs(res[0]) + fabs(res[1]) + fabs(res[2])) * 255. / 3.;
    if (isnan(losses[tid])) {
        losses[tid] = 255.;
        return;
    }
    for (int c = 0; c < 3; c++) {
        if (res[c] > huber)
            res[c] = huber - 0.5 * huber * huber;
        else if (res[c] < -huber)
            res[c] = 0.5 * huber * huber - huber;
    }
    double mask_loss = 0.;
    if (r->mask[ri] && acc < 1.) mask_loss = (r->mask[ri] / 255. - acc) * mask_coef;
    double wpre = acc < 1e-6 ? 1e-6 : acc;
    wpre = wpre > 1 - 1e-6 ? 1 - 1e-6 : wpre;
    mask_loss += (log(wpre) - log(1. - wpre)) * 1e-3;
    const int64_t n = s->n_act;
    const int nsh = n_active_sh(s);
    t = r->near_t[ri];
    accd = 0.;
    double accw = 0., acc_rgb[3] = {0., 0., 0.};
    while (t < far_t) {
        double bc[3];
        for (int a = 0; a < 3; a++) bc[a] = o[a] + t * d[a];
        if (!dense_open64(s, bk, bc) || !trilerp64(s, bc, shs, tri, wq, iq)) {
            t += bk && bk->bits ? empty_steps64(bk, bc, d, step) * step : step;
            continue;
        }
        const double sigma = softplus64(tri[0]);
        const double w = exp(-accd) * (1. - exp(-sigma * step));
        accw += w;
        double col[3], g[4];
        for (int c = 0; c < 3; c++) {
            col[c] = sigmoid64(tri[1 + c]);
            acc_rgb[c] += w * col[c];
            g[1 + c] = 0.6667 * w * res[c] * 0.1 * col[c] * (1. - col[c]);
        }
        accd += sigma * step;
        const double Tn = exp(-accd);
        g[0] = 0.;
        for (int c = 0; c < 3; c++) g[0] += res[c] * (Tn * col[c] - (pred[3 * tid + c] - acc_rgb[c]));
        const double dd = softplus64_d(tri[0]);
        g[0] *= 0.6667 * step * dd;
        g[0] += step * dd * (acc - accw - Tn) * mask_loss;
        for (int q = 0; q < 8; q++) {
            const int64_t idx = iq[q];
            grad_add(&grad[idx], g[0] * wq[q]);
            for (int ch = 0; ch < 3; ch++) {
                int k0 = 0, k1 = s->sh_dim;
                if (s->hierarchy) {
                    k0 = s->band * s->band;
                    k1 = nsh;
                }
                for (int k = k0; k < k1; k++)
                    grad_add(&grad[(int64_t)(1 + ch * s->sh_dim + k) * n + idx], g[1 + ch] * wq[q] * (k < 9 ? shs[k] : 0.));
            }
        }
        t += fabs(step - w);
        if (bk && Tn < bk->t_stop) break;
    }
}

void orc64_forward_backward(const orc_scene* s, const orc_rays* r, const orc_bricks* bricks, int start,
                            int len, double mask_coef, double huber, double* pred, double* accw,
                            double* losses, double* grad)
{
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int tid = 0; tid < len; tid++)
        ray64(s, r, bricks, tid, tid + start, mask_coef, huber, pred, accw, losses, grad);
}

void orc64_tv6(const orc_scene* s, const double* params, double* grad, double lam_d, double lam_sh)
{
    const int64_t n = s->n_act;
    const int W = s->W, H = s->H, D = s->D;
    const int nsh = n_active_sh(s);
    const int lo = s->hierarchy ? s->band * s->band : 0;
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int64_t dv = 0; dv < (int64_t)W * H * D; dv++) {
        const int x = (int)(dv % W), y = (int)((dv / W) % H), z = (int)(dv / ((int64_t)W * H));
        if (x < 1 || x > W - 2 || y < 1 || y > H - 2 || z < 1 || z > D - 2) continue;
        int64_t self = dv;
        int64_t nb[6] = {dv - (int64_t)W * H, dv - W, dv - 1, dv + 1, dv + W, dv + (int64_t)W * H};
        if (s->sparse) {
            if (!s->in_cage[dv]) continue;
            self = s->index_offsets[dv];
            /* the reference gates sparse TV with inCageInfo[indexOffsets[v]] */
            if (!s->in_cage[self]) continue;
            for (int k = 0; k < 6; k++) {
                const uint32_t ci = s->index_offsets[nb[k]];
                nb[k] = ci == 0 ? self : (int64_t)ci;
            }
        }
        for (int e = 0; e < 1 + 3 * s->sh_dim; e++) {
            double lam = lam_d;
            if (e > 0) {
                const int k = (e - 1) % s->sh_dim;
                if (k < lo || k >= nsh) continue;
                lam = lam_sh;
            }
            const double v = params[(int64_t)e * n + self];
            double sum = 0., disp = 0.;
            for (int k = 0; k < 6; k++) {
                const double dlt = v - params[(int64_t)e * n + nb[k]];
                sum += dlt * dlt;
                disp += dlt;
            }
            grad[(int64_t)e * n + self] += lam * disp / (sqrt(sum) / 6. + 1e-6);
        }
    }
}

void orc64_adam(const orc_scene* s, double* params, double* grad, double* m, double* v,
                double lr, double sh_lr, int timestep)
{
    const double b1 = 0.9, b2 = 0.999, eps = 1e-6;
    const int64_t n = s->n_act;
    const int na = 1 + 3 * s->sh_dim;
    const int nsh = n_active_sh(s);
    const double bc1 = 1. - pow(b1, timestep), bc2 = 1. - pow(b2, timestep);
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int64_t p = 0; p < n; p++) {
        for (int e = 0; e < na; e++) {
            if (e > 0 && s->hierarchy) {
                const int k = (e - 1) % s->sh_dim;
                if (k < s->band * s->band || k >= nsh) continue;
            }
            const int64_t i = (int64_t)e * n + p;
            const double g = grad[i];
            m[i] = b1 * m[i] + (1. - b1) * g;
            v[i] = b2 * v[i] + (1. - b2) * g * g;
            double lrp = e == 0 ? lr : sh_lr;
            if (e == 0 && !s->sparse && s->adaptive_lr) lrp *= s->adaptive_lr[p];
            double np = params[i] - lrp * (m[i] / bc1) / (sqrt(v[i] / bc2) + eps);
            if (e == 0 && np < 0.) np = 0.;
            params[i] = np;
            grad[i] = 0.;
        }
    }
}

/* ------------------------------------------------------ coarse-to-fine upsampling */

/* getIndex (SceneUtils.cu:250-260): clamped from above only. */
static inline int64_t up_index(int col, int row, int depth, int W, int H, int D)
{
    col = col < W ? col : W - 1;
    row = row < H ? row : H - 1;
    depth = depth < D ? depth : D - 1;
    return (int64_t)depth * W * H + (int64_t)row * W + col;
}

void orc_upsample(const orc_scene* s, int dW, int dH, int dD, int dst_sh, float threshold,
                  int low_band_only, float* dst)
{
    const int64_t n = (int64_t)dW * dH * dD;
    const int64_t na = s->n_act;
    const int sh = s->sh_dim;
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int64_t p = 0; p < n; p++) {
        const int col = (int)(p % dW), row = (int)((p / dW) % dH), depth = (int)(p / ((int64_t)dW * dH));
        /* pixelCol * 1.f * src.sceneWidth / dest.sceneWidth, in float */
        const float bc[3] = {(float)col * 1.f * (float)s->W / (float)dW, (float)row * 1.f * (float)s->H / (float)dH,
                             (float)depth * 1.f * (float)s->D / (float)dD};
        const uint32_t b[3] = {(uint32_t)bc[0], (uint32_t)bc[1], (uint32_t)bc[2]};
        float tri[1 + 3 * 25];
        for (int i = 0; i < 1 + 3 * sh; i++) tri[i] = 0.f;
        int val = 1;
        if (s->sparse) val = s->occ[up_index((int)b[0], (int)b[1], (int)b[2], s->W - 1, s->H - 1, s->D - 1)] != 0;
        if (val) {
            const double x = (double)(bc[0] - (float)b[0]);
            const double y = (double)(bc[1] - (float)b[1]);
            const double z = (double)(bc[2] - (float)b[2]);
            const int nsh = low_band_only ? 1 : sh;
            for (int q = 0; q < 8; q++) {
                int64_t idx = up_index((int)(b[0] + k_corner[q][0]), (int)(b[1] + k_corner[q][1]),
                                       (int)(b[2] + k_corner[q][2]), s->W, s->H, s->D);
                if (s->sparse) idx = s->index_offsets[idx];
                const double c = corner_weight(q, x, y, z);
                tri[0] = (float)fma(c, (double)s->params[idx], (double)tri[0]);
                for (int i = 0; i < nsh; i++)
                    for (int ch = 0; ch < 3; ch++) {
                        const int e = 1 + ch * sh + i;
                        tri[e] = (float)fma(c, (double)s->params[(int64_t)e * na + idx], (double)tri[e]);
                    }
            }
        }
        dst[p] = (!val || tri[0] < threshold) ? 0.f : tri[0];
        const int nw = low_band_only ? 1 : sh;
        for (int i = 0; i < nw; i++)
            for (int ch = 0; ch < 3; ch++)
                dst[(int64_t)(1 + ch * dst_sh + i) * n + p] = tri[1 + ch * sh + i];
    }
}


/* ------------------------------------------------------------------ carving, bounding box */
/* The device's double -> int conversion (cvt.rzi.s32.f64): truncation, saturating, NaN -> 0. */
static int sat_i32(double v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int)-2147483647 - 1;
    return (int)v;
}

/* silhouetteCarving (SVRF/RenderUtils.cu:181-254); projectWorld2Image (:120-132) accumulates
 * each image coordinate with fused multiply-adds from 0, as nvcc compiles it. */
void orc_carve_silhouette(float* density, float* lr, int W, int H, int D, const double* P, int img_w,
                          int img_h, const uint8_t* red, const uint8_t* green, const uint8_t* blue,
                          const uint8_t* mask, int radius)
{
    const int64_t WH = (int64_t)W * H;
#pragma omp parallel for schedule(static)
    for (int64_t pix = 0; pix < WH; pix++) {
        const int row = (int)(pix / W), col = (int)(pix % W);
        for (int depth = 0; depth < D; depth++) {
            const double world[4] = {col + 0.5, row + 0.5, (double)depth, 1.};
            double image[3];
            for (int r = 0; r < 3; r++) {
                image[r] = 0.;
                for (int c = 0; c < 4; c++) image[r] = fma(P[r * 4 + c], world[c], image[r]);
            }
            image[0] /= image[2];
            image[1] /= image[2];
            const int imageRow = sat_i32(image[1]), imageCol = sat_i32(image[0]);
            int save = 0;
            for (int nr = -radius; nr < radius + 1 && !save; nr++) {
                const double pr = (double)imageRow + nr;
                for (int nc = -radius; nc < radius + 1; nc++) {
                    const double pc = (double)imageCol + nc;
                    if (pc < 0 || pc >= img_w || pr < 0 || pr >= img_h) continue;
                    const int p = sat_i32(pr * img_w + pc);
                    if ((mask && mask[p]) || red[p] || green[p] || blue[p]) {
                        save = 1;
                        break;
                    }
                }
            }
            if (!save) {
                const int64_t v = depth * WH + pix;
                density[v] = 0.f;
                lr[v] = 0.f;
            }
        }
    }
}

/* getBoundingBoxZ (RenderUtils.cu:256-286), getMaxRadius (:288-321) and the host reduction
 * (:351-464); the radius terms compile to fused multiply-adds on the device. */
double orc_bbox(const float* lr, int W, int H, int D, int* bbox)
{
    const int64_t WH = (int64_t)W * H;
    int b[6] = {W, -1, H, -1, D, -1};
    double best = 0.;
    for (int64_t pix = 0; pix < WH; pix++) {
        const int row = (int)(pix / W), col = (int)(pix % W);
        int depth = 0;
        while (lr[depth * WH + pix] < 1e-6 && depth + 1 < D) ++depth;
        const int rmin = depth;
        int rmax = depth;
        while (depth + 1 < D) {
            ++depth;
            if (lr[depth * WH + pix] > 1e-6) rmax = depth;
        }
        if (rmin != depth) {
            if (col < b[0]) b[0] = col;
            if (col > b[1]) b[1] = col;
            if (row < b[2]) b[2] = row;
            if (row > b[3]) b[3] = row;
            if (rmin < b[4]) b[4] = rmin;
            if (rmax > b[5]) b[5] = rmax;
        }
        const double dr = row - H / 2., dc = col - W / 2.;
        const double temp = fma(dr, dr, dc * dc);
        for (int d = 0; d < D; d++) {
            if (lr[d * WH + pix] > 1e-6) {
                const double dd = d - D / 2.;
                const double distance = sqrt(fma(dd, dd, temp));
                if (distance > best) best = distance;
            }
        }
    }
    for (int i = 0; i < 6; i++) bbox[i] = b[i];
    return best / W * 2.;
}

/* ---------------------------------------------------------------- jitter (R12) */
/* Standard normal quantile from the mathematics: the root of 0.5 erfc(z / sqrt 2) = q for the
 * upper tail (q <= 0.5, z >= 0), by Newton's method on libm's erfc, which keeps relative
 * accuracy in the tail.  Returns z with P(Z > z) = q. */
static double upper_quantile(double q)
{
    const double pi = 3.14159265358979323846, sqrt2 = 1.41421356237309504880;
    if (q >= 0.5) return 0.;
    /* start from the tail expansion z ~ sqrt(-2 ln q) - (ln(-2 ln q) + ln 4pi) / (2 sqrt(-2 ln q)) */
    const double l = sqrt(-2. * log(q));
    double z = q < 0.3 ? l - (log(l * l) + log(4. * pi)) / (2. * l) : 0.;
    if (z < 0.) z = 0.;
    for (int it = 0; it < 100; it++) {
        const double f = 0.5 * erfc(z / sqrt2) - q;
        const double pdf = exp(-0.5 * z * z) / sqrt(2. * pi);
        const double dz = f / pdf;
        z += dz;
        if (fabs(dz) <= 1e-17 * (1. + fabs(z))) break;
    }
    return z;
}

/* randGPU(dest, len, radius, 1) (SVRF/Utils.cu:1002-1044) restated.  Generator state i < min(len,
 * 20000) is dimension i of the scrambled Sobol sequence with direction numbers dirs[i][0..63]
 * and scramble word scramble32[i] (the reference copies the 64-bit constants into a 32-bit
 * array), started at point i + first.  Point n of a dimension is, in the Gray-code form of
 * Antonov and Saleev, x_n = c XOR (XOR of v_b over the set bits b of n ^ (n >> 1)); state i's
 * j-th draw is point i + first + j.  A 64-bit point x becomes N(0,1) through the inverse
 * normal CDF at the centre of its cell, p = (x + 1/2) / 2^64 (mirrored as 1 - p above one
 * half so the tail keeps its precision).  Offset k = draw k / 20000 of state k % 20000, times
 * radius / 4; only the entries the reference's square grid of 32x32 blocks reaches are
 * written (the rest keep their value). */
void orc_sobol_offsets(const uint64_t* dirs, const uint32_t* scramble32, int len, uint64_t first, double radius,
                       double* out)
{
    const int n_states = len < 20000 ? len : 20000;
    const int square = (int)(sqrt(len * 1.0) + 0.5);
    const int64_t side = (square + 31) / 32;
    const int64_t reach = side * side * 1024;
    const int n_write = reach < len ? (int)reach : len;
    for (int k = 0; k < n_write; k++) {
        const int i = k % 20000;
        if (i >= n_states) continue;
        const uint64_t n = (uint64_t)i + first + (uint64_t)(k / 20000);
        const uint64_t gray = n ^ (n >> 1);
        uint64_t x = (uint64_t)scramble32[i];
        for (int b = 0; b < 64; b++)
            if ((gray >> b) & 1u) x ^= dirs[(size_t)i * 64 + b];
        double z;
        if (x >> 63) {
            const uint64_t m = ~x; /* 2^64 - 1 - x */
            z = upper_quantile(((double)m + 0.5) * 0x1p-64);
        } else {
            z = -upper_quantile(((double)x + 0.5) * 0x1p-64);
        }
        out[k] = z / 4. * radius + 0.;
    }
}
