/*
 * twisty_oracle.c -- CPU oracle for the path-integral Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see twisty_oracle.h): the checker, never the product.
 * Compiled by oracle/Makefile with -ffp-contract=off -mno-fma so that every float
 * expression below rounds exactly as written, left to right.
 *
 * Each function restates the reference function named in its comment (paths relative
 * to the reference repository root).
 */
#define _GNU_SOURCE
#include "twisty_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* Twisty/MathConsts.h:8 -- the reference's pi is a float constant. */
static const float TWISTY_PI_F = 3.141592653589793f;

/* ------------------------------------------------------------------------------------
 * Philox-4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as
 * 1, 2, 3", SC'11). Multipliers and Weyl key increments are the published constants.
 * ---------------------------------------------------------------------------------- */
void tor_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static inline uint32_t mulhi_u32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

/* One proposal per chain step, from Philox counter (step, chain, experiment, 'TWST') and
 * key (seed). Ranges follow the reference CPU runner
 * (Twisty/FullExperimentRunnerOptimalPerturb.cpp:483-490,501-502): sub-chain length
 * k in U{2..min(k_max, N-2)}, left index in U{1..N-k-1}, angle in U(-max_angle, max_angle)
 * (the reference fixes k_max = 25 and max_angle = pi). */
void tor_draw_step(uint64_t seed, uint32_t experiment, uint32_t chain, uint32_t step,
                   uint32_t n_segments, uint32_t k_max, float max_angle,
                   uint32_t *k, uint32_t *left, float *angle)
{
    const uint32_t ctr[4] = {step, chain, experiment, 0x54575354u};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t r[4];
    tor_philox4x32_10(ctr, key, r);
    uint32_t km = n_segments - 2;
    if (k_max < km) km = k_max;
    const uint32_t kk = 2u + mulhi_u32(r[0], km - 1u);
    *k = kk;
    *left = 1u + mulhi_u32(r[1], n_segments - kk - 1u);
    const float u = (float)(((int32_t)r[2]) >> 8) * 0x1p-23f + 0x1p-24f; /* open (-1, 1) */
    *angle = u * max_angle;
}

/* sin and cos of angle/2 for |angle| <= pi: Taylor polynomials to degree 13 / 14 in
 * Horner form with explicit fused multiply-adds, evaluated identically on CPU and GPU.
 * Truncation error at |angle/2| = pi/2 is below 7e-10, under half an FP32 ulp of 1. */
void tor_sincos_half(float angle, float *s, float *c)
{
    const float a = angle * 0.5f;
    const float z = a * a;
    float ps = 1.0f / 6227020800.0f;        /*  1/13! */
    ps = fmaf(ps, z, -1.0f / 39916800.0f);  /* -1/11! */
    ps = fmaf(ps, z, 1.0f / 362880.0f);     /*  1/9!  */
    ps = fmaf(ps, z, -1.0f / 5040.0f);      /* -1/7!  */
    ps = fmaf(ps, z, 1.0f / 120.0f);        /*  1/5!  */
    ps = fmaf(ps, z, -1.0f / 6.0f);         /* -1/3!  */
    *s = fmaf(a * z, ps, a);
    float pc = -1.0f / 87178291200.0f;      /* -1/14! */
    pc = fmaf(pc, z, 1.0f / 479001600.0f);  /*  1/12! */
    pc = fmaf(pc, z, -1.0f / 3628800.0f);   /* -1/10! */
    pc = fmaf(pc, z, 1.0f / 40320.0f);      /*  1/8!  */
    pc = fmaf(pc, z, -1.0f / 720.0f);       /* -1/6!  */
    pc = fmaf(pc, z, 1.0f / 24.0f);         /*  1/4!  */
    pc = fmaf(pc, z, -0.5f);                /* -1/2!  */
    *c = fmaf(z, pc, 1.0f);
}

/* ------------------------------------------------------------------------------------
 * Weight lookup table (Twisty/PathWeightUtils.cpp)
 * ---------------------------------------------------------------------------------- */
void tor_wparams_default(tor_wparams *wp, float mu, float eps, float scatter, float absorption,
                         uint32_t num_steps_int, uint32_t bins)
{
    wp->mu = mu;
    wp->eps = eps;
    wp->scatter = scatter;
    wp->absorption = absorption;
    wp->min_bound = 0.0f;
    wp->max_bound = 10.0f / eps; /* Twisty/ExperimentRunner.cpp:169-171 */
    wp->bias = 1.0f;
    wp->num_steps_int = num_steps_int;
    wp->num_curvature_steps = bins;
}

/* GaussianPhase + SimpleGaussianPhase (PathWeightUtils.cpp:19-33), in float. */
float tor_gaussian_phase_f32(float p, float m)
{
    const float np = sqrtf((TWISTY_PI_F * m) * 0.5f) / (1.0f - expf(-2.0f / m));
    const float val = (-m * p * p) * 0.5f;
    return np * expf(val);
}

/* IntegrandRT (PathWeightUtils.cpp:350-369). Parameter names are the reference's: the
 * caller passes config mu as `eps` and config eps as `mu` (PathWeightUtils.cpp:401). */
double tor_integrand_rt(double p, double kds, double bds, double eps, double mu)
{
    const double phase = (double)tor_gaussian_phase_f32((float)p, (float)mu);
    const double scattering = p * exp(bds * phase - 1.0 * (eps * eps * p * p * 0.5));
    double sin_term = p;
    if (kds > 0.0) sin_term = sin(kds * p) / kds;
    return scattering * sin_term;
}

static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* WeightLookupTableIntegral::Integrate (PathWeightUtils.cpp:371-433): composite Simpson
 * whose odd loop stops at index n-3 and even loop at n-4 (nodes n-2, n-1 dropped),
 * terms sorted ascending then summed in double, result cast to float. */
static float integrate_f32(float curvature, const tor_wparams *wp, float ds, double *scratch)
{
    const double kds = (double)(curvature * ds);
    const double bds = (double)(wp->scatter * ds);
    const uint32_t n = wp->num_steps_int;
    const double h = (double)((wp->max_bound - wp->min_bound) / (float)n);
    const double weight = (double)(1.0f / 3.0f) * h;
    const double start = (double)wp->min_bound;
    const double reg = (double)wp->mu, pm = (double)wp->eps;
    memset(scratch, 0, sizeof(double) * (n + 1));
    scratch[0] = tor_integrand_rt(start, kds, bds, reg, pm) * weight;
    scratch[n] = tor_integrand_rt((double)wp->max_bound, kds, bds, reg, pm) * weight;
    for (uint32_t i = 1; i < n / 2; ++i) {
        const double p = start + ((double)(2 * i - 1) * h);
        scratch[2 * i - 1] = tor_integrand_rt(p, kds, bds, reg, pm) * weight * 4.0;
    }
    for (uint32_t i = 1; i < n / 2 - 1; ++i) {
        const double p = start + ((double)(2 * i) * h);
        scratch[2 * i] = tor_integrand_rt(p, kds, bds, reg, pm) * weight * 2.0;
    }
    qsort(scratch, n + 1, sizeof(double), cmp_double);
    double sum = 0.0;
    for (uint32_t i = 0; i <= n; ++i) sum += scratch[i];
    const double tp = (double)TWISTY_PI_F;
    return (float)((sum / (2.0 * tp * tp)) * (double)wp->bias);
}

typedef struct {
    const tor_wparams *wp;
    float ds, step, min_k;
    float *lut;
    uint32_t i0, i1;
} lut32_job;

static void *lut32_worker(void *arg)
{
    lut32_job *j = (lut32_job *)arg;
    double *scratch = (double *)malloc(sizeof(double) * (j->wp->num_steps_int + 1));
    for (uint32_t i = j->i0; i < j->i1; ++i) {
        const float kappa = j->min_k + ((float)(int64_t)i * j->step);
        j->lut[i] = integrate_f32(kappa, j->wp, j->ds, scratch);
    }
    free(scratch);
    return NULL;
}

/* WeightLookupTableIntegral ctor + Initialize (PathWeightUtils.cpp:281-348). */
int tor_lut_build_f32(const tor_wparams *wp, float ds, float *lut, tor_lut_meta *meta, int n_threads)
{
    const uint32_t bins = wp->num_curvature_steps;
    if (bins < 2 || (wp->num_steps_int % 2) != 0 || wp->num_steps_int < 4 || !(ds > 0.0f)) return -1;
    const float min_k = 0.0f;
    const float max_k = (float)((2.0 / (double)ds) * (double)1.01f);
    const float step = (max_k - min_k) / (float)(bins - 1);
    if (n_threads < 1) n_threads = 1;
    if ((uint32_t)n_threads > bins) n_threads = (int)bins;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * n_threads);
    lut32_job *jobs = (lut32_job *)malloc(sizeof(lut32_job) * n_threads);
    for (int t = 0; t < n_threads; ++t) {
        jobs[t].wp = wp; jobs[t].ds = ds; jobs[t].step = step; jobs[t].min_k = min_k; jobs[t].lut = lut;
        jobs[t].i0 = (uint32_t)((uint64_t)bins * t / n_threads);
        jobs[t].i1 = (uint32_t)((uint64_t)bins * (t + 1) / n_threads);
        pthread_create(&th[t], NULL, lut32_worker, &jobs[t]);
    }
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    /* Entry 0 is Integrate(0.0f), identical to min_k + 0*step. */
    float mn = lut[0], mx = lut[0];
    for (uint32_t i = 1; i < bins; ++i) {
        const float v = lut[i];
        if (v < mn && v >= 0.0f) mn = v;
        if (v > mx && v >= 0.0f) mx = v;
    }
    for (uint32_t i = 0; i < bins; ++i)
        if (lut[i] <= 0.0f) lut[i] = mn;
    meta->min_k = min_k; meta->max_k = max_k; meta->step = step;
    meta->min_w = mn; meta->max_w = mx; meta->ds = ds;
    meta->bins = bins; meta->pad = 0;
    return 0;
}

/* FP64 twin of the table: the same node set and weights, double pi, phase function in
 * double, and a Neumaier-compensated sum in place of sort-then-sum. */
static double integrand_f64(double p, double kds, double bds, double reg, double m)
{
    const double np = sqrt((M_PI * m) * 0.5) / (1.0 - exp(-2.0 / m));
    const double phase = np * exp(-m * p * p * 0.5);
    const double scattering = p * exp(bds * phase - reg * reg * p * p * 0.5);
    return scattering * (kds > 0.0 ? sin(kds * p) / kds : p);
}

static double integrate_f64(double kappa, const tor_wparams *wp, double ds)
{
    const double kds = kappa * ds, bds = (double)wp->scatter * ds;
    const uint32_t n = wp->num_steps_int;
    const double maxb = 10.0 / (double)wp->eps;
    const double h = maxb / (double)n;
    const double reg = (double)wp->mu, m = (double)wp->eps;
    double s = 0.0, c = 0.0;
#define TOR_NEU(x)                                              \
    do {                                                        \
        const double _x = (x), _t = s + _x;                     \
        c += (fabs(s) >= fabs(_x)) ? (s - _t) + _x : (_x - _t) + s; \
        s = _t;                                                 \
    } while (0)
    TOR_NEU(integrand_f64(0.0, kds, bds, reg, m));
    TOR_NEU(integrand_f64(maxb, kds, bds, reg, m));
    for (uint32_t i = 1; i < n / 2; ++i) TOR_NEU(4.0 * integrand_f64((double)(2 * i - 1) * h, kds, bds, reg, m));
    for (uint32_t i = 1; i < n / 2 - 1; ++i) TOR_NEU(2.0 * integrand_f64((double)(2 * i) * h, kds, bds, reg, m));
#undef TOR_NEU
    return (s + c) * (h / 3.0) / (2.0 * M_PI * M_PI) * (double)wp->bias;
}

typedef struct {
    const tor_wparams *wp;
    double ds, step;
    double *lut;
    uint32_t i0, i1;
} lut64_job;

static void *lut64_worker(void *arg)
{
    lut64_job *j = (lut64_job *)arg;
    for (uint32_t i = j->i0; i < j->i1; ++i) j->lut[i] = integrate_f64((double)i * j->step, j->wp, j->ds);
    return NULL;
}

int tor_lut_build_f64(const tor_wparams *wp, double ds, double *lut, tor_lut_meta64 *meta, int n_threads)
{
    const uint32_t bins = wp->num_curvature_steps;
    if (bins < 2 || (wp->num_steps_int % 2) != 0 || wp->num_steps_int < 4 || !(ds > 0.0)) return -1;
    const double max_k = (2.0 / ds) * 1.01;
    const double step = max_k / (double)(bins - 1);
    if (n_threads < 1) n_threads = 1;
    if ((uint32_t)n_threads > bins) n_threads = (int)bins;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * n_threads);
    lut64_job *jobs = (lut64_job *)malloc(sizeof(lut64_job) * n_threads);
    for (int t = 0; t < n_threads; ++t) {
        jobs[t].wp = wp; jobs[t].ds = ds; jobs[t].step = step; jobs[t].lut = lut;
        jobs[t].i0 = (uint32_t)((uint64_t)bins * t / n_threads);
        jobs[t].i1 = (uint32_t)((uint64_t)bins * (t + 1) / n_threads);
        pthread_create(&th[t], NULL, lut64_worker, &jobs[t]);
    }
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    double mn = lut[0], mx = lut[0];
    for (uint32_t i = 1; i < bins; ++i) {
        if (lut[i] < mn && lut[i] >= 0.0) mn = lut[i];
        if (lut[i] > mx && lut[i] >= 0.0) mx = lut[i];
    }
    for (uint32_t i = 0; i < bins; ++i)
        if (lut[i] <= 0.0) lut[i] = mn;
    meta->min_k = 0.0; meta->max_k = max_k; meta->step = step;
    meta->min_w = mn; meta->max_w = mx; meta->ds = ds;
    meta->bins = bins; meta->pad = 0;
    return 0;
}

/* ------------------------------------------------------------------------------------
 * Curve operations (Twisty/CurvePerturbUtils.cpp)
 * ---------------------------------------------------------------------------------- */

/* RotateQuatByQuat (CurvePerturbUtils.cpp:91-111). */
static void quat_mul_f32(const float a[4], const float b[4], float r[4])
{
    const float t0 = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    const float t1 = a[0] * b[1] + a[1] * b[0] - a[2] * b[3] + a[3] * b[2];
    const float t2 = a[0] * b[2] + a[1] * b[3] + a[2] * b[0] - a[3] * b[1];
    const float t3 = a[0] * b[3] - a[1] * b[2] + a[2] * b[1] + a[3] * b[0];
    r[0] = t0; r[1] = t1; r[2] = t2; r[3] = t3;
}

/* RotateVectorByQuaternion (CurvePerturbUtils.cpp:113-127): q^-1 (x) (p (x) q). */
void tor_rotate_by_quat_f32(const float q[4], float v[3])
{
    float pq[4] = {0.0f, v[0], v[1], v[2]};
    const float inv[4] = {q[0], -q[1], -q[2], -q[3]};
    quat_mul_f32(pq, q, pq);
    quat_mul_f32(inv, pq, pq);
    v[0] = pq[1]; v[1] = pq[2]; v[2] = pq[3];
}

/* UpdateTangentsFromPos (CurvePerturbUtils.cpp:147-154); Normalized() as x*(1/sqrt(x.x)). */
void tor_tangents_f32(const float *pos, uint32_t n_segments, float *tan)
{
    for (uint32_t i = 0; i < n_segments; ++i) {
        const float dx = pos[3 * (i + 1) + 0] - pos[3 * i + 0];
        const float dy = pos[3 * (i + 1) + 1] - pos[3 * i + 1];
        const float dz = pos[3 * (i + 1) + 2] - pos[3 * i + 2];
        const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
        tan[3 * i + 0] = dx * inv;
        tan[3 * i + 1] = dy * inv;
        tan[3 * i + 2] = dz * inv;
    }
}

/* UpdateCurvaturesFromTangents_RadiativeTransfer (CurvePerturbUtils.cpp:157-166), with the
 * loop bound N-1 of its _CudaSafe twin (:219-243): kappa_i = |(t_{i+1} - t_i) * N/S|. */
void tor_curvatures_f32(const float *tan, uint32_t n_segments, float arclength, float *curv)
{
    const float inv_ds = (float)n_segments / arclength;
    for (uint32_t i = 0; i + 1 < n_segments; ++i) {
        const float x = (tan[3 * (i + 1) + 0] - tan[3 * i + 0]) * inv_ds;
        const float y = (tan[3 * (i + 1) + 1] - tan[3 * i + 1]) * inv_ds;
        const float z = (tan[3 * (i + 1) + 2] - tan[3 * i + 2]) * inv_ds;
        curv[i] = sqrtf(x * x + y * y + z * z);
    }
}

/* WeightCurveViaCurvatureLog10_CudaSafe (Twisty/PathWeighters.cpp:27-104). A NaN
 * curvature (degenerate segment) makes the path invalid here; the reference would cast
 * floor(NaN) to an index and read outside the table. bins[i] gets the left bin index.
 * Returns 1 for a valid path, 0 for an invalid one. */
int tor_weight_curvatures_f32(const float *curv, uint32_t n, const float *lut, const tor_lut_meta *m,
                              float absorption, double *log10w, int32_t *bins, uint32_t *n_clamped)
{
    *log10w = 0.0;
    if (!curv || n == 0) return 0;
    const double absorption_factor = (double)expf(-absorption * m->ds);
    const int32_t size = (int32_t)m->bins;
    const float mn = m->min_k, mx = m->max_k, step = m->step;
    double running = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        float c = curv[i];
        if (isnan(c)) return 0;
        if ((c < mn) && fabsf(c - mn) < 1e-3) c = mn;
        if ((c > mx) && fabsf(mx - c) < 1e-3) c = mx;
        if (c < mn) { c = mn; if (n_clamped) ++*n_clamped; }
        if (c > mx) { c = mx; if (n_clamped) ++*n_clamped; }
        const float dist = c - mn;
        const float real_idx = dist / step;
        const int32_t left = (int32_t)floorf(real_idx);
        int32_t right = left + 1;
        if (left == size - 1) right--;
        if (bins) bins[i] = left;
        const float lv = lut[left], rv = lut[right];
        const float interp = dist - ((float)left * step);
        double v = (double)(lv * (1.0f - interp) + (rv * interp));
        v *= absorption_factor;
        const double lg = log10(v);
        if (isnan(lg)) return 0;
        running += lg;
    }
    if (isnan(running)) return 0;
    *log10w = running;
    return 1;
}

int tor_weigh_paths_f32(const float *pos, uint64_t n_paths, uint32_t n_segments, float arclength,
                        const float *lut, const tor_lut_meta *m, float absorption,
                        double *log10w, uint8_t *valid, int32_t *bins, float *curv)
{
    if (n_segments < 2) return -1;
    float *tan = (float *)malloc(sizeof(float) * 3 * n_segments);
    float *cv = (float *)malloc(sizeof(float) * (n_segments - 1));
    for (uint64_t p = 0; p < n_paths; ++p) {
        const float *pp = pos + p * 3 * (uint64_t)(n_segments + 1);
        tor_tangents_f32(pp, n_segments, tan);
        tor_curvatures_f32(tan, n_segments, arclength, cv);
        double w = 0.0;
        const int ok = tor_weight_curvatures_f32(cv, n_segments - 1, lut, m, absorption, &w,
                                                 bins ? bins + p * (n_segments - 1) : NULL, NULL);
        log10w[p] = w;
        if (valid) valid[p] = (uint8_t)ok;
        if (curv) memcpy(curv + p * (n_segments - 1), cv, sizeof(float) * (n_segments - 1));
    }
    free(tan);
    free(cv);
    return 0;
}

/* FP64 twin of tangents, curvatures and the weigher (same algorithm, double throughout). */
static void tangents_f64(const double *pos, uint32_t n, double *tan)
{
    for (uint32_t i = 0; i < n; ++i) {
        const double dx = pos[3 * (i + 1) + 0] - pos[3 * i + 0];
        const double dy = pos[3 * (i + 1) + 1] - pos[3 * i + 1];
        const double dz = pos[3 * (i + 1) + 2] - pos[3 * i + 2];
        const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        tan[3 * i + 0] = dx * inv;
        tan[3 * i + 1] = dy * inv;
        tan[3 * i + 2] = dz * inv;
    }
}

static void curvatures_f64(const double *tan, uint32_t n, double arclength, double *curv)
{
    const double inv_ds = (double)n / arclength;
    for (uint32_t i = 0; i + 1 < n; ++i) {
        const double x = (tan[3 * (i + 1) + 0] - tan[3 * i + 0]) * inv_ds;
        const double y = (tan[3 * (i + 1) + 1] - tan[3 * i + 1]) * inv_ds;
        const double z = (tan[3 * (i + 1) + 2] - tan[3 * i + 2]) * inv_ds;
        curv[i] = sqrt(x * x + y * y + z * z);
    }
}

static int weight_curvatures_f64(const double *curv, uint32_t n, const double *lut, const tor_lut_meta64 *m,
                                 double absorption, double *log10w, int32_t *bins)
{
    *log10w = 0.0;
    if (n == 0) return 0;
    const double absorption_factor = exp(-absorption * m->ds);
    const int32_t size = (int32_t)m->bins;
    double running = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double c = curv[i];
        if (isnan(c)) return 0;
        if (c < m->min_k) c = m->min_k;
        if (c > m->max_k) c = m->max_k;
        const double dist = c - m->min_k;
        int32_t left = (int32_t)floor(dist / m->step);
        if (left > size - 1) left = size - 1;
        int32_t right = left + 1;
        if (left == size - 1) right = left;
        if (bins) bins[i] = left;
        const double interp = dist - (double)left * m->step;
        const double v = (lut[left] * (1.0 - interp) + lut[right] * interp) * absorption_factor;
        const double lg = log10(v);
        if (isnan(lg)) return 0;
        running += lg;
    }
    *log10w = running;
    return 1;
}

int tor_weigh_paths_f64(const double *pos, uint64_t n_paths, uint32_t n_segments, double arclength,
                        const double *lut, const tor_lut_meta64 *m, double absorption,
                        double *log10w, uint8_t *valid, int32_t *bins, double *curv)
{
    if (n_segments < 2) return -1;
    double *tan = (double *)malloc(sizeof(double) * 3 * n_segments);
    double *cv = (double *)malloc(sizeof(double) * (n_segments - 1));
    for (uint64_t p = 0; p < n_paths; ++p) {
        const double *pp = pos + p * 3 * (uint64_t)(n_segments + 1);
        tangents_f64(pp, n_segments, tan);
        curvatures_f64(tan, n_segments, arclength, cv);
        double w = 0.0;
        const int ok = weight_curvatures_f64(cv, n_segments - 1, lut, m, absorption, &w,
                                             bins ? bins + p * (n_segments - 1) : NULL);
        log10w[p] = w;
        if (valid) valid[p] = (uint8_t)ok;
        if (curv) memcpy(curv + p * (n_segments - 1), cv, sizeof(double) * (n_segments - 1));
    }
    free(tan);
    free(cv);
    return 0;
}

/* ------------------------------------------------------------------------------------
 * CombinedWeightValues_C (Twisty/CombinedWeightUtils.h:22-174)
 * ---------------------------------------------------------------------------------- */
#define TOR_MAX_DOUBLE_LOG10 300
#define TOR_MAX_PATHS_LOG10 6

void tor_cw_reset(tor_cw *c)
{
    c->n = 0;
    c->total = 0.0;
    c->offset = 0.0;
    c->max_log10 = 0.0;
    c->pad = 0;
}

void tor_cw_add(tor_cw *c, double v)
{
    if (c->n == 0) {
        c->max_log10 = v;
        c->offset = TOR_MAX_DOUBLE_LOG10 - (c->max_log10 + TOR_MAX_PATHS_LOG10);
        c->total += pow(10.0, (v + c->offset));
        c->n++;
        return;
    }
    if (c->max_log10 >= v) {
        c->total += pow(10.0, (v + c->offset));
        c->n++;
        return;
    }
    const double new_offset = TOR_MAX_DOUBLE_LOG10 - (v + TOR_MAX_PATHS_LOG10);
    const double delta = new_offset - c->offset;
    const double lt = log10(c->total);
    const double adj = lt + delta;
    c->total = pow(10.0, adj);
    c->max_log10 = v;
    c->offset = new_offset;
    c->total += pow(10.0, (v + c->offset));
    c->n++;
}

void tor_cw_combine(const tor_cw *a0, const tor_cw *b0, tor_cw *out)
{
    tor_cw a = *a0, b = *b0;
    if (a.n > 0 && b.n == 0) { *out = a; return; }
    if (b.n > 0 && a.n == 0) { *out = b; return; }
    if (b.max_log10 > a.max_log10) {
        tor_cw t = b;
        b = a;
        a = t;
    }
    tor_cw r;
    tor_cw_reset(&r);
    if (a.max_log10 == b.max_log10) {
        r.max_log10 = a.max_log10;
        r.n = a.n + b.n;
        r.offset = a.offset;
        r.total = a.total + b.total;
        *out = r;
        return;
    }
    const double delta = a.offset - b.offset;
    const double lb = log10(b.total);
    const double adj = lb + delta;
    const double nb = pow(10.0, adj);
    r.max_log10 = a.max_log10;
    r.n = a.n + b.n;
    r.offset = a.offset;
    r.total = a.total + nb;
    *out = r;
}

/* ExtractFinalValue (CombinedWeightUtils.h:160-174) returned as its log10. */
double tor_cw_extract_log10(const tor_cw *c)
{
    if (c->n == 0) return -INFINITY;
    return log10(c->total) - c->offset;
}

/* log10 of sum_i 10^v_i in long double (the reference sums extracted chunks in a
 * 100-digit decimal type: FullExperimentRunnerOptimalPerturb.cpp:347-378). */
double tor_log10_sum(const double *v, uint64_t n)
{
    double mx = -INFINITY;
    for (uint64_t i = 0; i < n; ++i)
        if (v[i] > mx) mx = v[i];
    if (mx == -INFINITY) return -INFINITY;
    long double s = 0.0L;
    for (uint64_t i = 0; i < n; ++i)
        if (v[i] > -INFINITY) s += powl(10.0L, (long double)v[i] - (long double)mx);
    return (double)((long double)mx + log10l(s));
}

/* ------------------------------------------------------------------------------------
 * Path normaliser (Twisty/PathWeightUtils.cpp:643-752). The reference accumulates in a
 * 100-digit decimal; long double stands in.
 * ---------------------------------------------------------------------------------- */
static long double k4_(float z, float ds)
{
    float result = (z < 2.0) ? 1.0f : 0.0f;
    result /= z;
    result = (float)((double)result * (2.0 * (double)TWISTY_PI_F));
    const float inv_ds = (float)(1.0 / (double)ds);
    result *= (inv_ds * inv_ds * inv_ds);
    return (long double)result;
}

static long double f5_(float x, float z, float ds)
{
    const float r = (float)sqrt((double)(z * z) + 1.0 - (2.0 * (double)z * (double)x));
    return k4_(r, ds);
}

static long double fn_(int order, float x, float z, float ds)
{
    if (order == 5) return f5_(x, z, ds);
    const float r = (float)sqrt((double)(z * z) + 1.0 - (2.0 * (double)z * (double)x));
    long double result = 0.0L;
    const uint32_t steps = 1000;
    const float xmin = -1.0f, xmax = 1.0f;
    const float dx = (xmax - xmin) / (float)steps;
    for (uint32_t i = 0; i < steps; ++i) {
        const float xv = xmin + (float)i * dx;
        result += fn_(order - 1, xv, r, ds);
    }
    result *= (long double)((2.0 * (double)TWISTY_PI_F) * (double)dx);
    return result;
}

/* K5..K10 all recurse through F7 (the macro at PathWeightUtils.cpp:705 names F##7). */
static long double kn_(double z, double ds)
{
    long double result = 0.0L;
    const uint32_t steps = 10000;
    const float xmin = -1.0f, xmax = 1.0f;
    const float dx = (xmax - xmin) / (float)steps;
    for (uint32_t i = 0; i < steps; ++i) {
        const float xv = xmin + (float)i * dx;
        result += fn_(7, xv, (float)z, (float)ds);
    }
    result *= (long double)((2.0 * (double)TWISTY_PI_F) * (double)dx);
    return result;
}

double tor_norm_log10(int n_segments, float ds, const float bc[12])
{
    const float inv = 1.0f / ds;
    float zx = (bc[6] - bc[0]) * inv, zy = (bc[7] - bc[1]) * inv, zz = (bc[8] - bc[2]) * inv;
    zx = zx - bc[9]; zy = zy - bc[10]; zz = zz - bc[11];
    zx = zx - bc[3]; zy = zy - bc[4]; zz = zz - bc[5];
    const float z = sqrtf(zx * zx + zy * zy + zz * zz);
    long double v;
    switch (n_segments) {
        case 4: v = k4_(z, ds); break;
        case 5:
        case 6: v = kn_((double)z, (double)ds); break;
        default: v = 1.0L; break;
    }
    return (double)log10l(v);
}

/* ------------------------------------------------------------------------------------
 * Markov chains: the per-thread loop of GeometryRandom
 * (Twisty/FullExperimentRunnerOptimalPerturb.cpp:469-595) with Philox proposals.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    int f64;
    const float *init_pos;
    uint32_t n;
    double arclength;
    const float *lut32;
    const tor_lut_meta *m32;
    const double *lut64;
    const tor_lut_meta64 *m64;
    double absorption;
    uint64_t seed;
    uint32_t experiment, chain0, c0, c1, steps, burn_in, k_max;
    float max_angle;
    double *path_log10;
    uint8_t *path_valid;
    double *chain_log10;
    uint64_t *chain_valid;
    float *final32;
    double *final64;
    const tor_chain_opts *opts;
} chain_job;

typedef struct {
    long double mx, s;
    uint64_t n;
} lse_acc;

static void lse_add(lse_acc *a, double v)
{
    const long double x = (long double)v;
    if (a->n == 0 || x > a->mx) {
        a->s = (a->n == 0 ? 0.0L : a->s * powl(10.0L, a->mx - x)) + 1.0L;
        a->mx = x;
    } else {
        a->s += powl(10.0L, x - a->mx);
    }
    a->n++;
}

static double lse_value(const lse_acc *a) { return a->n ? (double)(a->mx + log10l(a->s)) : -INFINITY; }

static void *chain_worker_f32(void *arg)
{
    chain_job *j = (chain_job *)arg;
    const uint32_t n = j->n;
    float *pos = (float *)malloc(sizeof(float) * 3 * (n + 1));
    float *tan = (float *)malloc(sizeof(float) * 3 * n);
    float *cv = (float *)malloc(sizeof(float) * (n - 1));
    for (uint32_t c = j->c0; c < j->c1; ++c) {
        memcpy(pos, j->init_pos, sizeof(float) * 3 * (n + 1));
        lse_acc acc = {0.0L, 0.0L, 0};
        const uint32_t total = j->burn_in + j->steps;
        for (uint32_t s = 0; s < total; ++s) {
            uint32_t k, left;
            float angle;
            tor_draw_step(j->seed, j->experiment, j->chain0 + c, s, n, j->k_max, j->max_angle, &k, &left, &angle);
            const uint32_t right = left + k;
            const float lx = pos[3 * left], ly = pos[3 * left + 1], lz = pos[3 * left + 2];
            const float dx = pos[3 * right] - lx, dy = pos[3 * right + 1] - ly, dz = pos[3 * right + 2] - lz;
            const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
            const float ax = dx * inv, ay = dy * inv, az = dz * inv;
            float sn, cs;
            tor_sincos_half(angle, &sn, &cs);
            const float q[4] = {cs, ax * sn, ay * sn, az * sn};
            for (uint32_t i = left + 1; i < right; ++i) {
                float v[3] = {pos[3 * i] - lx, pos[3 * i + 1] - ly, pos[3 * i + 2] - lz};
                tor_rotate_by_quat_f32(q, v);
                pos[3 * i] = v[0] + lx;
                pos[3 * i + 1] = v[1] + ly;
                pos[3 * i + 2] = v[2] + lz;
            }
            if (s < j->burn_in) continue;
            tor_tangents_f32(pos, n, tan);
            tor_curvatures_f32(tan, n, (float)j->arclength, cv);
            double w = 0.0;
            const int ok = tor_weight_curvatures_f32(cv, n - 1, j->lut32, j->m32, (float)j->absorption, &w, NULL, NULL);
            const uint64_t pi = (uint64_t)c * j->steps + (s - j->burn_in);
            if (j->path_log10) j->path_log10[pi] = w;
            if (j->path_valid) j->path_valid[pi] = (uint8_t)ok;
            if (ok) lse_add(&acc, w);
        }
        if (j->chain_log10) j->chain_log10[c] = lse_value(&acc);
        if (j->chain_valid) j->chain_valid[c] = acc.n;
        if (j->final32) memcpy(j->final32 + (uint64_t)c * 3 * (n + 1), pos, sizeof(float) * 3 * (n + 1));
    }
    free(pos);
    free(tan);
    free(cv);
    return NULL;
}

/* d log10 v / d kappa of the FP64 table's segment weight, as the adjoint defines it. The
 * reference's blend moves within a bin by (L_{b+1} - L_b) per unit of curvature (its
 * interpolation weight is in curvature units, PathWeighters.cpp:79-82) and jumps by nearly
 * L_{b+1} - L_b at every bin edge, so its pathwise derivative misses almost all of the change
 * that an expectation over paths sees. The adjoint takes the slope of the expected weight
 * instead: averaged over a bin, the staircase equals the linear interpolant of the table taken
 * half a bin to the left, whose slope at kappa is (L_{j+1} - L_j) / step with
 * j = floor(kappa / step - 1/2); divided by the weight itself. Clamped curvatures are flat. */
static double dlog10_dkappa_f64(double kappa, const double *lut, const tor_lut_meta64 *m)
{
    if (!(kappa >= m->min_k) || kappa > m->max_k) return 0.0;
    const int32_t size = (int32_t)m->bins;
    const double dist = kappa - m->min_k;
    int32_t left = (int32_t)floor(dist / m->step);
    if (left > size - 1) left = size - 1;
    const int32_t right = left == size - 1 ? left : left + 1;
    const double interp = dist - (double)left * m->step;
    const double v = lut[left] * (1.0 - interp) + lut[right] * interp;
    int32_t jl = (int32_t)floor(dist / m->step - 0.5);
    if (jl < 0) jl = 0;
    if (jl > size - 2) jl = size - 2;
    return (lut[jl + 1] - lut[jl]) / m->step / (v * M_LN10);
}

/* Receiver-position gradient of one path's log10 weight (FP64): moving points N-1 and N
 * together changes only the segment vector v_{N-2}, hence t_{N-2} and the curvatures
 * kappa_{N-3} = |t_{N-2} - t_{N-3}| N/S and kappa_{N-2} = |t_{N-1} - t_{N-2}| N/S. */
static void receiver_grad_f64(const double *pos, const double *tan, const double *cv, uint32_t n, double arclength,
                              const double *lut, const tor_lut_meta64 *m, double g[3])
{
    const double inv_ds = (double)n / arclength;
    const double *t3 = tan + 3 * (n - 3), *t2 = tan + 3 * (n - 2), *t1 = tan + 3 * (n - 1);
    const double vx = pos[3 * (n - 1)] - pos[3 * (n - 2)], vy = pos[3 * (n - 1) + 1] - pos[3 * (n - 2) + 1],
                 vz = pos[3 * (n - 1) + 2] - pos[3 * (n - 2) + 2];
    const double len2 = sqrt(vx * vx + vy * vy + vz * vz);
    g[0] = g[1] = g[2] = 0.0;
    for (int which = 0; which < 2; ++which) {
        double d[3];
        double sign;
        if (which == 0) { for (int q = 0; q < 3; ++q) d[q] = t2[q] - t3[q]; sign = 1.0; }
        else { for (int q = 0; q < 3; ++q) d[q] = t1[q] - t2[q]; sign = -1.0; }
        const double dn = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (!(dn > 0.0)) continue;
        const double dl = dlog10_dkappa_f64(cv[n - 3 + which], lut, m);
        const double dk = dl * inv_ds * sign / dn;
        const double dt = d[0] * t2[0] + d[1] * t2[1] + d[2] * t2[2];
        for (int q = 0; q < 3; ++q) g[q] += dk * (d[q] - dt * t2[q]) / len2;
    }
}

/* The FP64 twin chain: positions, rotation and weighting in double; the proposal
 * (k, left, angle) is the same Philox draw, its half-angle sine/cosine taken in double. */
static void *chain_worker_f64(void *arg)
{
    chain_job *j = (chain_job *)arg;
    const uint32_t n = j->n;
    double *pos = (double *)malloc(sizeof(double) * 3 * (n + 1));
    double *pw = (double *)malloc(sizeof(double) * 3 * (n + 1));
    double *tan = (double *)malloc(sizeof(double) * 3 * n);
    double *cv = (double *)malloc(sizeof(double) * (n - 1));
    const tor_chain_opts *o = j->opts;
    const int shift = o && o->has_shift;
    for (uint32_t c = j->c0; c < j->c1; ++c) {
        for (uint32_t i = 0; i < 3 * (n + 1); ++i) pos[i] = (double)j->init_pos[i];
        lse_acc acc = {0.0L, 0.0L, 0};
        long double gacc[4] = {0.0L, 0.0L, 0.0L, 0.0L};
        const uint32_t total = j->burn_in + j->steps;
        for (uint32_t s = 0; s < total; ++s) {
            uint32_t k, left;
            float angle;
            tor_draw_step(j->seed, j->experiment, j->chain0 + c, s, n, j->k_max, j->max_angle, &k, &left, &angle);
            const uint32_t right = left + k;
            const double lx = pos[3 * left], ly = pos[3 * left + 1], lz = pos[3 * left + 2];
            const double dx = pos[3 * right] - lx, dy = pos[3 * right + 1] - ly, dz = pos[3 * right + 2] - lz;
            const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
            const double ax = dx * inv, ay = dy * inv, az = dz * inv;
            const double ha = 0.5 * (double)angle;
            const double sn = sin(ha), cs = cos(ha);
            /* rotation matrix of the unit quaternion (cs, a*sn) applied as q^-1 p q */
            const double qw = cs, qx = ax * sn, qy = ay * sn, qz = az * sn;
            const double r00 = 1 - 2 * (qy * qy + qz * qz), r01 = 2 * (qx * qy - qw * qz), r02 = 2 * (qx * qz + qw * qy);
            const double r10 = 2 * (qx * qy + qw * qz), r11 = 1 - 2 * (qx * qx + qz * qz), r12 = 2 * (qy * qz - qw * qx);
            const double r20 = 2 * (qx * qz - qw * qy), r21 = 2 * (qy * qz + qw * qx), r22 = 1 - 2 * (qx * qx + qy * qy);
            for (uint32_t i = left + 1; i < right; ++i) {
                const double vx = pos[3 * i] - lx, vy = pos[3 * i + 1] - ly, vz = pos[3 * i + 2] - lz;
                pos[3 * i] = r00 * vx + r01 * vy + r02 * vz + lx;
                pos[3 * i + 1] = r10 * vx + r11 * vy + r12 * vz + ly;
                pos[3 * i + 2] = r20 * vx + r21 * vy + r22 * vz + lz;
            }
            if (s < j->burn_in) continue;
            const double *pe = pos;
            if (shift) {
                /* the weights see the receiver moved: points N-1 and N shifted, the chain unchanged */
                memcpy(pw, pos, sizeof(double) * 3 * (n + 1));
                for (uint32_t i = n - 1; i <= n; ++i)
                    for (int q = 0; q < 3; ++q) pw[3 * i + q] += o->eval_shift[q];
                pe = pw;
            }
            tangents_f64(pe, n, tan);
            curvatures_f64(tan, n, j->arclength, cv);
            double w = 0.0;
            const int ok = weight_curvatures_f64(cv, n - 1, j->lut64, j->m64, j->absorption, &w, NULL);
            const uint64_t pi = (uint64_t)c * j->steps + (s - j->burn_in);
            if (j->path_log10) j->path_log10[pi] = w;
            if (j->path_valid) j->path_valid[pi] = (uint8_t)ok;
            if (ok) lse_add(&acc, w);
            if (ok && o && o->grad_chains) {
                double g[3];
                receiver_grad_f64(pe, tan, cv, n, j->arclength, j->lut64, j->m64, g);
                const long double wt = powl(10.0L, (long double)w - (long double)o->ref_log10);
                for (int q = 0; q < 3; ++q) gacc[q] += wt * (long double)g[q];
                gacc[3] += wt;
            }
        }
        if (j->chain_log10) j->chain_log10[c] = lse_value(&acc);
        if (j->chain_valid) j->chain_valid[c] = acc.n;
        if (j->final64) memcpy(j->final64 + (uint64_t)c * 3 * (n + 1), pos, sizeof(double) * 3 * (n + 1));
        if (o && o->grad_chains)
            for (int q = 0; q < 4; ++q) o->grad_chains[(uint64_t)c * 4 + q] = (double)gacc[q];
    }
    free(pos);
    free(pw);
    free(tan);
    free(cv);
    return NULL;
}

static int run_chains(chain_job *proto, uint32_t n_chains, int n_threads)
{
    if (proto->n < 4) return -1;
    if (n_threads < 1) n_threads = 1;
    if ((uint32_t)n_threads > n_chains) n_threads = (int)(n_chains ? n_chains : 1);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * n_threads);
    chain_job *jobs = (chain_job *)malloc(sizeof(chain_job) * n_threads);
    for (int t = 0; t < n_threads; ++t) {
        jobs[t] = *proto;
        jobs[t].c0 = (uint32_t)((uint64_t)n_chains * t / n_threads);
        jobs[t].c1 = (uint32_t)((uint64_t)n_chains * (t + 1) / n_threads);
        pthread_create(&th[t], NULL, proto->f64 ? chain_worker_f64 : chain_worker_f32, &jobs[t]);
    }
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    return 0;
}

int tor_run_chains_f32(const float *init_pos, uint32_t n_segments, float arclength,
                       const float *lut, const tor_lut_meta *m, float absorption,
                       uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                       uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                       double *path_log10, uint8_t *path_valid, double *chain_log10,
                       uint64_t *chain_valid, float *final_pos, int n_threads)
{
    chain_job j;
    memset(&j, 0, sizeof(j));
    j.f64 = 0; j.init_pos = init_pos; j.n = n_segments; j.arclength = arclength;
    j.lut32 = lut; j.m32 = m; j.absorption = absorption; j.seed = seed;
    j.experiment = experiment; j.chain0 = chain0; j.steps = steps; j.burn_in = burn_in;
    j.k_max = k_max; j.max_angle = max_angle; j.path_log10 = path_log10; j.path_valid = path_valid;
    j.chain_log10 = chain_log10; j.chain_valid = chain_valid; j.final32 = final_pos;
    return run_chains(&j, n_chains, n_threads);
}

int tor_run_chains_f64_opts(const float *init_pos, uint32_t n_segments, double arclength,
                            const double *lut, const tor_lut_meta64 *m, double absorption,
                            uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                            uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                            double *chain_log10, uint64_t *chain_valid, const tor_chain_opts *opts,
                            int n_threads)
{
    if (n_segments < 4) return -1;
    chain_job j;
    memset(&j, 0, sizeof(j));
    j.f64 = 1; j.init_pos = init_pos; j.n = n_segments; j.arclength = arclength;
    j.lut64 = lut; j.m64 = m; j.absorption = absorption; j.seed = seed;
    j.experiment = experiment; j.chain0 = chain0; j.steps = steps; j.burn_in = burn_in;
    j.k_max = k_max; j.max_angle = max_angle;
    j.chain_log10 = chain_log10; j.chain_valid = chain_valid; j.opts = opts;
    return run_chains(&j, n_chains, n_threads);
}

int tor_run_chains_f64(const float *init_pos, uint32_t n_segments, double arclength,
                       const double *lut, const tor_lut_meta64 *m, double absorption,
                       uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                       uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                       double *path_log10, uint8_t *path_valid, double *chain_log10,
                       uint64_t *chain_valid, double *final_pos, int n_threads)
{
    chain_job j;
    memset(&j, 0, sizeof(j));
    j.f64 = 1; j.init_pos = init_pos; j.n = n_segments; j.arclength = arclength;
    j.lut64 = lut; j.m64 = m; j.absorption = absorption; j.seed = seed;
    j.experiment = experiment; j.chain0 = chain0; j.steps = steps; j.burn_in = burn_in;
    j.k_max = k_max; j.max_angle = max_angle; j.path_log10 = path_log10; j.path_valid = path_valid;
    j.chain_log10 = chain_log10; j.chain_valid = chain_valid; j.final64 = final_pos;
    return run_chains(&j, n_chains, n_threads);
}
