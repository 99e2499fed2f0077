// lut.cu -- weight lookup tables, built on the device in FP64.
//
// The reference builds its table with an OpenMP loop over bins, each bin a composite
// Simpson quadrature of IntegrandRT whose terms are sorted then summed
// (Twisty/PathWeightUtils.cpp:281-433). The faithful form and the derivative tables use one
// CTA per bin: every thread takes a strided share of the nodes and keeps a
// Neumaier-compensated FP64 sum, and the CTA combines the partial sums pairwise. The plain
// FP64 form (single tables and batches) uses lut_build_fast_kernel: one thread per bin over
// node weights shared by all bins (the integrand factors into a bin-independent weight times
// sin(kds p)). The compensated sums replace the sort (they are at least as accurate), so the
// float table matches the reference's to within one float ulp rather than bit for bit.
//
// The node set keeps the reference's rule exactly: weights h/3 * {1, 4, 2, ..., 4, 2, 1}
// with the odd loop ending at node n-3 and the even loop at n-4 (nodes n-2 and n-1 are
// dropped), and the config mu/eps swap of IntegrandRT's call (PathWeightUtils.cpp:401).
#include "kernels.h"
#include "device_common.cuh"

#include <cfloat>
#include <math_constants.h>

namespace twisty {
namespace {

constexpr int kLutThreads = 256;
// bins whose secant (fixed-point form) errs by more than this per segment are steep; a table
// with more than bins / kSteepFractionDev of them takes the exact blend (same rule on the host)
constexpr double kSecantBoundDev = 1e-7;
constexpr uint32_t kSteepFractionDev = 16;

struct Integrand {
    double kds, bds, reg, m;   // reg = config mu, m = config eps (phase parameter)
    int faithful;
    float np_f;                // float phase normaliser (faithful)
    double np_d, dlnnp_dm;     // double phase normaliser and its log-derivative in m
};

__device__ __forceinline__ double phase(const Integrand &g, double p)
{
    if (g.faithful) {
        // GaussianPhase / SimpleGaussianPhase in float (PathWeightUtils.cpp:19-33)
        const float pf = (float)p, mf = (float)g.m;
        const float val = __fmul_rn(__fmul_rn(__fmul_rn(-mf, pf), pf), 0.5f);
        return (double)__fmul_rn(g.np_f, expf(val));
    }
    return g.np_d * exp(-g.m * p * p * 0.5);
}

// f(p) = p exp(bds*phase(p) - reg^2 p^2/2) * sin(kds p)/kds   (IntegrandRT, :350-369)
__device__ __forceinline__ double integrand(const Integrand &g, double p)
{
    const double ph = phase(g, p);
    const double scattering = p * exp(g.bds * ph - 1.0 * (g.reg * g.reg * p * p * 0.5));
    return scattering * (g.kds > 0.0 ? sin(g.kds * p) / g.kds : p);
}

// Derivatives of f (double form): df/dbds, df/dp, df/dm.
__device__ __forceinline__ void integrand_derivs(const Integrand &g, double p, double &f, double &f_bds,
                                                 double &f_p, double &f_m)
{
    const double ph = g.np_d * exp(-g.m * p * p * 0.5);
    const double e = exp(g.bds * ph - g.reg * g.reg * p * p * 0.5);
    double s, sp;
    if (g.kds > 0.0) {
        double sn, cs;
        sincos(g.kds * p, &sn, &cs);
        s = sn / g.kds;
        sp = cs;
    } else {
        s = p;
        sp = 1.0;
    }
    f = p * e * s;
    f_bds = f * ph;
    const double ph_p = -g.m * p * ph;
    f_p = e * s + p * e * (g.bds * ph_p - g.reg * g.reg * p) * s + p * e * sp;
    const double ph_m = ph * (g.dlnnp_dm - 0.5 * p * p);
    f_m = f * g.bds * ph_m;
}

struct Neumaier {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x)
    {
        const double t = s + x;
        c += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// One bin of one table, integrated by the whole CTA.
__device__ __forceinline__ void build_bin(const LutBuildSpec &s, uint32_t bin, double *out64, double *d_mus,
                                          double *d_eps, double *red)
{
    const uint32_t n = s.num_steps_int;
    Integrand g;
    g.faithful = s.faithful;
    g.reg = (double)s.mu;
    g.m = (double)s.eps;
    double h, weight, start, maxb, tp;
    if (s.faithful) {
        const float kappa = __fadd_rn(s.min_k, __fmul_rn((float)bin, s.step));
        g.kds = (double)__fmul_rn(kappa, s.ds);
        g.bds = (double)__fmul_rn(s.scatter, s.ds);
        g.np_f = __fdiv_rn(__fsqrt_rn(__fmul_rn(__fmul_rn(dev::kPiF, s.eps), 0.5f)),
                           __fsub_rn(1.0f, expf(__fdiv_rn(-2.0f, s.eps))));
        h = (double)__fdiv_rn(__fsub_rn(s.max_bound, s.min_bound), (float)n);
        weight = (double)(1.0f / 3.0f) * h;
        start = (double)s.min_bound;
        maxb = (double)s.max_bound;
        tp = (double)dev::kPiF;
    } else {
        const double ds = (double)s.ds;
        g.kds = (double)bin * s.step64 * ds;
        g.bds = (double)s.scatter * ds;
        maxb = 10.0 / (double)s.eps;
        h = maxb / (double)n;
        weight = h / 3.0;
        start = 0.0;
        tp = CUDART_PI;
    }
    const double em = exp(-2.0 / g.m);
    g.np_d = sqrt((CUDART_PI * g.m) * 0.5) / (1.0 - em);
    g.dlnnp_dm = 0.5 / g.m - (2.0 / (g.m * g.m)) * em / (1.0 - em);

    Neumaier acc, acc_mus, acc_eps;
    for (uint32_t j = threadIdx.x; j <= n; j += blockDim.x) {
        double c;
        if (j == 0 || j == n) c = 1.0;
        else if (j >= n - 2) c = 0.0;            // dropped nodes n-2, n-1
        else c = (j & 1u) ? 4.0 : 2.0;
        if (c == 0.0) continue;
        const double p = (j == n) ? maxb : start + (double)j * h;
        if (s.derivatives && !s.faithful) {
            double f, f_bds, f_p, f_m;
            integrand_derivs(g, p, f, f_bds, f_p, f_m);
            acc.add(c * f);
            acc_mus.add(c * f_bds);
            acc_eps.add(c * (-p * f_p / g.m + f_m));
        } else {
            acc.add(integrand(g, p) * weight * c);
        }
    }
    const double total = block_sum(acc.value(), red);
    if (s.derivatives && !s.faithful) {
        const double t_mus = block_sum(acc_mus.value(), red);
        const double t_eps = block_sum(acc_eps.value(), red);
        if (threadIdx.x == 0) {
            const double scale = weight / (2.0 * tp * tp) * (double)s.bias;
            const double I = total * scale;
            out64[bin] = I;
            // d/d(mu_s): bds = mu_s * ds
            d_mus[bin] = t_mus * scale * (double)s.ds;
            // d/d(eps): h and every node move with maxBound = 10/eps
            d_eps[bin] = -I / g.m + t_eps * scale;
        }
    } else if (threadIdx.x == 0) {
        out64[bin] = (total / (2.0 * tp * tp)) * (double)s.bias;
    }
}

__global__ void __launch_bounds__(kLutThreads) lut_build_kernel(LutBuildSpec s, double *out64,
                                                                 double *d_mus, double *d_eps)
{
    __shared__ double red[kLutThreads / 32];
    build_bin(s, blockIdx.x, out64, d_mus, d_eps, red);
}

// The FP64 form without derivatives factors: node j contributes w_j sin(kds p_j) / kds with
// w_j = c_j (h/3) p_j exp(bds phase(p_j) - reg^2 p_j^2 / 2) the same for every bin. A CTA
// of kFastThreads threads covers that many consecutive bins of one table: it stages w_j for a
// chunk of nodes in shared memory and each thread sweeps its bin over the chunk, stepping
// (sin, cos)(kds j h) by the rotation through kds h and restarting from sincos every kRun
// nodes, so the phase drift stays at the level of the direct argument's own rounding
// (kds j h carries a relative error of one ulp either way). Runs are summed plainly and
// folded into a Neumaier total; node n (p = maxBound exactly) is added with a direct sin;
// bin 0 (kds = 0) takes the limit sin(kds p)/kds -> p. Against the per-node quadrature
// (lut_build_kernel) it replaces two exp and one sin per node and bin by five FMAs.
constexpr int kFastThreads = 128;
constexpr uint32_t kFastChunk = 1024;
constexpr uint32_t kRun = 64;

__device__ __forceinline__ void build_fast(const LutBuildSpec &s, uint32_t bin0, double *out64, double *sw)
{
    const uint32_t n = s.num_steps_int;
    const double m = (double)s.eps, reg = (double)s.mu;
    const double ds = (double)s.ds;
    const double bds = (double)s.scatter * ds;
    const double maxb = 10.0 / m;
    const double h = maxb / (double)n;
    const double weight = h / 3.0;
    const double np_d = sqrt((CUDART_PI * m) * 0.5) / (1.0 - exp(-2.0 / m));
    const uint32_t bin = bin0 + threadIdx.x;
    const double kds = (double)bin * s.step64 * ds;
    const bool zero_k = !(kds > 0.0);
    double st, ct;
    sincos(kds * h, &st, &ct);
    // Past p_cut the weight is exactly zero in FP64 (bds phase(p) <= bds np_d, so the exponent
    // is below -750 and exp underflows to 0): those nodes add nothing and are not visited.
    // With the regulariser of the usual configurations most of [0, 10/eps] lies there.
    uint32_t n_eff = n;
    if (reg > 0.0) {
        const double p_cut = sqrt(2.0 * (bds * np_d + 750.0)) / reg;
        const double j_cut = ceil(p_cut / h) + 2.0;
        if (j_cut < (double)n) n_eff = (uint32_t)j_cut;
    }
    Neumaier acc;
    for (uint32_t c0 = 0; c0 < n_eff; c0 += kFastChunk) {
        const uint32_t cn = min(kFastChunk, n_eff - c0);
        __syncthreads();   // the previous chunk is consumed
        for (uint32_t i = threadIdx.x; i < cn; i += blockDim.x) {
            const uint32_t j = c0 + i;
            const double c = (j == 0) ? 1.0 : (j >= n - 2) ? 0.0 : ((j & 1u) ? 4.0 : 2.0);
            const double p = (double)j * h;
            const double ph = np_d * exp(-m * p * p * 0.5);
            sw[i] = (p * exp(bds * ph - reg * reg * p * p * 0.5)) * weight * c;
        }
        __syncthreads();
        if (zero_k) {
            double run = 0.0;
            for (uint32_t i = 0; i < cn; ++i) run = fma(sw[i], (double)(c0 + i) * h, run);
            acc.add(run);
        } else {
            for (uint32_t r0 = 0; r0 < cn; r0 += kRun) {
                double sn, cs;
                sincos(kds * ((double)(c0 + r0) * h), &sn, &cs);
                const uint32_t rn = min(kRun, cn - r0);
                double run = 0.0;
#pragma unroll 8
                for (uint32_t i = 0; i < rn; ++i) {
                    run = fma(sw[r0 + i], sn, run);
                    const double t = fma(sn, ct, cs * st);
                    cs = fma(cs, ct, -(sn * st));
                    sn = t;
                }
                acc.add(run);
            }
        }
    }
    const double ph = np_d * exp(-m * maxb * maxb * 0.5);
    const double wn = (maxb * exp(bds * ph - reg * reg * maxb * maxb * 0.5)) * weight;
    acc.add(zero_k ? wn * maxb : wn * sin(kds * maxb));
    if (bin < s.bins) {
        const double total = zero_k ? acc.value() : acc.value() / kds;
        out64[bin] = (total / (2.0 * CUDART_PI * CUDART_PI)) * (double)s.bias;
    }
}

__global__ void __launch_bounds__(kFastThreads) lut_build_fast_kernel(LutBuildSpec s, double *out64)
{
    __shared__ double sw[kFastChunk];
    build_fast(s, blockIdx.x * kFastThreads, out64, sw);
}

// Tables of many experiments (FP64 form, no derivatives): blockIdx.y selects the
// experiment, its table at out64 + y*bins.
__global__ void __launch_bounds__(kFastThreads) lut_build_batch_kernel(const LutBuildSpec *__restrict__ specs,
                                                                        uint32_t bins, double *out64)
{
    __shared__ double sw[kFastChunk];
    const LutBuildSpec s = specs[blockIdx.y];
    build_fast(s, blockIdx.x * kFastThreads, out64 + (size_t)blockIdx.y * bins, sw);
}

// Replace non-positive entries by the smallest non-negative one and emit the float copy
// (WeightLookupTableIntegral::Initialize, PathWeightUtils.cpp:305-347). One CTA per table:
// blockIdx.x selects table x of a batch (lut + x*bins, out32 + x*bins, minmax + 3x).
__global__ void __launch_bounds__(1024) lut_finalize_kernel(uint32_t bins, double *lut, float *out32,
                                                            double *minmax)
{
    lut += (size_t)blockIdx.x * bins;
    if (out32) out32 += (size_t)blockIdx.x * bins;
    if (minmax) minmax += 3 * (size_t)blockIdx.x;
    __shared__ double smin[32], smax[32];
    __shared__ int sarg[32];
    // The reference keeps entries in float, so min/max selection runs on the float values.
    double mn = (double)(float)lut[0], mx = mn;
    int arg = 0;
    for (uint32_t i = 1 + threadIdx.x; i < bins; i += blockDim.x) {
        const double v = (double)(float)lut[i];
        if (v < mn && v >= 0.0) { mn = v; arg = (int)i; }
        if (v > mx && v >= 0.0) mx = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double omn = __shfl_xor_sync(0xffffffffu, mn, o);
        const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
        if (omn < mn || (omn == mn && oarg < arg)) { mn = omn; arg = oarg; }
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { smin[w] = mn; smax[w] = mx; sarg[w] = arg; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        mn = l < nw ? smin[l] : DBL_MAX;
        mx = l < nw ? smax[l] : -DBL_MAX;
        arg = l < nw ? sarg[l] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            const double omn = __shfl_xor_sync(0xffffffffu, mn, o);
            const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
            if (omn < mn || (omn == mn && oarg < arg)) { mn = omn; arg = oarg; }
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (l == 0) { smin[0] = mn; smax[0] = mx; sarg[0] = arg; }
    }
    __syncthreads();
    mn = smin[0];
    const double mn64 = lut[sarg[0]];
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) {
        double v = lut[i];
        if ((float)v <= 0.0f) v = mn64;
        lut[i] = v;
        if (out32) out32[i] = (float)v;
    }
    if (threadIdx.x == 0 && minmax) {
        minmax[0] = mn;
        minmax[1] = smax[0];
        minmax[2] = (double)sarg[0];
    }
}

// Compensated-form tables of one experiment per CTA, the device twin of the host's
// compensated_tables (same rules): lin = (L_i, L_{i+1} - L_i); fix = (round((log10 L_i - c0)
// 2^s) as uint32, log10(1 + step (L_{i+1}/L_i - 1))) with c0 = min log10 L - 64 2^-s and the
// largest s <= 30 keeping (N+1) (range 2^s + 65) below 2^31, else the wide form with
// 32 (range 2^s + 65) below 2^32. Bins whose secant error exceeds 1e-7 per segment are
// steep: slope NaN (paths crossing them are re-weighed through lin), counted in lf[x].steep.
// ok[x] = 1 when the fixed form is usable: every entry positive, at most bins/16 steep bins,
// s >= 22.
__global__ void __launch_bounds__(1024) comp_tables_kernel(uint32_t bins, const float *__restrict__ lut32,
                                                           const float *__restrict__ steps,
                                                           const uint32_t *__restrict__ nsegs, float2 *fix,
                                                           float2 *lin, LogFixed *lf, int *ok)
{
    __shared__ double s_lo[32], s_hi[32], s_err[32];
    __shared__ int s_bad[32], s_steep[32];
    const uint32_t x = blockIdx.x;
    const float *L = lut32 + (size_t)x * bins;
    fix += (size_t)x * bins;
    lin += (size_t)x * bins;
    const double st = (double)steps[x];
    double lo = DBL_MAX, hi = -DBL_MAX, err = 0.0;
    int bad = 0, steep = 0;
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) {
        const float a = L[i], b = L[i + 1 < bins ? i + 1 : i];
        lin[i] = make_float2(a, b - a);
        if (!(a > 0.0f) || !isfinite(a)) {
            bad = 1;
            continue;
        }
        const double lg = log10((double)a);
        lo = fmin(lo, lg);
        hi = fmax(hi, lg);
        if (i + 1 < bins) {
            const double r = (double)b / (double)a - 1.0;
            const double e = (st * r) * (st * r) / (8.0 * 2.302585092994046);
            if (e > kSecantBoundDev) ++steep;
            else err = fmax(err, e);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        steep += __shfl_xor_sync(0xffffffffu, steep, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) { s_lo[w] = lo; s_hi[w] = hi; s_err[w] = err; s_bad[w] = bad; s_steep[w] = steep; }
    __syncthreads();
    if (w == 0) {
        lo = l < nw ? s_lo[l] : DBL_MAX;
        hi = l < nw ? s_hi[l] : -DBL_MAX;
        err = l < nw ? s_err[l] : 0.0;
        bad = l < nw ? s_bad[l] : 0;
        steep = l < nw ? s_steep[l] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
            bad |= __shfl_xor_sync(0xffffffffu, bad, o);
            steep += __shfl_xor_sync(0xffffffffu, steep, o);
        }
        if (l == 0) { s_lo[0] = lo; s_hi[0] = hi; s_err[0] = err; s_bad[0] = bad; s_steep[0] = steep; }
    }
    __syncthreads();
    lo = s_lo[0];
    hi = s_hi[0];
    err = s_err[0];
    bad = s_bad[0];
    steep = s_steep[0];
    double cap = floor(2147483647.0 / (double)(nsegs[x] + 1));
    int s = 30;
    while (s > 0 && (hi - lo) * ldexp(1.0, s) + 65.0 > cap) --s;
    int wide = 0;
    if (s < 22) {
        wide = 1;
        cap = floor(4294967295.0 / 32.0);
        s = 30;
        while (s > 0 && (hi - lo) * ldexp(1.0, s) + 65.0 > cap) --s;
    }
    const bool usable = !bad && (uint32_t)steep <= bins / kSteepFractionDev && s >= 22;
    const double inv_scale = ldexp(1.0, -s);
    if (threadIdx.x == 0) {
        lf[x] = usable ? LogFixed{lo - 64.0 * inv_scale, inv_scale, wide, steep} : LogFixed{0.0, 0.0, 0, steep};
        ok[x] = usable ? 1 : 0;
    }
    if (!usable) return;
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) {
        const double e = 64.0 + rint((log10((double)L[i]) - lo) * ldexp(1.0, s));
        const uint32_t u = (uint32_t)fmin(e, cap - 1.0);
        float delta = 0.0f;
        if (i + 1 < bins) {
            const double r = (double)L[i + 1] / (double)L[i] - 1.0;
            delta = ((st * r) * (st * r) / (8.0 * 2.302585092994046) > kSecantBoundDev) ? __int_as_float(0x7fffffff)
                                                                                       : (float)log10(1.0 + st * r);
        }
        fix[i] = make_float2(__uint_as_float(u), delta);
    }
}

}  // namespace

cudaError_t launch_lut_build_batch(const LutBuildSpec *d_specs, uint32_t n, uint32_t bins, double *out64,
                                   cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    if (bins < 2 || n > 65535u) return cudaErrorInvalidValue;
    lut_build_batch_kernel<<<dim3((bins + kFastThreads - 1) / kFastThreads, n), kFastThreads, 0, st>>>(d_specs, bins,
                                                                                                      out64);
    return cudaGetLastError();
}

cudaError_t launch_lut_finalize_batch(uint32_t n, uint32_t bins, double *lut64, float *out32, double *minmax,
                                      cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    lut_finalize_kernel<<<n, 1024, 0, st>>>(bins, lut64, out32, minmax);
    return cudaGetLastError();
}

cudaError_t launch_comp_tables_batch(uint32_t n, uint32_t bins, const float *lut32, const float *steps,
                                     const uint32_t *nsegs, float2 *fix, float2 *lin, LogFixed *lf, int *ok,
                                     cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    comp_tables_kernel<<<n, 1024, 0, st>>>(bins, lut32, steps, nsegs, fix, lin, lf, ok);
    return cudaGetLastError();
}

cudaError_t launch_lut_build(const LutBuildSpec &s, double *out64, double *d_mus, double *d_eps, cudaStream_t st)
{
    if (s.bins < 2 || s.num_steps_int < 4 || (s.num_steps_int & 1u)) return cudaErrorInvalidValue;
    if (!s.faithful && !s.derivatives)
        lut_build_fast_kernel<<<(s.bins + kFastThreads - 1) / kFastThreads, kFastThreads, 0, st>>>(s, out64);
    else
        lut_build_kernel<<<s.bins, kLutThreads, 0, st>>>(s, out64, d_mus, d_eps);
    return cudaGetLastError();
}

cudaError_t launch_lut_finalize(uint32_t bins, double *lut64, float *out32, double *minmax, cudaStream_t st)
{
    lut_finalize_kernel<<<1, 1024, 0, st>>>(bins, lut64, out32, minmax);
    return cudaGetLastError();
}

}  // namespace twisty
