// chain_plain.cu -- the plain FP32 drop-in form, the FP64 yardstick form, the FP64 global
// reduction over chains, and the reference-semantics weigher of given paths.
//
// Plain form: the design of the reference's GPU kernel
// (Twisty/FullExperimentRunnerOptimalPerturbOptimized_GPU.cu:689-918) -- one Markov chain
// per thread with its positions, tangents and curvatures in global memory (one
// contiguous block per chain), every tangent and curvature recomputed each step, FP64
// log10 per segment and a CombinedWeightValues_C accumulator per chain -- with the grid
// sized for 148 SMs instead of the reference's fixed 128x64 threads, Philox in place of
// cuRAND, and the reference CPU runner's proposal ranges
// (Twisty/FullExperimentRunnerOptimalPerturb.cpp:483-519). All FP32 arithmetic is
// spelled with round-to-nearest intrinsics in the reference's operation order, so a chain
// here is bit-identical to the same chain run by the CPU oracle.
#include "kernels.h"

#include <algorithm>
#include "device_common.cuh"

#include <cfloat>

namespace twisty {
namespace {

using dev::CombinedWeight;

constexpr int kPlainThreads = 128;

__global__ void __launch_bounds__(kPlainThreads) plain_chain_kernel(ChainSpec c, const float *__restrict__ init_pos,
                                                                     float *__restrict__ state,
                                                                     const float *__restrict__ lut, LutMetaF mf,
                                                                     ChainOut *__restrict__ out,
                                                                     float *__restrict__ exp_pos,
                                                                     double *__restrict__ exp_w)
{
    const uint32_t chain = blockIdx.x * blockDim.x + threadIdx.x;
    if (chain >= c.n_chains) return;
    const uint32_t N = c.n_segments;
    const size_t stride = plain_state_floats_per_chain(N);
    float *pos = state + (size_t)chain * stride;  // (N+1)*3
    float *tan = pos + 3 * (N + 1);               // N*3
    float *curv = tan + 3 * N;                    // N-1
    for (uint32_t i = 0; i < 3 * (N + 1); ++i) pos[i] = init_pos[i];
    const dev::LutMeta m{mf.min_k, mf.max_k, mf.step, mf.bins};

    CombinedWeight cw;
    dev::cw_reset(cw);
    uint32_t failed = 0, clamped = 0;
    const uint32_t steps = (chain == c.n_chains - 1) ? c.last_steps : c.steps;
    const uint32_t total = c.burn_in + steps;
    for (uint32_t s = 0; s < total; ++s) {
        const dev::Proposal pr = dev::draw_step(c.seed, c.experiment, c.chain0 + chain, s, N, c.k_eff, c.max_angle);
        const uint32_t left = pr.left, right = pr.left + pr.k;
        const float lx = pos[3 * left], ly = pos[3 * left + 1], lz = pos[3 * left + 2];
        const float dx = __fsub_rn(pos[3 * right], lx), dy = __fsub_rn(pos[3 * right + 1], ly),
                    dz = __fsub_rn(pos[3 * right + 2], lz);
        const float inv = dev::rinvnorm(dx, dy, dz);
        const float ax = __fmul_rn(dx, inv), ay = __fmul_rn(dy, inv), az = __fmul_rn(dz, inv);
        float sn, cs;
        dev::sincos_half(pr.angle, sn, cs);
        const float q[4] = {cs, __fmul_rn(ax, sn), __fmul_rn(ay, sn), __fmul_rn(az, sn)};
        for (uint32_t i = left + 1; i < right; ++i) {
            float x = __fsub_rn(pos[3 * i], lx), y = __fsub_rn(pos[3 * i + 1], ly), z = __fsub_rn(pos[3 * i + 2], lz);
            dev::rrotate(q, x, y, z);
            pos[3 * i] = __fadd_rn(x, lx);
            pos[3 * i + 1] = __fadd_rn(y, ly);
            pos[3 * i + 2] = __fadd_rn(z, lz);
        }
        if (s < c.burn_in) continue;
        // UpdateTangentsFromPos (CurvePerturbUtils.cpp:147-154)
        for (uint32_t i = 0; i < N; ++i) {
            float x = __fsub_rn(pos[3 * i + 3], pos[3 * i]), y = __fsub_rn(pos[3 * i + 4], pos[3 * i + 1]),
                  z = __fsub_rn(pos[3 * i + 5], pos[3 * i + 2]);
            if (c.has_eval_shift && i == N - 2) {
                x = __fadd_rn(x, c.eval_shift[0]);
                y = __fadd_rn(y, c.eval_shift[1]);
                z = __fadd_rn(z, c.eval_shift[2]);
            }
            const float r = dev::rinvnorm(x, y, z);
            tan[3 * i] = __fmul_rn(x, r);
            tan[3 * i + 1] = __fmul_rn(y, r);
            tan[3 * i + 2] = __fmul_rn(z, r);
        }
        // UpdateCurvaturesFromTangents_RadiativeTransfer (CurvePerturbUtils.cpp:157-166, bound N-1)
        for (uint32_t i = 0; i + 1 < N; ++i) {
            const float x = __fmul_rn(__fsub_rn(tan[3 * i + 3], tan[3 * i]), c.inv_ds);
            const float y = __fmul_rn(__fsub_rn(tan[3 * i + 4], tan[3 * i + 1]), c.inv_ds);
            const float z = __fmul_rn(__fsub_rn(tan[3 * i + 5], tan[3 * i + 2]), c.inv_ds);
            curv[i] = __fsqrt_rn(dev::rdot3(x, y, z));
        }
        // WeightCurveViaCurvatureLog10_CudaSafe (PathWeighters.cpp:27-104)
        double running = 0.0;
        bool ok = true;
        for (uint32_t i = 0; i + 1 < N; ++i) {
            double blend;
            if (dev::rbin_blend(curv[i], lut, m, blend, clamped) < 0) { ok = false; break; }
            const double lg = log10(blend * c.absorption_factor);
            if (isnan(lg)) { ok = false; break; }
            running += lg;
        }
        if (ok && !isnan(running)) dev::cw_add(cw, running);
        else ++failed;
        if (exp_w) {
            // export replay: every weighted path of this chain, in step order (a weights-only
            // replay passes no position buffer)
            const size_t pidx = (size_t)chain * c.steps + (s - c.burn_in);
            if (exp_pos) {
                float *dst = exp_pos + pidx * 3 * (size_t)(N + 1);
                for (uint32_t i = 0; i < 3 * (N + 1); ++i) dst[i] = pos[i];
            }
            exp_w[pidx] = (ok && !isnan(running)) ? running : NAN;
        }
    }
    ChainOut o;
    o.log10_sum = dev::cw_log10(cw);
    o.valid = cw.n;
    o.failed = failed;
    o.clamped = clamped;
    o.pad = 0;
    out[chain] = o;
}

// ------------------------------------------------------------------------------------
// FP64 form: positions, rotation, tangents, curvatures, table and weights in double. The
// proposal sequence is the same Philox draw; the rotation is the matrix of the unit
// quaternion (cos a/2, axis sin a/2) applied as q^-1 p q, as the reference's quaternion
// sandwich (CurvePerturbUtils.cpp:113-127). Tangents are recomputed on the fly, so only
// the positions live in global memory.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double lse_term(double &mx, double &sum, double &comp, double v, uint32_t n)
{
    if (n == 0) { mx = v; sum = 1.0; comp = 0.0; return 0.0; }
    if (v > mx) {
        const double f = exp10(mx - v);
        sum = sum * f;
        comp = comp * f;
        mx = v;
        v = 1.0;
    } else {
        v = exp10(v - mx);
    }
    const double y = v - comp, t = sum + y;
    comp = (t - sum) - y;
    sum = t;
    return 0.0;
}

__global__ void __launch_bounds__(kPlainThreads) fp64_chain_kernel(ChainSpec c, const float *__restrict__ init_pos,
                                                                    double *__restrict__ state,
                                                                    const double *__restrict__ lut, double min_k,
                                                                    double max_k, double step, int32_t bins,
                                                                    ChainOut *__restrict__ out)
{
    const uint32_t chain = blockIdx.x * blockDim.x + threadIdx.x;
    if (chain >= c.n_chains) return;
    const uint32_t N = c.n_segments;
    double *pos = state + (size_t)chain * 3 * (N + 1);
    for (uint32_t i = 0; i < 3 * (N + 1); ++i) pos[i] = (double)init_pos[i];
    const double arclength = (double)c.arclength;
    const double inv_ds = (double)N / arclength;
    const double absorption_factor = c.absorption_factor;
    double mx = 0.0, sum = 0.0, comp = 0.0;
    uint32_t valid = 0, failed = 0, clamped = 0;
    const uint32_t steps = (chain == c.n_chains - 1) ? c.last_steps : c.steps;
    const uint32_t total = c.burn_in + steps;
    for (uint32_t s = 0; s < total; ++s) {
        const dev::Proposal pr = dev::draw_step(c.seed, c.experiment, c.chain0 + chain, s, N, c.k_eff, c.max_angle);
        const uint32_t left = pr.left, right = pr.left + pr.k;
        const double lx = pos[3 * left], ly = pos[3 * left + 1], lz = pos[3 * left + 2];
        const double dx = pos[3 * right] - lx, dy = pos[3 * right + 1] - ly, dz = pos[3 * right + 2] - lz;
        const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        const double ax = dx * inv, ay = dy * inv, az = dz * inv;
        double sn, cs;
        sincos(0.5 * (double)pr.angle, &sn, &cs);
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
        if (s < c.burn_in) continue;
        double running = 0.0;
        bool ok = true;
        double px = 0, py = 0, pz = 0;  // previous tangent
        for (uint32_t i = 0; i < N; ++i) {
            double x = pos[3 * i + 3] - pos[3 * i], y = pos[3 * i + 4] - pos[3 * i + 1], z = pos[3 * i + 5] - pos[3 * i + 2];
            if (c.has_eval_shift && i == N - 2) {
                x += (double)c.eval_shift[0];
                y += (double)c.eval_shift[1];
                z += (double)c.eval_shift[2];
            }
            const double r = 1.0 / sqrt(x * x + y * y + z * z);
            const double tx = x * r, ty = y * r, tz = z * r;
            if (i > 0) {
                const double cx = (tx - px) * inv_ds, cy = (ty - py) * inv_ds, cz = (tz - pz) * inv_ds;
                double kappa = sqrt(cx * cx + cy * cy + cz * cz);
                if (isnan(kappa)) { ok = false; break; }
                if (kappa < min_k) kappa = min_k;
                if (kappa > max_k) {
                    if (kappa - max_k >= 1e-3) ++clamped;
                    kappa = max_k;
                }
                const double dist = kappa - min_k;
                int32_t l = (int32_t)floor(dist / step);
                if (l > bins - 1) l = bins - 1;
                const int32_t rr = (l == bins - 1) ? l : l + 1;
                const double interp = dist - (double)l * step;
                const double v = (lut[l] * (1.0 - interp) + lut[rr] * interp) * absorption_factor;
                const double lg = log10(v);
                if (isnan(lg)) { ok = false; break; }
                running += lg;
            }
            px = tx; py = ty; pz = tz;
        }
        if (ok) { lse_term(mx, sum, comp, running, valid); ++valid; }
        else ++failed;
    }
    ChainOut o;
    o.log10_sum = valid ? mx + log10(sum + comp) : -INFINITY;
    o.valid = valid;
    o.failed = failed;
    o.clamped = clamped;
    o.pad = 0;
    out[chain] = o;
}

// ------------------------------------------------------------------------------------
// FP64 global reduction over chains: log10 of the summed weight, and the standard error
// of that sum from the spread of the chain sums (chains are independent; their within-
// chain correlation is absorbed by treating each chain sum as one observation).
// ------------------------------------------------------------------------------------
// With ranges set, CTA x reduces the chains ranges[x] = (first, count) into out[x] (one
// experiment of a batch per CTA).
__global__ void __launch_bounds__(1024) reduce_kernel(const ChainOut *__restrict__ chains, uint32_t n,
                                                       ReduceOut *__restrict__ out, const uint2 *__restrict__ ranges)
{
    if (ranges) {
        const uint2 rg = ranges[blockIdx.x];
        chains += rg.x;
        n = rg.y;
        out += blockIdx.x;
    }
    __shared__ double sd[32], sd2[32], sd3[32];
    __shared__ unsigned long long su[3][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    double mx = -INFINITY;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, chains[i].log10_sum);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (l == 0) sd[w] = mx;
    __syncthreads();
    if (w == 0) {
        double v = l < nw ? sd[l] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) sd[0] = v;
    }
    __syncthreads();
    mx = sd[0];
    __syncthreads();
    double s1 = 0.0, c1 = 0.0, s2 = 0.0;
    unsigned long long nv = 0, nf = 0, nc = 0;
    if (mx > -INFINITY) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const ChainOut ch = chains[i];
            const double x = (ch.log10_sum > -INFINITY) ? exp10(ch.log10_sum - mx) : 0.0;
            const double y = x - c1, t = s1 + y;
            c1 = (t - s1) - y;
            s1 = t;
            s2 += x * x;
        }
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        nv += chains[i].valid;
        nf += chains[i].failed;
        nc += chains[i].clamped;
    }
    s1 -= c1;
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        nv += __shfl_xor_sync(0xffffffffu, nv, o);
        nf += __shfl_xor_sync(0xffffffffu, nf, o);
        nc += __shfl_xor_sync(0xffffffffu, nc, o);
    }
    if (l == 0) { sd2[w] = s1; sd3[w] = s2; su[0][w] = nv; su[1][w] = nf; su[2][w] = nc; }
    __syncthreads();
    if (w == 0) {
        s1 = l < nw ? sd2[l] : 0.0;
        s2 = l < nw ? sd3[l] : 0.0;
        nv = l < nw ? su[0][l] : 0;
        nf = l < nw ? su[1][l] : 0;
        nc = l < nw ? su[2][l] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            nv += __shfl_xor_sync(0xffffffffu, nv, o);
            nf += __shfl_xor_sync(0xffffffffu, nf, o);
            nc += __shfl_xor_sync(0xffffffffu, nc, o);
        }
        if (l == 0) {
            ReduceOut r;
            r.max_chain_log10 = mx;
            r.log10_sum = (mx > -INFINITY && s1 > 0.0) ? mx + log10(s1) : -INFINITY;
            double se = NAN;
            if (n > 1 && s1 > 0.0) {
                const double mean = s1 / n;
                const double var = fmax(0.0, (s2 - n * mean * mean) / (n - 1));
                se = sqrt(n * var) / s1;
            }
            r.rel_se = se;
            r.valid = nv;
            r.failed = nf;
            r.clamped = nc;
            *out = r;
        }
    }
}

// ------------------------------------------------------------------------------------
// Weigh given paths with the reference's FP32 semantics: one path per thread.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) weigh_plain_kernel(const float *__restrict__ pos, uint64_t n_paths,
                                                           uint32_t N, float inv_ds, const float *__restrict__ lut,
                                                           LutMetaF mf, double absorption_factor,
                                                           double *__restrict__ log10w, uint8_t *__restrict__ valid,
                                                           int32_t *__restrict__ bins)
{
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_paths) return;
    const float *pp = pos + p * 3 * (uint64_t)(N + 1);
    const dev::LutMeta m{mf.min_k, mf.max_k, mf.step, mf.bins};
    double running = 0.0;
    bool ok = true;
    uint32_t clamped = 0;
    float px = 0.f, py = 0.f, pz = 0.f;
    for (uint32_t i = 0; i < N; ++i) {
        const float x = __fsub_rn(pp[3 * i + 3], pp[3 * i]), y = __fsub_rn(pp[3 * i + 4], pp[3 * i + 1]),
                    z = __fsub_rn(pp[3 * i + 5], pp[3 * i + 2]);
        const float r = dev::rinvnorm(x, y, z);
        const float tx = __fmul_rn(x, r), ty = __fmul_rn(y, r), tz = __fmul_rn(z, r);
        if (i > 0) {
            const float cx = __fmul_rn(__fsub_rn(tx, px), inv_ds), cy = __fmul_rn(__fsub_rn(ty, py), inv_ds),
                        cz = __fmul_rn(__fsub_rn(tz, pz), inv_ds);
            const float kappa = __fsqrt_rn(dev::rdot3(cx, cy, cz));
            double blend = 0.0;
            const int32_t b = ok ? dev::rbin_blend(kappa, lut, m, blend, clamped) : -1;
            if (bins) bins[p * (N - 1) + (i - 1)] = b;
            if (ok) {
                if (b < 0) ok = false;
                else {
                    const double lg = log10(blend * absorption_factor);
                    if (isnan(lg)) ok = false;
                    else running += lg;
                }
            }
        }
        px = tx; py = ty; pz = tz;
    }
    log10w[p] = ok ? running : 0.0;
    if (valid) valid[p] = ok ? 1 : 0;
}

}  // namespace

cudaError_t launch_plain_chains(const ChainSpec &c, const float *init_pos, float *state, const float *lut,
                                LutMetaF m, ChainOut *out, cudaStream_t st, float *exp_pos, double *exp_w)
{
    if (c.n_chains == 0) return cudaSuccess;
    const uint32_t blocks = (c.n_chains + kPlainThreads - 1) / kPlainThreads;
    plain_chain_kernel<<<blocks, kPlainThreads, 0, st>>>(c, init_pos, state, lut, m, out, exp_pos, exp_w);
    return cudaGetLastError();
}

cudaError_t launch_fp64_chains(const ChainSpec &c, const float *init_pos, double *state, const double *lut,
                               double min_k, double max_k, double step, int32_t bins, ChainOut *out, cudaStream_t st)
{
    const uint32_t blocks = (c.n_chains + kPlainThreads - 1) / kPlainThreads;
    fp64_chain_kernel<<<blocks, kPlainThreads, 0, st>>>(c, init_pos, state, lut, min_k, max_k, step, bins, out);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const ChainOut *chains, uint32_t n, ReduceOut *out, cudaStream_t st)
{
    reduce_kernel<<<1, 1024, 0, st>>>(chains, n, out, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_reduce_segments(const ChainOut *chains, const uint2 *ranges, uint32_t n_segments, ReduceOut *out,
                                   cudaStream_t st)
{
    if (n_segments == 0) return cudaSuccess;
    reduce_kernel<<<n_segments, 1024, 0, st>>>(chains, 0, out, ranges);
    return cudaGetLastError();
}

cudaError_t launch_weigh_plain(const float *pos, uint64_t n_paths, uint32_t n_segments, float inv_ds,
                               const float *lut, LutMetaF m, double absorption_factor, double *log10w,
                               uint8_t *valid, int32_t *bins, cudaStream_t st)
{
    if (n_paths == 0) return cudaSuccess;
    const uint64_t blocks = (n_paths + 127) / 128;
    weigh_plain_kernel<<<(unsigned)blocks, 128, 0, st>>>(pos, n_paths, n_segments, inv_ds, lut, m,
                                                         absorption_factor, log10w, valid, bins);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------ path histogram
namespace {
// Linear path weights 10^(w + log10_norm) counted into nbins equal buckets over [lo, hi]: below
// lo into the first, above hi into the last (the reference's rule,
// FullExperimentRunnerOptimalPerturb.cpp:562-575, whose index for a weight of exactly hi is one
// past its last bucket: here the last); NaN (unwritten or invalid) weights are not counted.
__global__ void __launch_bounds__(256) weight_histogram_kernel(const double *__restrict__ w, uint64_t n,
                                                               double log10_norm, double lo, double hi,
                                                               uint32_t nbins, unsigned long long *__restrict__ counts)
{
    extern __shared__ unsigned int h[];
    for (uint32_t i = threadIdx.x; i < nbins; i += blockDim.x) h[i] = 0u;
    __syncthreads();
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const double x = w[p];
        if (isnan(x)) continue;
        const double v = exp10(x + log10_norm);
        uint32_t b;
        if (v < lo) b = 0;
        else if (v > hi) b = nbins - 1;
        else b = min((uint32_t)((v - lo) / (hi - lo) * (double)nbins), nbins - 1);
        atomicAdd(&h[b], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nbins; i += blockDim.x)
        if (h[i]) atomicAdd(&counts[i], (unsigned long long)h[i]);
}
}  // namespace

cudaError_t launch_weight_histogram(const double *w, uint64_t n, double log10_norm, double lo, double hi, uint32_t nbins,
                                    unsigned long long *counts, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 8);
    weight_histogram_kernel<<<(unsigned)blocks, 256, sizeof(unsigned int) * nbins, st>>>(w, n, log10_norm, lo, hi, nbins,
                                                                                         counts);
    return cudaGetLastError();
}

}  // namespace twisty
