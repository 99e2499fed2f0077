// norm.cu -- the path normaliser's nested quadrature for N = 5 and 6 on the device.
//
// NormalizerStuff::Norm (Twisty/PathWeightUtils.cpp:721-752) returns K5(z) or K6(z) for
// N = 5, 6. Both macros expand to the same 10000-point sum over F7 (the macro at :705
// names F##7), F7 is a 1000-point sum over F6, F6 a 1000-point sum over F5 = K4: 1e10 K4
// evaluations. Each thread here owns one (outer, middle) node pair and sums the 1000 inner
// K4 terms in FP64; CTAs write partial sums that a second kernel adds in a fixed order.
// The float arithmetic of the node positions, radii and K4 itself is the reference's;
// the reference accumulates in a 100-digit decimal, here the accumulation is FP64.
#include "kernels.h"
#include "device_common.cuh"

namespace twisty {
namespace {

constexpr int kNormThreads = 256;

__device__ __forceinline__ float radius(float x, float z)
{
    // rMag = sqrt((z*z) + 1.0 - (2.0*z*x)): float z*z, the rest in double, stored as float
    return (float)sqrt((double)__fmul_rn(z, z) + 1.0 - (2.0 * (double)z * (double)x));
}

__device__ __forceinline__ double k4(float z, float ds)
{
    float result = (z < 2.0f) ? 1.0f : 0.0f;
    result = __fdiv_rn(result, z);
    result = (float)((double)result * (2.0 * (double)dev::kPiF));
    const float inv_ds = (float)(1.0 / (double)ds);
    result = __fmul_rn(result, __fmul_rn(__fmul_rn(inv_ds, inv_ds), inv_ds));
    return (double)result;
}

__global__ void __launch_bounds__(kNormThreads) norm_partial_kernel(float z, float ds, double *partials)
{
    __shared__ double red[kNormThreads / 32];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (t < 10000u * 1000u) {
        const uint32_t i = t / 1000u, jm = t % 1000u;
        const float dxk = __fdiv_rn(2.0f, 10000.0f);
        const float dx = __fdiv_rn(2.0f, 1000.0f);
        const float xk = __fadd_rn(-1.0f, __fmul_rn((float)i, dxk));
        const float r7 = radius(xk, z);                       // F7(x_i, z)
        const float xm = __fadd_rn(-1.0f, __fmul_rn((float)jm, dx));
        const float r6 = radius(xm, r7);                      // F6(x_j, r7)
        for (uint32_t l = 0; l < 1000u; ++l) {
            const float xl = __fadd_rn(-1.0f, __fmul_rn((float)l, dx));
            s += k4(radius(xl, r6), ds);                      // F5(x_l, r6) = K4(...)
        }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kNormThreads / 32; ++w) b += red[w];
        partials[blockIdx.x] = b;
    }
}

__global__ void __launch_bounds__(1024) norm_final_kernel(const double *partials, uint32_t n, double *out)
{
    __shared__ double red[32];
    double s = 0.0, c = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double y = partials[i] - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
    s -= c;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += red[w];
        const double two_pi = 2.0 * (double)dev::kPiF;
        const double f = two_pi * (double)__fdiv_rn(2.0f, 1000.0f);
        const double fk = two_pi * (double)__fdiv_rn(2.0f, 10000.0f);
        *out = b * f * f * fk;
    }
}

}  // namespace

uint32_t norm_partial_blocks() { return (10000u * 1000u + kNormThreads - 1) / kNormThreads; }

cudaError_t launch_norm_k56(float z, float ds, double *partials, double *out, cudaStream_t st)
{
    const uint32_t blocks = norm_partial_blocks();
    norm_partial_kernel<<<blocks, kNormThreads, 0, st>>>(z, ds, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    norm_final_kernel<<<1, 1024, 0, st>>>(partials, blocks, out);
    return cudaGetLastError();
}

}  // namespace twisty
