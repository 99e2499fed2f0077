// peak.cu -- the FP32 issue rate the chain kernels' roofline is quoted against, measured on the
// device at hand: every lane runs independent FMA chains (the FP32 pipe's full rate needs
// several in flight per lane), so the kernel's time is the pipe's, not its latency.
#include "kernels.h"
#include "../../include/twisty_b200.h"

#include <algorithm>
#include <string>

namespace twisty {
void set_free_error(const std::string &msg);
}

namespace {

constexpr int kChains = 8;       // independent accumulators per lane
constexpr int kUnroll = 16;      // FMA rounds per loop trip (keeps the loop's own instructions under 1 %)

__global__ void __launch_bounds__(256) fp32_fma_kernel(float *out, int trips, float a, float b)
{
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (float)(threadIdx.x + c);
    for (int t = 0; t < trips; ++t) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1234.5f) out[0] = s;   // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" twisty_status twisty_measure_fp32_peak(int device, double *lane_instr_per_s)
{
    if (!lane_instr_per_s) return TWISTY_ERR_INVALID_ARGUMENT;
    auto cuda_fail = [](cudaError_t e, const char *what) {
        cudaGetLastError();
        twisty::set_free_error(std::string(what) + ": " + cudaGetErrorString(e));
        return TWISTY_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return cuda_fail(e, "device query");
    float *out = nullptr;
    e = cudaMalloc(&out, sizeof(float));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256, trips = 4096;
    double best = 0.0;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {   // the first is a warm-up
        cudaEventRecord(a);
        fp32_fma_kernel<<<blocks, threads>>>(out, trips, 0.999999f, 1e-7f);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        const double fmas = (double)blocks * threads * trips * kUnroll * kChains;
        if (rep > 0 && ms > 0.f) best = std::max(best, fmas / (ms * 1e-3));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "FMA kernel");
    *lane_instr_per_s = best;
    return TWISTY_OK;
}
