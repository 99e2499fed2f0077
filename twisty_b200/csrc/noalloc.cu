// noalloc.cu -- twisty_run_noalloc: a compensated-form pass that allocates no memory.
//
// Some callers cannot call cudaMalloc when they run a pass: an application whose own
// caching allocator has reserved nearly all of the device (an allocation made behind its
// back can fail, or leave its accounting wrong), or a pipeline that must not stall, since
// cudaMalloc and cudaFree may synchronize the whole device. The context-based entry points
// allocate their per-chain result buffer when they prepare a run; this entry point instead
// keeps that scratch in a fixed array compiled into the library and takes every input and
// output from device memory the caller owns. It launches the same compensated chain
// kernel and FP64 reduction as the context path.
#include "kernels.h"
#include "../../include/twisty_b200.h"

#include <atomic>
#include <cmath>
#include <string>

namespace twisty {
void set_free_error(const std::string &msg);
}

namespace {

using twisty::ChainOut;

static_assert(sizeof(ChainOut) == 24, "scratch entry size");
static_assert(sizeof(twisty::ReduceOut) == sizeof(twisty_noalloc_result), "result layout");

// Per-chain results of the pass: TWISTY_NOALLOC_MAX_CHAINS x 24 bytes = 384 KiB on every
// device that loads the library. Host code must not pass this symbol to a kernel: on the
// host it only names a stand-in, and the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) ChainOut g_noalloc_chains[TWISTY_NOALLOC_MAX_CHAINS];

constexpr int kMaxDevices = 64;
std::atomic<void *> g_scratch_addr[kMaxDevices];

twisty_status bad(const char *msg)
{
    twisty::set_free_error(msg);
    return TWISTY_ERR_INVALID_ARGUMENT;
}

twisty_status cuda_fail(cudaError_t e, const char *what)
{
    cudaGetLastError();
    twisty::set_free_error(std::string(what) + ": " + cudaGetErrorString(e));
    return TWISTY_ERR_CUDA;
}

}  // namespace

extern "C" twisty_status twisty_run_noalloc(const twisty_noalloc_args *a, void *stream)
{
    using namespace twisty;
    if (!a) return bad("args is NULL");
    if (!a->table || !a->init_segments || !a->result) return bad("table, init_segments and result must be device pointers");
    if (a->num_segments < 4 || a->num_segments > 1024) return bad("num_segments must be in [4, 1024]");
    // the cap comes first: the size arithmetic below (shared-memory bytes, the signed bin count
    // the kernel clamps to) must not wrap
    if (a->bins < 2 || a->bins > TWISTY_NOALLOC_MAX_BINS) return bad("bins must be in [2, TWISTY_NOALLOC_MAX_BINS = 2^24]");
    if (!(a->curvature_step > 0.0f) || !(a->max_curvature > a->min_curvature))
        return bad("table metadata is invalid");
    if (a->num_chains == 0 || a->num_chains > TWISTY_NOALLOC_MAX_CHAINS)
        return bad("num_chains must be in [1, TWISTY_NOALLOC_MAX_CHAINS = 16384]: the fixed scratch holds 16384 chains");
    if (a->paths == 0) return bad("paths must be at least 1");
    if (a->max_sub_chain < 2 || a->max_sub_chain > 64) return bad("max_sub_chain must be in [2, 64]");
    if (!(a->max_angle >= 0.0f) || a->max_angle > 3.1415927f) return bad("max_angle must be in [0, pi]");
    if (!(a->arclength > 0.0f)) return bad("arclength must be positive");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return bad("device ordinal beyond the supported range");
    // Set-up, once per device, with that device current. The address stays valid for the life of
    // the device's primary context; after cudaDeviceReset it is stale (documented in the header).
    void *scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        e = cudaGetSymbolAddress(&scratch, g_noalloc_chains);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the scratch array");
        g_scratch_addr[dev].store(scratch, std::memory_order_release);
    }

    const uint32_t N = a->num_segments;
    ChainSpec c{};
    c.n_segments = N;
    c.arclength = a->arclength;
    c.ds = a->arclength / (float)N;
    c.inv_ds = (float)N / a->arclength;
    c.seed = a->seed;
    c.experiment = a->experiment_id;
    c.chain0 = a->chain_offset;
    const uint64_t L = (a->paths + a->num_chains - 1) / a->num_chains;
    if (L > 0xFFFFFFFFull - a->burn_in) return bad("too many paths per chain");
    const uint64_t C = (a->paths + L - 1) / L;
    c.n_chains = (uint32_t)C;
    c.steps = (uint32_t)L;
    c.last_steps = (uint32_t)(a->paths - (C - 1) * L);
    c.burn_in = a->burn_in;
    c.k_eff = a->max_sub_chain < N - 2 ? a->max_sub_chain : N - 2;
    c.max_angle = a->max_angle;
    c.absorption_factor = (double)std::exp(-a->absorption * c.ds);
    c.has_eval_shift = 0;

    // the default shape and table placement of twisty_run's forward pass (shared memory when the
    // table fits beside the shape's chain state, else gathered through L1)
    CompTuning t = comp_default_tuning(N, false, a->paths, a->burn_in);
    t.exact_blend = 1;  // the table is the linear (L_i, L_{i+1} - L_i) form
    if (!comp_tuning_supported(t, N, c.k_eff)) return bad("no compensated kernel shape for this N");
    t.lut_global = comp_table_through_l1(t, a->bins, true) ? 1 : 0;
    if (!comp_fit_smem(t, a->bins, true)) return bad("the chain state of this N does not fit in shared memory");
    const LutMetaF m{a->min_curvature, a->max_curvature, a->curvature_step, (int32_t)a->bins};
    cudaStream_t st = (cudaStream_t)stream;
    e = launch_comp_chains(c, t, a->init_segments, static_cast<const float2 *>(a->table),
                           static_cast<const float2 *>(a->table), m, static_cast<ChainOut *>(scratch), nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "chain kernel");
    e = launch_reduce(static_cast<const ChainOut *>(scratch), c.n_chains, static_cast<ReduceOut *>(a->result), st);
    if (e != cudaSuccess) return cuda_fail(e, "reduction");
    return TWISTY_OK;
}
