"""twisty_run_noalloc, the entry point for callers that cannot allocate device memory.

Such callers (an application whose own allocator holds the GPU's memory, or a pipeline
that must not stall on cudaMalloc/cudaFree) own every buffer: here the inputs and the
result live in torch tensors the test allocates, and the entry point itself only uses the
scratch array compiled into the library. Its result must match the context-based
twisty_run on the same table, initial curve and proposals, on two calls in a row (the
second call reuses the shared scratch the first one filled). The cases cover the kernel
shapes 1 x 16, 1 x 24 (N = 16, 24, whose passes here are long against their 2 burn-in steps,
so both entry points take the one-lane shapes, which also turn the shorter side of each move),
4 x 12 (N = 40, which turns the shorter side too), 4 x 16, 4 x 17, 8 x 24, 16 x 24 and 32 x 24 (N = 64, 66, 192, 384, 768) and both table placements:
a 4096-bin table staged in shared memory and a 20000-bin table gathered through L1 where
staging it would cost the shape warps.

This file is collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import twisty_b200 as T
from twisty_b200 import _abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bins", [4096, 20000])
@pytest.mark.parametrize("N", [16, 24, 40, 64, 66, 192, 384, 768])
def test_noalloc_pass_matches_twisty_run_twice(N, bins):
    import torch

    S = 0.16 * N
    chains, steps, burn = 4096, 100 if N <= 192 else 40, 2 if N <= 24 else 50
    p = T.default_params(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=4000,
                         num_curvature_steps=bins, form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64,
                         perturb_seed=77, num_chains=chains, paths_to_generate=chains * steps,
                         paths_to_skip=burn, max_sub_chain=32, max_angle=0.1)
    bc = T.make_bc((0, 0, 0), (1, 0, 0), (0.8 * S, 0, 0), (1, 0, 0), S)
    init = T.bootstrap_curve(p, bc)
    with T.Context(p) as ctx:
        lut, info = ctx.build_lut(np.float32(S) / np.float32(N))
        ctx.set_lut(lut, info)
        ctx.set_initial_curve(init)
        ref = ctx.run(bc)
    assert ref.total_paths == chains * steps

    # caller-owned device inputs and output
    table = np.stack([lut, np.append(lut[1:] - lut[:-1], np.float32(0))], axis=1).astype(np.float32)
    segs = (init[1:] - init[:-1]).astype(np.float32)
    d_table = torch.from_numpy(table).cuda()
    d_segs = torch.from_numpy(segs).cuda()
    d_result = torch.zeros(C.sizeof(_abi.NoAllocResult), dtype=torch.uint8, device="cuda")
    args = _abi.NoAllocArgs(
        table=d_table.data_ptr(), bins=lut.size, min_curvature=info.min_curvature,
        max_curvature=info.max_curvature, curvature_step=info.curvature_step, init_segments=d_segs.data_ptr(),
        num_segments=N, arclength=S, absorption=0.0, seed=77, experiment_id=0, chain_offset=0,
        num_chains=chains, paths=chains * steps, burn_in=burn, max_sub_chain=32, max_angle=0.1,
        result=d_result.data_ptr())
    lib = _abi.load()
    results = []
    for _ in range(2):
        d_result.zero_()
        torch.cuda.synchronize()
        assert lib.twisty_run_noalloc(C.byref(args), None) == _abi.OK, lib.twisty_last_error(None)
        torch.cuda.synchronize()
        r = _abi.NoAllocResult.from_buffer_copy(d_result.cpu().numpy().tobytes())
        results.append(r)
    for r in results:
        assert r.valid_paths == chains * steps and r.failed_paths == 0
        # same proposals and table; the two paths differ only in how a segment's log-weight is
        # interpolated (the exact blend here, the fixed-point secant table in the context run,
        # whose per-segment error is below 1e-7 in log10)
        tol = 1e-5 + 1e-7 * (N - 1)
        assert abs(r.log10_weight - ref.log10_weight) < tol, (r.log10_weight, ref.log10_weight)
        # the standard error comes from the spread of the chains' sums, which the interpolation
        # difference moves by ~1e-7 of a chain's weight per segment: at N = 768 the estimates of
        # a 4e-6 relative error differ by 0.3 %
        assert r.rel_std_error == pytest.approx(ref.rel_std_error, rel=2e-2)
    assert results[0].log10_weight == results[1].log10_weight


def test_noalloc_rejects_more_chains_than_the_scratch_holds():
    args = _abi.NoAllocArgs(table=1, bins=16, min_curvature=0.0, max_curvature=1.0, curvature_step=1.0 / 15,
                            init_segments=1, num_segments=8, arclength=1.0, num_chains=_abi.NOALLOC_MAX_CHAINS + 1,
                            paths=10, max_sub_chain=4, max_angle=0.1, result=1)
    lib = _abi.load()
    assert lib.twisty_run_noalloc(C.byref(args), None) == _abi.ERR_INVALID_ARGUMENT
    assert b"16384" in lib.twisty_last_error(None)


@pytest.mark.parametrize("bins", [0, 1, _abi.NOALLOC_MAX_BINS + 1, 0xFFFFFFFF])
def test_noalloc_rejects_bin_counts_out_of_range(bins):
    """Checked before any size arithmetic: no launch happens for these (the pointers are dummies)."""
    args = _abi.NoAllocArgs(table=1, bins=bins, min_curvature=0.0, max_curvature=1.0, curvature_step=1.0 / 15,
                            init_segments=1, num_segments=8, arclength=1.0, num_chains=16, paths=10, max_sub_chain=4,
                            max_angle=0.1, result=1)
    lib = _abi.load()
    assert lib.twisty_run_noalloc(C.byref(args), None) == _abi.ERR_INVALID_ARGUMENT
    assert b"bins" in lib.twisty_last_error(None)
