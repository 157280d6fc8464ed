"""pt_dmumu_accumulate_device_noalloc: the D_mumu binning entry point that
allocates no device memory.

It exists for callers that cannot let a library call cudaMalloc: a host
that owns all device memory through its own pool (the Julia host's CUDA.jl
pool, the campaign server's HBM-budget admission) cannot account for an
allocation made behind its back, and cudaFree stalls every stream on the
device.  Its per-CTA partials live in a fixed 16 MiB device array.

The test calls it through the C ABI twice in a row, on inputs of different
shapes, and checks each result against the allocating entry point
pt_dmumu_accumulate_device with the tolerances of the other statistics
tests (counts exact, FP64 sums to 1e-12).  This file is collected last so
that a run stopping at the first failure has already run every other test;
it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import random_mu_cache
from particle_transport_b200 import _lib
from particle_transport_b200.stats import dmumu_noalloc_fits, new_dmumu_accumulators
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps

pytestmark = pytest.mark.gpu

ORDER = ("dmumu_counts", "dmumu_sum_delta", "dmumu_sum_delta2", "particle_counts", "particle_means", "particle_m2s",
         "pair_sum_squares", "pair_counts")


def _call(fn, d_mu, n, nsave, sp, ss, d_lags, d_edges, n_bins, mode, bin_abs, acc, ctx=None):
    ctx = ctx or _lib.torch_context(d_mu)
    _lib.call(fn, ctx.handle, _lib.ptr(d_mu), n, nsave, sp, ss, _lib.ptr(d_lags), int(d_lags.shape[0]),
              _lib.ptr(d_edges), n_bins, mode, int(bin_abs), *[_lib.ptr(acc[k]) for k in ORDER])


def _compare(new, ref):
    for k in ("dmumu_counts", "pair_counts", "particle_counts"):
        assert np.array_equal(new[k], ref[k]), k
    for k in ("dmumu_sum_delta2", "pair_sum_squares", "particle_means"):
        assert np.allclose(new[k], ref[k], rtol=1e-12, atol=0), k
    scale = np.sqrt(np.maximum(ref["dmumu_counts"], 1) * ref["dmumu_sum_delta2"]) + 1e-30
    assert np.all(np.abs(new["dmumu_sum_delta"] - ref["dmumu_sum_delta"]) <= 1e-12 * scale)
    assert np.allclose(new["particle_m2s"], ref["particle_m2s"], rtol=1e-9, atol=0)


@pytest.mark.parametrize("case", [
    # n, nsave, n_lags, n_bins, mode, bin_abs, layout
    ((3000, 401, 24, 20, _lib.PT_START_SLIDING, True, "particle_fastest"),
     (517, 1201, 40, 50, _lib.PT_START_SLIDING, False, "time_fastest")),
    ((800, 300, 64, 16, _lib.PT_START_INJECTION, True, "time_fastest"),
     (2000, 161, 20, 20, _lib.PT_START_SLIDING, True, "particle_fastest")),
])
def test_noalloc_matches_allocating_entry_point_twice(case):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a GPU")
    for i, (n, nsave, n_lags, n_bins, mode, bin_abs, layout) in enumerate(case):
        mu = random_mu_cache(n, nsave, seed=100 * i + n, nan_frac=0.01)
        if layout == "particle_fastest":
            d_mu = torch.as_tensor(np.ascontiguousarray(mu.T), device="cuda")
            sp, ss = 1, n
        else:
            d_mu = torch.as_tensor(mu, device="cuda")
            sp, ss = nsave, 1
        lags = log_spaced_lag_steps(nsave - 1, n_lags)
        edges, _ = build_mu_edges_full(0.0, 1.0, n_bins, bin_abs=bin_abs)
        d_lags = torch.as_tensor(lags, device="cuda")
        d_edges = torch.as_tensor(edges, device="cuda")
        ref = new_dmumu_accumulators(len(lags), n_bins, device="cuda")
        new = new_dmumu_accumulators(len(lags), n_bins, device="cuda")
        _call("pt_dmumu_accumulate_device", d_mu, n, nsave, sp, ss, d_lags, d_edges, n_bins, mode, bin_abs, ref)
        _call("pt_dmumu_accumulate_device_noalloc", d_mu, n, nsave, sp, ss, d_lags, d_edges, n_bins, mode, bin_abs,
              new)
        torch.cuda.synchronize()
        _compare({k: v.cpu().numpy() for k, v in new.items()}, {k: v.cpu().numpy() for k, v in ref.items()})


@pytest.mark.parametrize("n, nsave, n_lags, n_bins", [
    (3000, 401, 256, 50),  # four passes of 64 lags
    (3000, 401, 64, 200),  # per-CTA partials of 32 lags x 200 bins: the 16 MiB array caps the grid at 108 CTAs
])
def test_noalloc_capped_grid_allocates_nothing(n, nsave, n_lags, n_bins):
    """On a fresh context, whose scratch is empty (an allocating path would
    have to cudaMalloc), the device's free memory is the same before and
    after a no-alloc call, and the result matches the allocating entry point
    on the shared context."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a GPU")
    mu = random_mu_cache(n, nsave, seed=n_bins, nan_frac=0.01)
    d_mu = torch.as_tensor(mu, device="cuda")
    lags = np.arange(1, n_lags + 1, dtype=np.int64)
    edges, _ = build_mu_edges_full(0.0, 1.0, n_bins)
    d_lags = torch.as_tensor(lags, device="cuda")
    d_edges = torch.as_tensor(edges, device="cuda")
    ref = new_dmumu_accumulators(n_lags, n_bins, device="cuda")
    warm = new_dmumu_accumulators(n_lags, n_bins, device="cuda")
    new = new_dmumu_accumulators(n_lags, n_bins, device="cuda")
    fresh = _lib.Context(0)
    try:
        fresh.use_stream(torch.cuda.current_stream())
        args = (d_mu, n, nsave, nsave, 1, d_lags, d_edges, n_bins, _lib.PT_START_SLIDING, True)
        # the first call on a device may load the kernels' module and look up the fixed array's address
        _call("pt_dmumu_accumulate_device_noalloc", *args, warm, ctx=fresh)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        _call("pt_dmumu_accumulate_device_noalloc", *args, new, ctx=fresh)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
    finally:
        fresh.close()
    _call("pt_dmumu_accumulate_device", *args, ref)
    torch.cuda.synchronize()
    ref_np = {k: v.cpu().numpy() for k, v in ref.items()}
    _compare({k: v.cpu().numpy() for k, v in new.items()}, ref_np)
    _compare({k: v.cpu().numpy() for k, v in warm.items()}, ref_np)


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a GPU")
    n, nsave = 4, 60000  # series longer than on-chip staging allows
    d_mu = torch.zeros((n, nsave), dtype=torch.float32, device="cuda")
    d_lags = torch.as_tensor(np.array([1, 2], np.int64), device="cuda")
    edges, _ = build_mu_edges_full(0.0, 1.0, 50)
    d_edges = torch.as_tensor(edges, device="cuda")
    acc = new_dmumu_accumulators(2, 50, device="cuda")
    with pytest.raises(_lib.PtError, match="too long"):
        _call("pt_dmumu_accumulate_device_noalloc", d_mu, n, nsave, nsave, 1, d_lags, d_edges, 50,
              _lib.PT_START_SLIDING, True, acc)
    assert C.sizeof(C.c_void_p) == 8


def test_noalloc_limit_matches_the_host_mirror():
    """The campaign server picks the entry point with
    stats.dmumu_noalloc_fits; the device takes the longest series that
    predicate accepts and refuses one save more."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("needs a GPU")
    n, n_lags, n_bins = 4, 64, 50
    top = max(k for k in range(15000, 30000) if dmumu_noalloc_fits(k, n_lags, n_bins))
    lags = np.arange(1, n_lags + 1, dtype=np.int64) * 97
    edges, _ = build_mu_edges_full(0.0, 1.0, n_bins)
    d_lags = torch.as_tensor(lags, device="cuda")
    d_edges = torch.as_tensor(edges, device="cuda")
    for nsave in (top, top + 1):
        mu = random_mu_cache(n, nsave, seed=nsave, nan_frac=0.01)
        d_mu = torch.as_tensor(mu, device="cuda")
        args = (d_mu, n, nsave, nsave, 1, d_lags, d_edges, n_bins, _lib.PT_START_SLIDING, True)
        new = new_dmumu_accumulators(n_lags, n_bins, device="cuda")
        if nsave == top:
            ref = new_dmumu_accumulators(n_lags, n_bins, device="cuda")
            _call("pt_dmumu_accumulate_device_noalloc", *args, new)
            _call("pt_dmumu_accumulate_device", *args, ref)
            torch.cuda.synchronize()
            _compare({k: v.cpu().numpy() for k, v in new.items()}, {k: v.cpu().numpy() for k, v in ref.items()})
        else:
            with pytest.raises(_lib.PtError, match="too long"):
                _call("pt_dmumu_accumulate_device_noalloc", *args, new)
