"""Parity of the CUDA lag statistics with the CPU oracle (needs a B200).

Bin counts and pair counts are compared bit for bit; FP64 sums and Welford
moments to 1e-12 relative (they differ only by summation order).  For the
signed sum of dmu the tolerance is relative to sqrt(count * sum dmu^2),
which bounds the sum of |dmu| the rounding acts on."""
import math

import numpy as np
import pytest

from helpers import random_mu_cache, zero_dmumu, zero_dpp
from particle_transport_b200 import stats as S
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def close(a, b, rtol=RTOL, scale=None):
    a, b = np.asarray(a, float), np.asarray(b, float)
    tol = rtol * (np.abs(b) if scale is None else np.maximum(np.abs(b), scale)) + 1e-300
    return np.all(np.abs(a - b) <= tol)


def gpu_dmumu(mu, lags, edges, start_mode="sliding", bin_abs=True, layout="time_fastest", acc=None):
    nl, nb = len(lags), len(edges) - 1
    acc = acc or S.new_dmumu_accumulators(nl, nb)
    S.process_mu_chunk_dmumu(mu, lags, edges, acc["particle_counts"], acc["particle_means"], acc["particle_m2s"],
                             acc["pair_sum_squares"], acc["pair_counts"], acc["dmumu_counts"], acc["dmumu_sum_delta"],
                             acc["dmumu_sum_delta2"], start_mode=start_mode, bin_abs=bin_abs, layout=layout)
    return acc


def check_dmumu(g, o):
    assert np.array_equal(g["dmumu_counts"], o["counts"])
    assert np.array_equal(g["pair_counts"], o["pair_n"])
    assert np.array_equal(g["particle_counts"], o["w_count"])
    assert close(g["dmumu_sum_delta2"], o["sum_d2"])
    scale = np.sqrt(np.maximum(o["counts"], 1) * o["sum_d2"]) + 1e-30
    assert close(g["dmumu_sum_delta"], o["sum_d"], scale=scale)
    assert close(g["pair_sum_squares"], o["pair_ss"])
    assert close(g["particle_means"], o["w_mean"], rtol=1e-11)
    assert close(g["particle_m2s"], o["w_m2"], rtol=1e-9, scale=1e-300 + np.abs(o["w_m2"]).max() * 1e-3)


CASES = [
    # n, nsave, n_lags, n_bins, bin_abs, nan_frac, mode
    (4096, 801, 20, 20, True, 0.0, "sliding"),
    (333, 257, 40, 24, True, 0.05, "sliding"),
    (100, 120, 7, 10, False, 0.1, "sliding"),
    (1000, 401, 64, 50, True, 0.0, "injection"),
    (50, 64, 33, 5, False, 0.0, "injection"),
    (64, 300, 300, 8, True, 0.0, "sliding"),   # > 256 lags: several lag batches
    (3, 40001, 12, 16, True, 0.01, "sliding"),  # long series: staged in global memory
]


@pytest.mark.parametrize("n,nsave,n_lags,n_bins,bin_abs,nan_frac,mode", CASES)
def test_dmumu_matches_oracle(cuda, oracle, n, nsave, n_lags, n_bins, bin_abs, nan_frac, mode):
    mu = random_mu_cache(n, nsave, seed=n + nsave, nan_frac=nan_frac)
    lags = log_spaced_lag_steps(nsave - 1, n_lags) if n_lags < nsave else np.arange(1, n_lags + 1)
    edges, _ = build_mu_edges_full(0.0, 1.0, n_bins, bin_abs=bin_abs)
    o = zero_dmumu(len(lags), n_bins)
    oracle.dmumu_accumulate(mu, lags, edges, o, injection=mode == "injection", bin_abs=bin_abs)
    g = gpu_dmumu(mu, lags, edges, start_mode=mode, bin_abs=bin_abs)
    check_dmumu(g, o)


@pytest.mark.parametrize("bin_abs", [True, False])
def test_dmumu_non_uniform_edges(cuda, oracle, bin_abs):
    """Edges that are not a uniform range (the bin lookup starts from a
    uniform guess and walks to the stored edges), with values on the edges."""
    lo = 0.0 if bin_abs else -1.0
    edges = lo + (1.0 - lo) * np.linspace(0.0, 1.0, 18) ** 2
    rng = np.random.default_rng(11)
    mu = random_mu_cache(700, 301, seed=5, nan_frac=0.02)
    on_edge = rng.random(mu.shape) < 0.05
    mu[on_edge] = rng.choice(edges.astype(np.float32), size=int(on_edge.sum()))
    lags = log_spaced_lag_steps(300, 16)
    o = zero_dmumu(len(lags), 17)
    oracle.dmumu_accumulate(mu, lags, edges, o, bin_abs=bin_abs)
    check_dmumu(gpu_dmumu(mu, lags, edges, bin_abs=bin_abs), o)


def test_dmumu_chunks_add_into(cuda, oracle):
    """Two chunks accumulated into the same arrays == one oracle pass."""
    mu = random_mu_cache(900, 200, seed=4, nan_frac=0.02)
    lags = log_spaced_lag_steps(199, 16)
    edges, _ = build_mu_edges_full(0.0, 1.0, 12)
    o = zero_dmumu(len(lags), 12)
    oracle.dmumu_accumulate(mu, lags, edges, o)
    acc = gpu_dmumu(np.ascontiguousarray(mu[:317]), lags, edges)
    acc = gpu_dmumu(np.ascontiguousarray(mu[317:]), lags, edges, acc=acc)
    check_dmumu(acc, o)


def test_dmumu_device_particle_fastest(cuda, oracle):
    torch = cuda
    mu = random_mu_cache(2000, 161, seed=8, nan_frac=0.01)
    lags = log_spaced_lag_steps(160, 20)
    edges, _ = build_mu_edges_full(0.0, 1.0, 20)
    o = zero_dmumu(len(lags), 20)
    oracle.dmumu_accumulate(mu, lags, edges, o)
    d_mu = torch.as_tensor(np.ascontiguousarray(mu.T), device="cuda")  # [nsave][n]: the cache as written
    acc = S.new_dmumu_accumulators(len(lags), 20, device="cuda")
    gpu_dmumu(d_mu, lags, edges, layout="particle_fastest", acc=acc)
    torch.cuda.synchronize()
    check_dmumu({k: v.cpu().numpy() for k, v in acc.items()}, o)


def test_dmumu_edge_values(cuda, oracle):
    """Values on edges, |mu| = 1, signed out-of-range, NaN and Inf."""
    vals = np.array([0.0, 0.05, 0.1, 1.0, -1.0, 0.5, np.nan, np.inf, -np.inf, 0.95, 0.999999, 1e-30], np.float32)
    rng = np.random.default_rng(3)
    mu = np.ascontiguousarray(rng.choice(vals, size=(97, 130)).astype(np.float32))
    lags = np.array([1, 2, 3, 64, 129, 130, 500])
    for bin_abs in (True, False):
        edges, _ = build_mu_edges_full(0.0, 1.0, 20, bin_abs=bin_abs)
        o = zero_dmumu(len(lags), 20)
        oracle.dmumu_accumulate(mu, lags, edges, o, bin_abs=bin_abs)
        check_dmumu(gpu_dmumu(mu, lags, edges, bin_abs=bin_abs), o)


def test_dmumu_rejects_bad_lags(cuda):
    from particle_transport_b200._lib import PtError
    mu = random_mu_cache(4, 10)
    edges, _ = build_mu_edges_full(0.0, 1.0, 4)
    with pytest.raises(PtError, match="lag"):
        gpu_dmumu(mu, np.array([0, 1]), edges)


@pytest.mark.parametrize("chunk,nsave,n_lags", [(500, 201, 24), (37, 1000, 40), (2, 30001, 5), (64, 1500, 300),
                                                 (16, 6000, 500)])
def test_dpp_matches_oracle(cuda, oracle, chunk, nsave, n_lags):
    rng = np.random.default_rng(chunk)
    p = 5.4e-19 * (1 + 1e-3 * np.cumsum(rng.normal(size=(nsave, 1, chunk)), axis=0))
    u = rng.normal(size=(nsave, 3, chunk))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    mom = np.ascontiguousarray((p * u).astype(np.float32))
    mom[rng.random(mom.shape) < 0.001] = np.nan
    lags = log_spaced_lag_steps(nsave - 1, n_lags)
    p0 = 5.4e-19
    o = zero_dpp(len(lags))
    oracle.dpp_accumulate(mom, lags, p0, o)
    g = S.new_dpp_accumulators(len(lags))
    S.process_momenta_chunk_dpp(mom, lags, p0, g["counts"], g["sum_delta_p"], g["sum_delta_p2"],
                                g["sum_delta_p_norm"], g["sum_delta_p_norm2"])
    assert np.array_equal(g["counts"], o["counts"])
    assert close(g["sum_delta_p2"], o["sum_dp2"])
    assert close(g["sum_delta_p_norm2"], o["sum_dpn2"])
    sc = np.sqrt(np.maximum(o["counts"], 1) * o["sum_dp2"])
    assert close(g["sum_delta_p"], o["sum_dp"], scale=sc)
    sc = np.sqrt(np.maximum(o["counts"], 1) * o["sum_dpn2"])
    assert close(g["sum_delta_p_norm"], o["sum_dpn"], scale=sc)


def test_energy_snapshots_bit_exact(cuda, oracle):
    rng = np.random.default_rng(0)
    mom = np.ascontiguousarray(rng.normal(scale=5e-19, size=(50, 3, 300)).astype(np.float32))
    mom[3, :, 7] = np.nan
    snaps = np.array([0, 3, 25, 49])
    o = np.full((600, 4), np.nan)
    oracle.energy_snapshots(mom, snaps, o, particle_offset=300)
    g = np.full((600, 4), np.nan)
    S.fill_energy_snapshots(g, mom, snaps, particle_offset=300)
    assert np.array_equal(g, o, equal_nan=True)


def test_energy_snapshots_device_bit_exact(cuda, oracle):
    torch = cuda
    rng = np.random.default_rng(0)
    mom = np.ascontiguousarray(rng.normal(scale=5e-19, size=(50, 3, 300)).astype(np.float32))
    mom[3, :, 7] = np.nan
    snaps = np.array([0, 3, 25, 49])
    o = np.full((600, 4), np.nan)
    oracle.energy_snapshots(mom, snaps, o, particle_offset=300)
    g = torch.full((600, 4), float("nan"), dtype=torch.float64, device="cuda")
    S.fill_energy_snapshots(g, torch.as_tensor(mom, device="cuda"), snaps, particle_offset=300)
    assert np.array_equal(g.cpu().numpy(), o, equal_nan=True)
    # an index outside the chunk's saves yields NaN, not a stray read
    g2 = torch.zeros((300, 2), dtype=torch.float64, device="cuda")
    S.fill_energy_snapshots(g2, torch.as_tensor(mom, device="cuda"), [1, 50])
    h = g2.cpu().numpy()
    o1 = np.full((300, 1), np.nan)
    oracle.energy_snapshots(mom, np.array([1]), o1)
    assert np.all(np.isnan(h[:, 1])) and np.array_equal(h[:, 0], o1[:, 0], equal_nan=True)


def test_energy_histogram(cuda, oracle):
    torch = cuda
    rng = np.random.default_rng(1)
    mom = np.ascontiguousarray(rng.normal(scale=5e-18, size=(20, 3, 5000)).astype(np.float32))
    snaps = np.array([0, 10, 19])
    e = np.full((5000, 3), np.nan)
    oracle.energy_snapshots(mom, snaps, e)
    counts = S.energy_histogram(torch.as_tensor(mom, device="cuda"), snaps, 0.01, 100.0, 256).cpu().numpy()
    for j in range(3):
        ref, _ = np.histogram(e[:, j], bins=np.exp(np.linspace(math.log(0.01), math.log(100.0), 257)))
        assert counts[j].sum() == ref.sum()
        assert np.abs(counts[j] - ref).sum() <= 4  # log rounding at bin edges


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reconstruct_mu_bit_exact(cuda, oracle, dtype):
    from helpers import copy_state, fortran_fields, small_problem
    pb = small_problem(n=12, n_particles=211)
    st = copy_state(pb.state)
    (pos, mom), _ = oracle.push_run(fortran_fields(pb.fields), pb.grid, st, np.ones(211, np.uint8), pb.dt, 120, 3,
                                    cache_mode=2, out_f64=dtype == np.float64)
    pos[5, 0, 3] = np.nan
    pos[6, 1, 4] = pb.grid.ymax * 1.01  # outside the box -> NaN
    ff = fortran_fields(pb.fields)[:3]
    if dtype == np.float64:
        o = oracle.reconstruct_mu_f64(pos, mom, ff, pb.grid)
    else:
        o = oracle.reconstruct_mu_f32(pos, mom, ff, pb.grid)
    g = S.reconstruct_mu_chunk(pos, mom, *pb.fields[:3], pb.grid, dtype=dtype)
    assert np.array_equal(g, o, equal_nan=True)
    assert np.isnan(g[3, 5]) and np.isnan(g[4, 6])


@pytest.mark.parametrize("b_layout", ["cells", "nodes"])
@pytest.mark.parametrize("dtype,mode,layout", [(np.float32, "sliding", "julia"), (np.float32, "injection", "cache"),
                                               (np.float64, "sliding", "cache")])
def test_phase_space_dmumu_fused_matches_oracle(cuda, oracle, dtype, mode, layout, b_layout, monkeypatch):
    """Fused phase-space D_mumu = oracle reconstruct_mu at the compute
    precision, then the oracle binning of that mu chunk -- with B read from
    8-corner cell records and from node records."""
    torch = cuda
    monkeypatch.setenv("PTB200_PHASE_SPACE_B", b_layout)
    from helpers import copy_state, fortran_fields, small_problem
    pb = small_problem(n=12, n_particles=517)
    st = copy_state(pb.state)
    f64 = dtype == np.float64
    (pos, mom), _ = oracle.push_run(fortran_fields(pb.fields), pb.grid, st, np.ones(517, np.uint8), pb.dt, 600, 3,
                                    cache_mode=2, out_f64=f64)
    pos[5, 0, 3] = np.nan
    pos[6, 1, 4] = pb.grid.ymax * 1.01  # outside the box -> NaN mu
    ff = fortran_fields(pb.fields)[:3]
    mu = (oracle.reconstruct_mu_f64 if f64 else oracle.reconstruct_mu_f32)(pos, mom, ff, pb.grid)  # (chunk, nsave)
    nsave = pos.shape[0]
    lags = log_spaced_lag_steps(nsave - 1, 24)
    edges, _ = build_mu_edges_full(0.0, 1.0, 16)
    o = zero_dmumu(len(lags), 16)
    # the reference bins Float64(mu) of the chunk at the compute precision; a Float32 chunk is exactly the oracle's input
    oracle.dmumu_accumulate(np.ascontiguousarray(mu, dtype=np.float32) if not f64 else mu, lags, edges, o,
                            injection=mode == "injection")
    tdt = torch.float64 if f64 else torch.float32
    if layout == "julia":
        P = torch.as_tensor(pos, dtype=tdt, device="cuda")
        M = torch.as_tensor(mom, dtype=tdt, device="cuda")
    else:  # the device phase-space cache (nsave, 6, n)
        cache = torch.cat([torch.as_tensor(pos, dtype=tdt), torch.as_tensor(mom, dtype=tdt)], dim=1).cuda()
        P, M = cache[:, 0:3], cache[:, 3:6]
    B = [torch.as_tensor(f, dtype=tdt, device="cuda") for f in pb.fields[:3]]
    g = S.new_dmumu_accumulators(len(lags), 16, device="cuda")
    S.process_phase_space_chunk_dmumu(P, M, *B, pb.grid, lags, edges, g["particle_counts"], g["particle_means"],
                                      g["particle_m2s"], g["pair_sum_squares"], g["pair_counts"], g["dmumu_counts"],
                                      g["dmumu_sum_delta"], g["dmumu_sum_delta2"], start_mode=mode)
    g = {k: v.cpu().numpy() for k, v in g.items()}
    check_dmumu(g, o)
    assert g["pair_counts"].sum() > 0
