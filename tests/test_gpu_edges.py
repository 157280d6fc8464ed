"""Edge cases of the device paths: empty inputs, all-NaN series, lags at
and beyond the series length, series longer than 65,535 saves (32-bit start
lists, staged in global memory), a single save, and every particle dead.

The oracle is the checker throughout; empty inputs must be accepted and leave
the add-into accumulators untouched."""
import numpy as np
import pytest

from helpers import copy_state, fortran_fields, random_mu_cache, small_problem, zero_dmumu, zero_dpp
from particle_transport_b200 import runner as R
from particle_transport_b200 import stats as S
from particle_transport_b200.fields import FieldLibrary
from particle_transport_b200.time_units import build_mu_edges_full

pytestmark = pytest.mark.gpu


def _dmumu(mu, lags, edges, **kw):
    acc = S.new_dmumu_accumulators(len(lags), len(edges) - 1)
    S.process_mu_chunk_dmumu(mu, lags, edges, acc["particle_counts"], acc["particle_means"], acc["particle_m2s"],
                             acc["pair_sum_squares"], acc["pair_counts"], acc["dmumu_counts"],
                             acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"], **kw)
    return acc


def _same(g, o):
    assert np.array_equal(g["dmumu_counts"], o["counts"])
    assert np.array_equal(g["pair_counts"], o["pair_n"])
    assert np.array_equal(g["particle_counts"], o["w_count"])
    assert np.allclose(g["dmumu_sum_delta2"], o["sum_d2"], rtol=1e-12, atol=0)
    assert np.allclose(g["pair_sum_squares"], o["pair_ss"], rtol=1e-12, atol=0)
    assert np.allclose(g["particle_means"], o["w_mean"], rtol=1e-11, atol=0)
    sc = 1e-12 * np.sqrt(np.maximum(o["counts"], 1) * o["sum_d2"]) + 1e-300
    assert np.all(np.abs(g["dmumu_sum_delta"] - o["sum_d"]) <= sc)


def test_empty_inputs_are_no_ops(cuda):
    torch = cuda
    edges, _ = build_mu_edges_full(0.0, 1.0, 8)
    lags = np.array([1, 2, 5])
    acc = _dmumu(np.zeros((0, 40), np.float32), lags, edges)
    assert all(np.all(v == 0) for v in acc.values())
    acc = _dmumu(random_mu_cache(5, 40), np.zeros(0, np.int64), edges)
    assert all(v.size == 0 for k, v in acc.items() if k in ("particle_counts", "pair_counts"))
    d = S.new_dpp_accumulators(3, device="cuda")
    S.process_momenta_chunk_dpp(torch.zeros((40, 3, 0), dtype=torch.float32, device="cuda"), lags, 1.0,
                                d["counts"], d["sum_delta_p"], d["sum_delta_p2"], d["sum_delta_p_norm"],
                                d["sum_delta_p_norm2"])
    assert int(d["counts"].sum().item()) == 0
    pb = small_problem(n=8, n_particles=4)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    empty = {k: np.zeros(0) for k in R.KEYS}
    ac = R.run_push_host(fl, empty, np.zeros(0, np.uint8), R.push_params(pb.dt, 10, 2, cache="none"))
    assert ac.shape == (10,) and np.all(ac == 0)
    from particle_transport_b200.particles import init_particles_device
    st = init_particles_device(fl, 0, 1.0)
    assert all(v.numel() == 0 for v in st.values())


def test_dmumu_all_nan_and_lags_beyond_series(cuda, oracle):
    mu = random_mu_cache(64, 50, seed=1)
    mu[::3] = np.nan  # every third particle dead from the start
    # 50 and beyond: no pair (lag >= nsave is skipped), past 2^32 too
    lags = np.array([1, 49, 50, 51, 1000, 2 ** 32 + 3], dtype=np.int64)
    edges, _ = build_mu_edges_full(0.0, 1.0, 10)
    o = zero_dmumu(len(lags), 10)
    oracle.dmumu_accumulate(mu, lags, edges, o)
    g = _dmumu(mu, lags, edges)
    _same(g, o)
    assert np.all(g["pair_counts"][2:] == 0) and g["pair_counts"][0] > 0
    nan = np.full((7, 30), np.nan, np.float32)
    g = _dmumu(nan, lags, edges)
    assert all(np.all(v == 0) for v in g.values())


@pytest.mark.parametrize("mode", ["sliding", "injection"])
def test_dmumu_series_longer_than_65535_saves(cuda, oracle, mode):
    """32-bit start lists; the series no longer fits on chip (global staging)."""
    mu = random_mu_cache(3, 70001, seed=11, nan_frac=0.001)
    lags = np.array([1, 7, 1000, 65536, 70000])
    edges, _ = build_mu_edges_full(0.0, 1.0, 16)
    o = zero_dmumu(len(lags), 16)
    oracle.dmumu_accumulate(mu, lags, edges, o, injection=mode == "injection")
    _same(_dmumu(mu, lags, edges, start_mode=mode), o)


def test_dmumu_single_save(cuda, oracle):
    mu = random_mu_cache(20, 1, seed=2)
    edges, _ = build_mu_edges_full(0.0, 1.0, 4)
    g = _dmumu(mu, np.array([1]), edges)
    assert all(np.all(v == 0) for v in g.values())


def test_dpp_nan_and_long_lags(cuda, oracle):
    rng = np.random.default_rng(5)
    mom = (5e-19 * (1 + 1e-3 * rng.normal(size=(300, 3, 40)))).astype(np.float32)
    mom[:, :, 7] = np.nan
    mom[100:, :, 3] = np.nan
    # lags at and past the series end are skipped (one beyond 2^32 too: the
    # range test must come before any narrowing of the lag)
    lags = np.array([1, 2, 299, 300, 400, 2 ** 32 + 5], dtype=np.int64)
    o = zero_dpp(len(lags))
    oracle.dpp_accumulate(mom, lags, 5e-19, o)
    g = S.new_dpp_accumulators(len(lags))
    S.process_momenta_chunk_dpp(np.ascontiguousarray(mom), lags, 5e-19, g["counts"], g["sum_delta_p"],
                                g["sum_delta_p2"], g["sum_delta_p_norm"], g["sum_delta_p_norm2"])
    assert np.array_equal(g["counts"], o["counts"])
    assert np.all(g["counts"][3:] == 0)
    assert np.allclose(g["sum_delta_p2"], o["sum_dp2"], rtol=1e-12, atol=0)
    assert np.allclose(g["sum_delta_p_norm2"], o["sum_dpn2"], rtol=1e-12, atol=0)


def test_all_dead_particles_push(cuda, oracle):
    """Every particle dead on entry: NaN rows, no state change, alive count 0."""
    pb = small_problem(n=10, n_particles=50)
    alive = np.zeros(50, np.uint8)
    st_o = copy_state(pb.state)
    al_o = alive.copy()
    mu_o, ac_o = oracle.push_run(fortran_fields(pb.fields), pb.grid, st_o, al_o, pb.dt, 40, 4, cache_mode=1)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    st_g = copy_state(pb.state)
    al_g = alive.copy()
    col = R.CacheCollector(50, R.n_saves(40, 4), "mu")
    ac_g = R.run_push_host(fl, st_g, al_g, R.push_params(pb.dt, 40, 4, cache="mu"), col)
    assert np.array_equal(col.mu, mu_o, equal_nan=True) and np.all(np.isnan(col.mu))
    assert np.array_equal(ac_g, ac_o) and np.all(ac_g == 0)
    for k in R.KEYS:
        assert np.array_equal(st_g[k], st_o[k]), k
    flb = FieldLibrary(pb.fields, pb.grid, "brick_bf16")
    col2 = R.CacheCollector(50, R.n_saves(40, 4), "mu")
    ac2 = R.run_push_host(flb, copy_state(pb.state), alive.copy(),
                          R.push_params(pb.dt, 40, 4, cache="mu", precision="f32", sort_every=8), col2)
    assert np.all(np.isnan(col2.mu)) and np.all(ac2 == 0)


def test_bf16_field_with_a_nan_node(cuda):
    """A non-finite node stays local in the BF16 bricks: their mean field is
    taken over the finite nodes only, so only the particles whose cells
    touch that node see NaN (all of them would, through the mean)."""
    pb = small_problem(n=16, n_particles=500)
    fields = [np.array(a, copy=True) for a in pb.fields]
    fields[2].reshape(-1)[1234] = np.nan
    flb = FieldLibrary(fields, pb.grid, "brick_bf16", B_ref_T=pb.B0)  # mean |B| of the field is NaN now
    col = R.CacheCollector(500, R.n_saves(40, 4), "mu")
    R.run_push_host(flb, copy_state(pb.state), np.ones(500, np.uint8),
                    R.push_params(pb.dt, 40, 4, cache="mu", precision="f32"), col)
    finite = np.isfinite(col.mu).all(axis=0)
    assert 0.9 < finite.mean() <= 1.0, finite.mean()
