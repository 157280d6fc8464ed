"""Golden fixture tests/golden/small_case.npz (made by tests/golden/make_golden.py
from a pure-Python restatement cross-checked against the C oracle).

CPU: the oracle reproduces the fixture bit for bit.
GPU: the CUDA FP64 push (host-buffer C-ABI entry point) and the D_mumu
kernel reproduce it -- push and counts bit for bit, FP64 sums to 1e-12."""
import os

import numpy as np
import pytest

from helpers import fortran_fields
from particle_transport_b200.fields import UniformGrid

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_case.npz")
KEYS = ("x1", "x2", "x3", "p1", "p2", "p3")


@pytest.fixture(scope="module")
def gold():
    z = np.load(FIX)
    n = [int(v) for v in z["grid_n"]]
    g = UniformGrid(*n, *[float(v) for v in z["grid"]])
    fields = [np.ascontiguousarray(f) for f in z["fields"]]
    state = {k: z[f"state_{k}"] for k in KEYS}
    return z, g, fields, state


def test_fixture_has_deaths_in_open_case(gold):
    z = gold[0]
    assert z["alive_count_open"][-1] < z["alive_count_open"][0]
    assert np.isnan(z["mu_open"]).any()


@pytest.mark.parametrize("periodic", [True, False])
def test_oracle_reproduces_golden_push(oracle, gold, periodic):
    z, g, fields, state = gold
    st = {k: v.copy() for k, v in state.items()}
    tag = "periodic" if periodic else "open"
    mu, ac = oracle.push_run(fortran_fields(fields), g, st, np.ones(len(st["x1"]), np.uint8), float(z["dt"]),
                             int(z["nsteps"]), int(z["stride"]), periodic=periodic, cache_mode=1)
    assert np.array_equal(mu, z[f"mu_{tag}"], equal_nan=True)
    assert np.array_equal(ac, z[f"alive_count_{tag}"])
    for k in KEYS:
        assert np.array_equal(st[k], z[f"final_{k}_{tag}"])


@pytest.mark.parametrize("mode", ["sliding", "injection"])
def test_oracle_reproduces_golden_dmumu(oracle, gold, mode):
    z = gold[0]
    from helpers import zero_dmumu
    acc = zero_dmumu(len(z["lags"]), len(z["edges"]) - 1)
    oracle.dmumu_accumulate(z["mu_cache"], z["lags"], z["edges"], acc, injection=mode == "injection", nthreads=1)
    for k, v in acc.items():
        assert np.array_equal(v, z[f"dmumu_{mode}_{k}"]), k


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [True, False])
def test_cuda_reproduces_golden_push(cuda, gold, periodic):
    from particle_transport_b200 import runner as R
    from particle_transport_b200.fields import FieldLibrary
    z, g, fields, state = gold
    st = {k: v.copy() for k, v in state.items()}
    n = len(st["x1"])
    nsteps, stride = int(z["nsteps"]), int(z["stride"])
    fl = FieldLibrary(fields, g, "ref_f64")
    col = R.CacheCollector(n, R.n_saves(nsteps, stride), "mu")
    ac = R.run_push_host(fl, st, np.ones(n, np.uint8), R.push_params(float(z["dt"]), nsteps, stride,
                                                                     periodic=periodic, cache="mu"), col)
    tag = "periodic" if periodic else "open"
    assert np.array_equal(col.mu, z[f"mu_{tag}"], equal_nan=True)
    assert np.array_equal(ac, z[f"alive_count_{tag}"])
    for k in KEYS:
        assert np.array_equal(st[k], z[f"final_{k}_{tag}"])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["sliding", "injection"])
def test_cuda_reproduces_golden_dmumu(cuda, gold, mode):
    from particle_transport_b200 import stats as S
    z = gold[0]
    nl, nb = len(z["lags"]), len(z["edges"]) - 1
    acc = S.new_dmumu_accumulators(nl, nb)
    S.process_mu_chunk_dmumu(np.ascontiguousarray(z["mu_cache"]), z["lags"], z["edges"], acc["particle_counts"],
                             acc["particle_means"], acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                             acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"], start_mode=mode)
    g = lambda k: z[f"dmumu_{mode}_{k}"]  # noqa: E731
    assert np.array_equal(acc["dmumu_counts"], g("counts"))
    assert np.array_equal(acc["pair_counts"], g("pair_n"))
    assert np.array_equal(acc["particle_counts"], g("w_count"))
    assert np.allclose(acc["dmumu_sum_delta2"], g("sum_d2"), rtol=1e-12, atol=0)
    assert np.allclose(acc["pair_sum_squares"], g("pair_ss"), rtol=1e-12, atol=0)
    assert np.allclose(acc["particle_means"], g("w_mean"), rtol=1e-12, atol=0)
    sc = 1e-12 * (np.sqrt(np.maximum(g("counts"), 1) * g("sum_d2")) + 1e-30)
    assert np.all(np.abs(acc["dmumu_sum_delta"] - g("sum_d")) <= sc)
