"""Host logic of the precision comparison (no GPU).

The precision forms are judged against the FP64 push with the FP64
statistic's own sampling error, measured by batch means.  Here the
ratio-estimator standard error is checked against the spread of many
independent samples, and the per-cell test against hand-built cells: a
resolved cell is held to the tolerance, an unresolved one to K_SIGMA
standard errors of the difference of two runs."""
import math

import numpy as np

from particle_transport_b200 import precision as P


def test_ratio_se_matches_the_spread_of_independent_samples():
    rng = np.random.default_rng(0)
    G, n, trials = 16, 2048, 300
    ratios, ests = [], []
    for _ in range(trials):
        c = rng.poisson(40, size=n)  # pairs per particle (unequal batch counts)
        s = np.array([rng.gamma(2.0, 1.0, size=k).sum() for k in c])  # correlated within a particle
        S, C = s.reshape(G, -1).sum(1), c.reshape(G, -1).sum(1)
        ratios.append(S.sum() / C.sum())
        ests.append(P.ratio_se(S[:, None], C[:, None])[0])
    emp = np.std(ratios) / np.mean(ratios)
    assert abs(np.mean(ests) / emp - 1.0) < 0.15, (np.mean(ests), emp)


def test_ratio_se_empty_cells_are_nan():
    S = np.zeros((4, 3))
    C = np.zeros((4, 3))
    S[:, 0], C[:, 0] = [1.0, 2.0, 1.5, 1.2], [10, 10, 10, 10]
    se = P.ratio_se(S, C)
    assert np.isfinite(se[0]) and np.all(np.isnan(se[1:]))


def test_cell_test_resolved_and_unresolved():
    ref = np.array([[1.0, 1.0, 1.0, 1.0]])
    se = np.array([[1e-4, 1e-4, 0.01, 0.01]])  # two resolved cells, two that are not
    band = P.K_SIGMA * math.sqrt(2.0) * 0.01
    form = np.array([[1.009, 1.011, 1.0 + 0.9 * band, 1.0 + 1.1 * band]])
    e = P.rel_err(form, ref, se)
    assert e["cells"] == 4 and e["resolved_cells"] == 2
    assert [c[1] for c in e["failing"]] == [1, 3]
    assert e["worst_cell"] == [0, 3]
    assert math.isclose(e["max_resolved"], 0.011, rel_tol=1e-9)
    # cells outside the mask or without a standard error are not judged
    e2 = P.rel_err(form, ref, np.array([[1e-4, np.nan, 0.01, 0.01]]), mask=np.array([[True, True, True, False]]))
    assert e2["cells"] == 2 and e2["failing"] == []
    # nor are cells the sample does not measure (standard error above the cap): counted apart
    e3 = P.rel_err(np.array([1.0, 3.0]), np.array([1.0, 1.0]), np.array([1e-4, 2 * P.SE_CAP]))
    assert e3["cells"] == 1 and e3["unmeasured_cells"] == 1 and e3["failing"] == []


def test_check_forms_reports_forms_and_floors():
    good = P.rel_err(np.array([1.001]), np.array([1.0]), np.array([1e-3]))
    bad = P.rel_err(np.array([1.5]), np.array([1.0]), np.array([1e-3]))
    r = {f: {p: good for p in P.PRODUCTS} for f in ("f32", "bf16") + P.FLOORS}
    assert P.check_forms(r) == []
    r["bf16"] = dict(r["bf16"], D_pp=bad)
    r["f64_resample"] = dict(r["f64_resample"], D_mumu=bad)
    fails = P.check_forms(r)
    assert {(f[0], f[1]) for f in fails} == {("bf16", "D_pp"), ("f64_resample", "D_mumu")}
