"""Host logic of the batch tuner and of the server's admission (no GPU).

tune_batch times real batches on a B200; here its timing trial is replaced
by a synthetic rate model, so the selection logic itself is checked: speed
classes, the cadence per class, K = the shortest cadence, each campaign's
sort_every, the blocks-per-SM choice and the JSON cache.  The server admits
waiting jobs in arrival order while the HBM budget has room, and holds every
later job behind one that does not fit."""
import math
from types import SimpleNamespace

import numpy as np

from particle_transport_b200 import batch as B
from particle_transport_b200.fields import C_LIGHT, M_P
from particle_transport_b200.particles import energy_to_gamma
from particle_transport_b200.server import CampaignServer, JobSpec


def campaign(E_GeV, n, dx=1.0):
    g = energy_to_gamma(E_GeV)
    p = g * M_P * C_LIGHT * math.sqrt(1 - 1 / g ** 2)
    fld = SimpleNamespace(grid=SimpleNamespace(dx=dx, dy=dx, dz=dx, nx=64))
    # a fixed number of steps per gyroperiod: dt grows with gamma; a 1 GeV
    # particle covers 0.1 cell per step, a 100 GeV one about 11
    g1 = energy_to_gamma(1.0)
    v1 = C_LIGHT * math.sqrt(1 - 1 / g1 ** 2)
    dt = 0.1 * dx / v1 * (g / g1)
    state = {"x1": np.zeros(n), "p1": np.array([p]), "p2": np.array([0.0]), "p3": np.array([0.0])}
    return dict(field=fld, state=state, dt=dt, nsteps=1000, stride=8, E=E_GeV)


def test_tune_batch_selection_and_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("PTB200_TUNE_CACHE", str(tmp_path))
    calls = []

    def fake_trial(camps, storage, capacity, K, bps, sort_every, steps, threads=256):
        calls.append((len(camps), K, bps, tuple(sort_every), threads))
        # slow particles prefer long cadences, fast ones short; 128 threads x 4 blocks per SM best
        cps = B.cells_per_step(camps[0]["field"], camps[0]["state"], camps[0]["dt"])
        best = 128 if cps < 0.5 else (16 if cps > 4 else 64)
        rate = 1e10 / (1 + abs(math.log2(K / best)))
        return rate * (1.0 if (threads, bps) == (128, 4) else 0.9)

    monkeypatch.setattr(B, "_trial", fake_trial)
    camps = [campaign(1.0, 1000), campaign(100.0, 2000), campaign(1.0, 500), campaign(100.0, 700)]
    t = B.tune_batch(camps, "brick_f32", 10_000, use_cache=True)
    cls = [B.speed_class(B.cells_per_step(c["field"], c["state"], c["dt"])) for c in camps]
    assert cls[0] == cls[2] and cls[1] == cls[3] and cls[0] < cls[1]
    assert t["cadence_steps"] == {cls[0]: 128, cls[1]: 16}
    assert t["K"] == 16 and not t["cached"]
    assert (t["threads_per_block"], t["particles_per_thread"], t["blocks_per_sm"]) == (128, 2, 4)
    assert t["sort_every"] == [8, 1, 8, 1]  # 128 / 16 and 16 / 16 epochs
    # each class timed alone at every cadence, then the whole batch at each launch shape
    assert sum(1 for c in calls if c[0] == 2) == 2 * 4
    assert sorted((c[4], c[2]) for c in calls if c[0] == 4) == sorted(B.LAUNCH_SHAPES)
    n_calls = len(calls)
    t2 = B.tune_batch(camps, "brick_f32", 10_000, use_cache=True)
    assert t2["cached"] and len(calls) == n_calls  # served from the JSON file
    for k in ("K", "threads_per_block", "blocks_per_sm", "sort_every"):
        assert t2[k] == t[k], k


def admission_server(budget, room=float("inf")):
    srv = CampaignServer.__new__(CampaignServer)
    srv.budget = budget
    srv.room = room
    srv.device_room = lambda: srv.room - srv.used
    srv.used = 0.0
    srv.queue = []
    srv.active = {}
    srv.admit_s = 0.0
    srv.admit_stats = CampaignServer.new_admit_stats()
    srv._need, srv._blocked_at, srv._blocked_t = {}, None, 0.0
    admitted = []

    def fake_admit(jid, spec, arrival):
        admitted.append(jid)
        srv.active[jid] = {"bytes": srv.job_bytes(spec)}
        srv.used += srv.job_bytes(spec)

    srv._admit = fake_admit
    return srv, admitted


def test_admission_in_order_under_the_budget():
    small = JobSpec("256", "total", 1.0, 10_000, 10.0)
    big = JobSpec("256", "total", 1.0, 4_000_000, 300.0)
    s_b, b_b = CampaignServer.job_bytes(small), CampaignServer.job_bytes(big)
    srv, admitted = admission_server(budget=b_b + 1.5 * s_b)
    for i, spec in enumerate([small, big, small, small]):
        srv.queue.append((i, spec, 0.0))
    assert srv.admit() == 2
    # job 2 no longer fits beside the big job and the first small one; job 3
    # waits behind it
    assert admitted == [0, 1] and [q[0] for q in srv.queue] == [2, 3]
    # the big job leaves: its bytes return to the budget, the rest are admitted
    srv.used -= b_b
    assert srv.admit() == 2 and admitted == [0, 1, 2, 3] and srv.queue == []


def test_admission_holds_later_jobs_behind_one_that_does_not_fit():
    small = JobSpec("256", "total", 1.0, 10_000, 10.0)
    big = JobSpec("256", "total", 1.0, 4_000_000, 300.0)
    srv, admitted = admission_server(budget=CampaignServer.job_bytes(big) * 0.5)
    srv.queue = [(0, big, 0.0), (1, small, 0.0)]
    assert srv.admit() == 0 and admitted == []  # FIFO: the small job does not overtake
    assert [q[0] for q in srv.queue] == [0, 1]


def test_tune_batch_rejects_cadences_that_do_not_divide():
    """A campaign sorts every (cadence / K) epochs with K the shortest cadence
    picked, so each candidate must be a multiple of every shorter one."""
    import pytest

    from particle_transport_b200.batch import check_cadences, tune_batch

    check_cadences((16, 32, 64, 128))
    check_cadences((64, 16))
    for bad in ((16, 48, 64), (32, 48), (0, 16), ()):
        with pytest.raises(ValueError):
            check_cadences(bad)
    with pytest.raises(ValueError, match="multiple"):
        tune_batch([], "brick_bf16", 1, cadences=(16, 48, 64))


def test_dmumu_noalloc_limits_and_job_bytes():
    """The host mirror of the no-alloc entry's limits: series of up to ~20k
    saves at 50 bins stage on chip, 60,000 do not (that call is refused on
    the device, tests/test_zz_no_alloc.py); a job whose series do not fit is
    charged the allocating entry's scratch bound at admission."""
    from particle_transport_b200 import stats as S
    from particle_transport_b200.server import CampaignServer, JobSpec

    assert S.dmumu_noalloc_fits(4001, 64, 50) and S.dmumu_noalloc_fits(20000, 64, 50)
    assert not S.dmumu_noalloc_fits(60000, 2, 50)
    top = max(n for n in range(15000, 30000) if S.dmumu_noalloc_fits(n, 64, 50))
    assert 20000 < top < 22000 and not S.dmumu_noalloc_fits(top + 1, 64, 50)
    assert S.dmumu_noalloc_fits(161, 64, 250) and not S.dmumu_noalloc_fits(401, 64, 250)
    b = S.dmumu_scratch_bound(60000, 64, 50)
    assert 0.5e9 < b < 2e9  # partials + 296 CTAs x 8 global staging slots of ~0.48 MB
    short = JobSpec("256", "total", 1.0, 100_000, 500.0)
    long = JobSpec("256", "total", 1.0, 100_000, 500.0, saves_per_gyroperiod=short.steps_per_gyroperiod)
    nsave = int(round(long.duration_gyroperiods * long.steps_per_gyroperiod))  # + 1 sample, stride 1
    assert not S.dmumu_noalloc_fits(nsave + 1, long.n_lags, long.n_bins)
    extra = S.dmumu_scratch_bound(nsave + 1, long.n_lags, long.n_bins)
    assert S.dmumu_noalloc_fits(4001, short.n_lags, short.n_bins)
    # the long job holds 8x the mu and D_pp momentum caches of the short one and is charged the scratch bound
    cache_diff = (4.0 * long.n_particles + 12.0 * long.dpp_particles) * (nsave + 1 - 4001)
    assert CampaignServer.job_bytes(long) - CampaignServer.job_bytes(short) == cache_diff + extra


def test_admission_also_needs_room_on_the_device():
    """The budget counts the jobs; the device also holds the libraries, the
    arena and scratch.  A job the budget admits waits while the device has
    no room for it, then goes in once a job ends."""
    small = JobSpec("256", "total", 1.0, 10_000, 10.0)
    big = JobSpec("256", "total", 1.0, 4_000_000, 300.0)
    s_b, b_b = CampaignServer.job_bytes(small), CampaignServer.job_bytes(big)
    srv, admitted = admission_server(budget=10 * b_b, room=b_b + 0.5 * s_b)
    srv.queue = [(0, big, 0.0), (1, small, 0.0), (2, small, 0.0)]
    srv.retry_s = 1e9
    assert srv.admit() == 1 and admitted == [0]  # the budget has room; the device does not
    checks = srv.admit_stats["room_checks"]
    assert srv.admit() == 0 and srv.admit_stats["room_checks"] == checks  # no retry before a job ends
    srv.used -= b_b  # the big job ends
    assert srv.admit() == 2 and admitted == [0, 1, 2]
    assert srv.admit_stats["admitted"] == 3 and srv.admit_stats["room_checks"] == 4
