"""Host-side scheduling policy of the campaign server (no GPU).

CampaignServer._select picks the jobs an epoch advances: with
schedule="srpt", the jobs with the least work left (particles x steps to
go), in that order, until they hold fill_particles particles; the batch is
told only when that set changes.  schedule="all" advances every job."""
from particle_transport_b200.server import CampaignServer, JobSpec


class FakeBatch:
    def __init__(self):
        self.calls = []

    def set_running(self, ids=None):
        self.calls.append(None if ids is None else list(ids))


def server(schedule="srpt", fill=1000, K=64):
    srv = CampaignServer.__new__(CampaignServer)
    srv.schedule = schedule
    srv.fill = fill
    srv.K = K
    srv.active = {}
    srv.batch = FakeBatch()
    srv._running_ids = None
    return srv


def job(srv, jid, n, nsteps, epochs=0, cid=None):
    srv.active[jid] = dict(spec=JobSpec("256", "total", 1.0, n, 1.0), cid=jid + 100 if cid is None else cid,
                           nsteps=nsteps, epochs=epochs)


def test_least_work_first_until_filled():
    srv = server(fill=1000)
    job(srv, 0, 800, 1000)           # 800k particle-steps
    job(srv, 1, 600, 100)            # 60k
    job(srv, 2, 100, 2000, epochs=30)  # 100 x (2000 - 1920) = 8k
    job(srv, 3, 5000, 10)            # 50k
    run = srv._select()
    # 2 (8k), 3 (50k): 5100 particles >= 1000, stop
    assert run == [2, 3]
    assert srv.batch.calls == [[102, 103]]
    # same set again: the batch is not called
    assert srv._select() == [2, 3]
    assert len(srv.batch.calls) == 1


def test_always_runs_one_job_and_ties_break_by_id():
    srv = server(fill=0)
    job(srv, 5, 10, 100)
    job(srv, 4, 10, 100)
    assert srv._select() == [4]
    srv = server(fill=10 ** 9)
    job(srv, 0, 10, 100)
    job(srv, 1, 20, 100)
    assert srv._select() == [0, 1]   # fill never reached: everything runs


def test_selection_follows_the_work_left():
    srv = server(fill=1)
    job(srv, 0, 100, 1000)           # 100k
    job(srv, 1, 1000, 200)           # 200k
    assert srv._select() == [0]
    srv.active[0]["epochs"] = 14     # 100 x (1000 - 896) = 10.4k
    assert srv._select() == [0]
    srv.active[1]["epochs"] = 3      # 1000 x (200 - 192) = 8k
    assert srv._select() == [1]
    assert srv.batch.calls == [[100], [101]]


def test_schedule_all_never_pauses():
    srv = server(schedule="all")
    job(srv, 0, 100, 1000)
    job(srv, 1, 1000, 200)
    assert sorted(srv._select()) == [0, 1]
    assert srv.batch.calls == []


def test_unknown_schedule_rejected():
    import pytest

    with pytest.raises(ValueError, match="schedule"):
        CampaignServer({}, {}, schedule="fifo")
