"""Campaign server: continuous batching of transport jobs on one B200.

A job is one campaign (field library, mode, energy, particle count,
duration, injection) plus its D_mumu / <dmu^2> products.  Jobs arrive at
any time (submit); each scheduler tick

  1. admits waiting jobs, in arrival order, while the HBM budget and the
     batch's slot arena have room (the job's particle state, mu cache and
     accumulators are charged against the budget);
  2. picks the jobs this epoch advances and runs one epoch (steps_per_epoch
     pushes of each of them, one persistent launch replayed from a CUDA
     graph).  With schedule="srpt" (the default) those are the jobs with the
     least work left (particles x steps to go), taken in that order until
     they hold fill_particles particles (262,144 by default: 1024 tiles,
     which keep every SM busy at ~75 % of the full-batch rate) while the
     others wait with their state on the device
     (pt_batch_set_running); small jobs then finish in a few epochs instead
     of sharing every epoch with the largest ones.  schedule="all" advances
     every admitted job in every epoch;
  3. for each job that reached its last step, launches its lag-pair binning
     on a side stream -- overlapping the next epoch -- and, once that
     finished, computes the products, records the latency and frees the job.

Particle state stays on the device from admission to the job's results; a
job's trajectory (and so its mu cache) is bit-identical whether it runs
alone or among others, and its D_mumu sums differ only by summation order.
The reference has no serving mode; it runs campaigns back to back
(run_mode_campaigns, src/multimode_multienergy_cache_pipeline.jl:2924).
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field as dfield

import numpy as np

from . import _lib
from . import stats as S
from .batch import Batch, ReferenceBatch, cells_per_step_gamma, sort_cadence
from .fields import FieldLibrary, M_P, Q_E
from .particles import energy_to_gamma, init_particles_device
from .time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0


@dataclass
class JobSpec:
    library: str                 # key of the field library (e.g. "256", "512")
    mode: str                    # total / alfven / fast / slow
    energy_GeV: float
    n_particles: int
    duration_gyroperiods: float
    injection: str = "isotropic"  # or "fixed_mu"
    mu0: float = 0.0
    seed: int = 0
    steps_per_gyroperiod: int = 64
    saves_per_gyroperiod: int = 8
    n_lags: int = 32
    n_bins: int = 20
    start_mode: str = "sliding"
    dpp_particles: int = 65536   # D_pp subset: particles 0 .. min(n, this) - 1 (0: no D_pp)


@dataclass
class JobResult:
    job_id: int
    spec: JobSpec
    arrival: float
    admitted: float
    finished: float
    particle_steps: int
    acc: dict = dfield(default_factory=dict)
    lags: np.ndarray = None
    edges: np.ndarray = None
    mu: np.ndarray = None        # the mu cache, when the server keeps it (keep_cache=True)
    dpp: dict = None             # D_pp sums of the subset on the same lags (counts, sum_delta_p, ...), p0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class CampaignServer:
    def __init__(self, libraries: dict, B0_ref_T: dict, hbm_budget_bytes: float = 150e9, storage: str = "brick_bf16",
                 steps_per_epoch: int = 64, capacity: int = 1 << 26, max_jobs: int = 256, blocks_per_sm: int = 0,
                 keep_cache: bool = False, device: int = 0, push: str = "f32", schedule: str = "srpt",
                 fill_particles: int = 1 << 18, max_epochs_in_flight: int = 2):
        """libraries: {library: {mode: FieldLibrary}} (brick storage for the
        FP32 push; REF_F64 for push="f64", the plain FP64 push);
        B0_ref_T: {library: total-field mean |B|} (time reference of every mode).
        A job's initial state is written on the device from its seed
        (pt_particles_init_device); fixed-mu injection takes the local field
        direction from the job's own field library."""
        import torch

        self.torch = torch
        self.libraries = libraries
        self.B0 = B0_ref_T
        self.budget = float(hbm_budget_bytes)
        self.K = int(steps_per_epoch)
        if push not in ("f32", "f64"):
            raise ValueError("push must be f32 or f64")
        if schedule not in ("srpt", "all"):
            raise ValueError("schedule must be srpt or all")
        self.schedule = schedule
        self.fill = int(fill_particles)
        # epochs enqueued but not finished on the device: the scheduler stays
        # this close to the device, so its choices (and new jobs) take effect
        # within a few epochs instead of behind a long launch queue
        self.depth = max(1, int(max_epochs_in_flight))
        self._inflight = collections.deque()
        self._running_ids = None  # campaign ids set running in the batch (None: all)
        self.push = push
        if push == "f64":
            self.batch = ReferenceBatch(steps_per_epoch=self.K, device=device)
        else:
            self.batch = Batch(capacity, max_campaigns=max_jobs, storage=storage, steps_per_epoch=self.K,
                               blocks_per_sm=blocks_per_sm, device=device)
        self.device = torch.device("cuda", device)
        self.side = torch.cuda.Stream(device=self.device)
        self.side_ctx = _lib.Context(device)
        self.keep_cache = keep_cache
        self.queue = []      # (job_id, spec, arrival)
        self.active = {}     # job_id -> record
        self.binning = {}    # job_id -> record (lag pairs running on the side stream)
        self.results = []
        self.used = 0.0
        self.reserve_bytes = float(2 << 30)  # kept free for the kernels' scratch and torch's workspaces
        self.next_id = 0
        self.epochs = 0
        self.admit_s = 0.0   # host seconds spent admitting jobs
        # where admission time goes: jobs admitted and the seconds of their
        # setup; attempts the device refused (out of memory, no slot range)
        self.admit_stats = self.new_admit_stats()
        self._need = {}               # job id -> bytes charged (job_bytes, computed once)
        self._blocked_at = None       # self.used when the head job last did not fit
        self._blocked_t = 0.0
        self._epoch_events = []

    # ------------------------------------------------------------ admission
    @staticmethod
    def new_admit_stats() -> dict:
        return {"admitted": 0, "admit_setup_s": 0.0, "refused_oom": 0, "refused_slots": 0, "refused_s": 0.0,
                "room_checks": 0, "room_s": 0.0}

    @staticmethod
    def job_bytes(spec: JobSpec) -> float:
        nsteps = int(round(spec.duration_gyroperiods * spec.steps_per_gyroperiod)) + 1
        stride = spec.steps_per_gyroperiod // spec.saves_per_gyroperiod
        nsave = (nsteps - 1) // stride + 1
        n = spec.n_particles
        n_dpp = min(n, max(0, spec.dpp_particles))
        bins = 0 if S.dmumu_noalloc_fits(nsave, spec.n_lags, spec.n_bins) else \
            S.dmumu_scratch_bound(nsave, spec.n_lags, spec.n_bins)  # the allocating entry's scratch
        return (n * (2 * 49 + 49) + 4.0 * n * nsave + 12.0 * n_dpp * nsave + 64 * spec.n_lags * (spec.n_bins + 1) +
                bins)

    def submit(self, spec: JobSpec, arrival: float = None) -> int:
        jid = self.next_id
        self.next_id += 1
        self.queue.append((jid, spec, time.perf_counter() if arrival is None else arrival))
        return jid

    def _admit(self, jid, spec, arrival):
        torch = self.torch
        fl, dt, nsteps, stride, every = job_campaign(spec, self.libraries, self.B0, self.K)
        nsave = (nsteps - 1) // stride + 1
        st = init_particles_device(fl, spec.n_particles, spec.energy_GeV, seed=spec.seed,
                                   injection_mode=spec.injection, mu0=spec.mu0)
        # the FP32 push writes a time-fastest mu cache [n][pitch] (a particle's
        # saves sit side by side and reach DRAM as whole sectors, and the binning stages each series
        # with coalesced reads); the FP64 push writes rows [nsave][n]
        pitch = (nsave + 7) // 8 * 8 if self.push == "f32" else 0
        shape = (spec.n_particles, pitch) if pitch else (nsave, spec.n_particles)
        cache = torch.empty(shape, dtype=torch.float32, device=self.device)
        n_dpp = min(spec.n_particles, max(0, spec.dpp_particles))
        mom = torch.empty((nsave, 3, n_dpp), dtype=torch.float32, device=self.device) if n_dpp else None
        extra = {"time_fastest": True} if pitch else {}
        cid = self.batch.add(fl, st, dt, nsteps, stride, cache=cache, mom_cache=mom, sort_every=every, **extra)
        self._running_ids = None  # a new campaign runs until the next selection
        self.active[jid] = dict(spec=spec, cid=cid, cache=cache, pitch=pitch, mom=mom, nsteps=nsteps, nsave=nsave,
                                arrival=arrival, admitted=time.perf_counter(), bytes=self.job_bytes(spec))
        self.used += self.job_bytes(spec)

    def admit(self) -> int:
        t0 = time.perf_counter()
        try:
            return self._admit_waiting()
        finally:
            self.admit_s += time.perf_counter() - t0

    def device_room(self) -> float:
        """Bytes a new job can still take on the device: free memory plus
        what torch holds cached but unused, less a reserve for workspaces.
        The HBM budget counts the jobs only; the field libraries, the slot
        arena and the scratch of the kernels live beside them, so admission
        checks both."""
        torch = self.torch
        free, _ = torch.cuda.mem_get_info(self.device)
        cached = torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        return float(free + cached) - self.reserve_bytes

    # a head job that did not fit is tried again once a job has released
    # its bytes (self.used fell), or after this many seconds: the budget and
    # the device's room change only when jobs end, and each refused attempt
    # costs a device-memory query or a failed allocation
    retry_s = 0.25

    def _admit_waiting(self) -> int:
        if not self.queue:
            return 0
        if self._blocked_at is not None:
            if self.used >= self._blocked_at and time.perf_counter() - self._blocked_t < self.retry_s:
                return 0
            self._blocked_at = None
        n = 0
        keep = []
        st = self.admit_stats
        need_of = self._need
        for jid, spec, arrival in self.queue:
            if keep:  # arrival order: every later job waits behind the first that does not fit
                keep.append((jid, spec, arrival))
                continue
            need = need_of.get(jid)
            if need is None:
                need = need_of[jid] = self.job_bytes(spec)
            fits = False
            if self.used + need <= self.budget:
                t0 = time.perf_counter()
                fits = need <= self.device_room()
                st["room_checks"] += 1
                st["room_s"] += time.perf_counter() - t0
            if fits:
                t0 = time.perf_counter()
                try:
                    self._admit(jid, spec, arrival)
                    need_of.pop(jid, None)
                    n += 1
                    st["admitted"] += 1
                    st["admit_setup_s"] += time.perf_counter() - t0
                    continue
                except _lib.PtError as e:  # no slot range free yet
                    if e.code not in (-3, -6):
                        raise
                    st["refused_slots"] += 1
                except self.torch.OutOfMemoryError:  # the device is fuller than it looked: wait for a job to end
                    self.torch.cuda.empty_cache()
                    st["refused_oom"] += 1
                st["refused_s"] += time.perf_counter() - t0
            keep.append((jid, spec, arrival))
            self._blocked_at, self._blocked_t = self.used, time.perf_counter()
        self.queue = keep
        return n

    # ------------------------------------------------------------ ticks
    def _start_binning(self, jid, rec):
        torch = self.torch
        spec = rec["spec"]
        done = torch.cuda.Event()
        done.record()  # after the job's last epoch on the main stream
        lags = log_spaced_lag_steps(rec["nsave"] - 1, spec.n_lags)
        edges, _ = build_mu_edges_full(0.0, 1.0, spec.n_bins)
        with torch.cuda.stream(self.side):
            self.side.wait_event(done)
            acc = S.new_dmumu_accumulators(len(lags), spec.n_bins, device=self.device)
            # pinned sources and non-blocking copies: a pageable copy would
            # wait here for the side stream, i.e. for the binning of every
            # job before this one, and stall the epochs behind it
            d_lags = torch.as_tensor(lags).pin_memory().to(self.device, non_blocking=True)
            d_edges = torch.as_tensor(edges).pin_memory().to(self.device, non_blocking=True)
            self.side_ctx.use_stream(self.side)
            cache = rec["cache"]
            sp, ss = (rec["pitch"], 1) if rec["pitch"] else (1, spec.n_particles)
            args = (self.side_ctx.handle, _lib.ptr(cache), spec.n_particles, rec["nsave"], sp, ss,
                    _lib.ptr(d_lags), len(lags), _lib.ptr(d_edges), spec.n_bins, S.START[spec.start_mode], 1,
                    *[_lib.ptr(acc[k]) for k in ("dmumu_counts", "dmumu_sum_delta", "dmumu_sum_delta2",
                                                 "particle_counts", "particle_means", "particle_m2s",
                                                 "pair_sum_squares", "pair_counts")])
            # the entry that allocates nothing: a scratch regrowth in the
            # allocating one would free memory, and cudaFree waits for the
            # whole device -- the epochs and every earlier job's binning.
            # All binning runs on this one side stream, so its calls never
            # overlap on the fixed scratch.  Series too long to stage on chip
            # take the allocating entry, whose scratch job_bytes counts; any
            # error of either entry is raised.
            if S.dmumu_noalloc_fits(rec["nsave"], len(lags), spec.n_bins):
                _lib.call("pt_dmumu_accumulate_device_noalloc", *args)
            else:
                _lib.call("pt_dmumu_accumulate_device", *args)
            dpp = None
            if rec["mom"] is not None:
                # D_pp of the subset with p0 = 1: the kernel normalises once per
                # lag (sum dp / p0, sum dp^2 / p0 / p0), so dividing by the true
                # p0 when the result is collected gives the same values without
                # reading p0 back here
                mom = rec["mom"]
                dpp = S.new_dpp_accumulators(len(lags), device=self.device)
                _lib.call("pt_dpp_accumulate_device", self.side_ctx.handle, _lib.ptr(mom), mom.shape[2],
                          rec["nsave"], _lib.ptr(d_lags), len(lags), 1.0,
                          *[_lib.ptr(dpp[k]) for k in ("counts", "sum_delta_p", "sum_delta_p2", "sum_delta_p_norm",
                                                       "sum_delta_p_norm2")])
            ev = torch.cuda.Event()
            ev.record(self.side)
        rec.update(acc=acc, dpp=dpp, lags=lags, edges=edges, ev=ev, keep=(d_lags, d_edges))
        self.binning[jid] = rec

    @staticmethod
    def _dpp_result(rec):
        """D_pp sums of a finished job normalised by p0 = |p| of its first
        particle at the first save (compute_dpp_full.jl:483), as the reference."""
        if rec["dpp"] is None:
            return None
        d = {k: v.cpu().numpy() for k, v in rec["dpp"].items()}
        m = rec["mom"][0, :, 0].cpu().double().numpy()
        p0 = math.sqrt(float(m[0]) * float(m[0]) + float(m[1]) * float(m[1]) + float(m[2]) * float(m[2]))
        if not (math.isfinite(p0) and p0 > 0.0):
            d["sum_delta_p_norm"] = np.full_like(d["sum_delta_p_norm"], np.nan)
            d["sum_delta_p_norm2"] = np.full_like(d["sum_delta_p_norm2"], np.nan)
        else:
            d["sum_delta_p_norm"] = d["sum_delta_p_norm"] / p0
            d["sum_delta_p_norm2"] = d["sum_delta_p_norm2"] / p0 / p0
        d["p0"] = p0
        return d

    def _work_left(self, rec) -> int:
        """Particle-steps a job still has to push."""
        return rec["spec"].n_particles * max(rec["nsteps"] - rec.get("epochs", 0) * self.K, 0)

    def _select(self):
        """Jobs the next epoch advances (see the module docstring)."""
        if self.schedule == "all":
            return list(self.active)
        order = sorted(self.active, key=lambda j: (self._work_left(self.active[j]), j))
        run, fill = [], 0
        for jid in order:
            if run and fill >= self.fill:
                break
            run.append(jid)
            fill += self.active[jid]["spec"].n_particles
        ids = sorted(self.active[j]["cid"] for j in run)
        if ids != self._running_ids:
            self.batch.set_running(ids)
            self._running_ids = ids
        return run

    def tick(self):
        """One scheduling step; returns the jobs finished in it."""
        self.admit()
        while self._inflight and self._inflight[0].query():
            self._inflight.popleft()
        if self.active and len(self._inflight) < self.depth:
            run = self._select()
            ev0, ev1 = self.torch.cuda.Event(enable_timing=True), self.torch.cuda.Event(enable_timing=True)
            ev0.record()
            self.batch.run(1)
            ev1.record()
            self._inflight.append(ev1)
            self._epoch_events.append((ev0, ev1))
            self.epochs += 1
            for jid in run:
                rec = self.active[jid]
                # a job advances K steps in every epoch it is selected for
                rec.setdefault("epochs", 0)
                rec["epochs"] += 1
                if rec["epochs"] * self.K >= rec["nsteps"]:
                    del self.active[jid]
                    self._start_binning(jid, rec)
        out = []
        for jid in list(self.binning):
            rec = self.binning[jid]
            if rec["ev"].query():
                spec = rec["spec"]
                # read back on the side stream, which has finished this job's
                # work: a copy on the main stream would wait for the epochs
                with self.torch.cuda.stream(self.side):
                    acc = {k: v.cpu().numpy() for k, v in rec["acc"].items()}
                    mu = None
                    if self.keep_cache:  # the reference's row layout [nsave][n]
                        mu = rec["cache"].cpu().numpy()
                        if rec["pitch"]:
                            mu = np.ascontiguousarray(mu[:, :rec["nsave"]].T)
                    dpp = self._dpp_result(rec)
                res = JobResult(jid, spec, rec["arrival"], rec["admitted"], time.perf_counter(),
                                spec.n_particles * (rec["nsteps"] - 1), acc, rec["lags"], rec["edges"], mu, dpp)
                self.batch.remove(rec["cid"])
                self._running_ids = None
                self.used -= rec["bytes"]
                del self.binning[jid]
                self.results.append(res)
                out.append(res)
        return out

    def device_busy_s(self) -> float:
        """Device seconds spent in epochs so far (CUDA events around each)."""
        self.torch.cuda.synchronize(self.device)
        return sum(a.elapsed_time(b) for a, b in self._epoch_events) / 1e3

    def idle(self) -> bool:
        return not (self.queue or self.active or self.binning)

    def run_until_idle(self, timeout_s: float = None):
        """Tick until every submitted job has returned its results (or
        timeout_s seconds passed); returns the results so far."""
        t0 = time.perf_counter()
        while not self.idle():
            if timeout_s is not None and time.perf_counter() - t0 > timeout_s:
                break
            epochs = self.epochs
            self.tick()
            if self.epochs == epochs:
                time.sleep(5e-5)  # nothing to enqueue now: epochs in flight, or binning to finish
        return self.results

    def close(self):
        self.batch.close()
        self.side_ctx.close()


def job_campaign(spec: JobSpec, libraries: dict, B0_ref_T: dict, steps_per_epoch: int):
    """The campaign of a job: (field library, dt, samples, save stride,
    re-sort cadence in epochs).  dt resolves steps_per_gyroperiod of the
    reference gyroperiod of the library's total field at the job's energy;
    fast particles leave their bricks within a few steps, so the cadence
    comes from the particle speed (taken from the energy: no device read)."""
    fl = libraries[spec.library][spec.mode]
    g0 = energy_to_gamma(spec.energy_GeV)
    Om = reference_Omega0(B0_ref_T[spec.library], g0, Q_E, M_P)
    dt = (2 * math.pi / spec.steps_per_gyroperiod) / Om
    nsteps = int(round(spec.duration_gyroperiods * spec.steps_per_gyroperiod)) + 1
    stride = spec.steps_per_gyroperiod // spec.saves_per_gyroperiod
    every = max(1, sort_cadence(cells_per_step_gamma(fl, g0, dt)) // steps_per_epoch)
    return fl, dt, nsteps, stride, every


def sample_jobs(n_jobs: int, rate_per_s: float, libraries, seed: int = 2026, n_range=(16_384, 8_388_608),
                energy_range=(1.0, 300.0), duration_range=(10.0, 300.0)):
    """A Poisson stream of jobs: arrival offsets (s) and specs, seeded by job index."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, size=n_jobs))
    specs = []
    for i in range(n_jobs):
        lib = libraries[int(rng.integers(len(libraries)))]
        mode = ("total", "alfven", "fast", "slow")[int(rng.integers(4))]
        E = float(np.exp(rng.uniform(np.log(energy_range[0]), np.log(energy_range[1]))))
        n = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        dur = float(rng.uniform(*duration_range))
        inj = "isotropic" if rng.random() < 0.5 else "fixed_mu"
        mu0 = float(rng.uniform(-1, 1))
        specs.append(JobSpec(lib, mode, E, n, dur, inj, mu0, seed=1000 + i))
    return t, specs
