"""Batched campaigns on one device (pt_batch_*) and the launch-shape autotuner.

A Batch holds many campaigns -- the mode x energy campaigns of a run
(run_mode_campaigns, src/multimode_multienergy_cache_pipeline.jl:2924, which
the reference runs one after another), or the jobs of the campaign server --
in one arena of particle slots.  Every epoch one persistent kernel advances
all of them by steps_per_epoch steps from their own device-resident step
counters; epochs replay as CUDA graphs.  Campaigns are added and removed
between epochs.

The tuner (tune_batch) picks a re-sort cadence per speed class of
campaigns (particles that cross a brick every few steps want frequent
sorts, slow ones do not), the steps per epoch and the resident blocks per
SM, timing each on throw-away copies of the campaigns, and caches the result
in a JSON file; autotune sweeps (steps per epoch, blocks per SM) pairs with
a sort before every epoch.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import _lib
from .fields import C_LIGHT, M_P, STORAGE, FieldLibrary

KEYS = ("x1", "x2", "x3", "p1", "p2", "p3")


class Batch:
    def __init__(self, capacity: int, max_campaigns: int = 64, storage: str = "brick_bf16", steps_per_epoch: int = 64,
                 sort: bool = True, blocks_per_sm: int = 0, device: int = 0, threads_per_block: int = 256):
        """threads_per_block (64, 128, 256) and blocks_per_sm (0: 2) set the
        persistent push kernel's launch shape; a thread advances 256 /
        threads_per_block particles of each 256-particle tile."""
        import torch

        self.storage = storage
        self.K = int(steps_per_epoch)
        self.device = torch.device("cuda", device)
        ctx = _lib.torch_context(device)
        out = C.c_void_p()
        _lib.call("pt_batch_create", ctx.handle, int(capacity), int(max_campaigns), STORAGE[storage], self.K,
                  int(bool(sort)), int(blocks_per_sm), C.byref(out))
        self.handle = out
        self.campaigns = {}
        if threads_per_block != 256:
            self.set_launch(threads_per_block, blocks_per_sm if blocks_per_sm > 0 else 2 * 256 // threads_per_block)

    def set_launch(self, threads_per_block: int, blocks_per_sm: int) -> None:
        """pt_batch_set_launch: launch shape of the persistent push kernel."""
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_set_launch", ctx.handle, self.handle, int(threads_per_block), int(blocks_per_sm))

    def add(self, field: FieldLibrary, state: dict, dt: float, nsteps: int, stride: int, periodic: bool = True,
            cache=None, ring: bool = False, deaths=None, alive=None, mom_cache=None, sort_every: int = 1,
            time_fastest: bool = False) -> int:
        """Add a campaign; state: SI arrays x1..p3 (numpy or CUDA tensors);
        cache: CUDA float tensor for the mu cache (or None), [rows][n] (the
        reference's row layout) or, with time_fastest, [n][rows] (each
        particle's saves contiguous, so they reach DRAM as whole sectors);
        mom_cache: CUDA float32 tensor [rows][3][n_mom] that receives the
        momenta of particles 0 .. n_mom-1 at every save (needs cache);
        sort_every: re-sort the campaign by brick before every sort_every-th
        epoch it runs (see sort_cadence for a choice by particle speed)."""
        import torch

        n = int(len(state["x1"]))
        st = {k: torch.as_tensor(np.asarray(state[k]) if not hasattr(state[k], "is_cuda") else state[k],
                                 dtype=torch.float64, device=self.device).contiguous() for k in KEYS}
        al = (torch.ones(n, dtype=torch.uint8, device=self.device) if alive is None
              else torch.as_tensor(alive, dtype=torch.uint8, device=self.device).contiguous())
        rows = pitch = 0
        if cache is not None:
            shape_ok = cache.dim() == 2 and cache.shape[0 if time_fastest else 1] == n
            if cache.dtype not in (torch.float32, torch.float64) or not shape_ok or not cache.is_contiguous():
                raise ValueError("cache must be a contiguous float tensor " + ("[n][rows]" if time_fastest else
                                                                               "[rows][n]"))
            if time_fastest:
                # rows a campaign writes: every save (or the ring's length); the pitch may pad them
                pitch = int(cache.shape[1])
                rows = pitch if ring else min(pitch, (int(nsteps) - 1) // int(stride) + 1)
            else:
                rows = int(cache.shape[0])
        n_mom = 0
        if mom_cache is not None:
            if (cache is None or mom_cache.dtype != torch.float32 or mom_cache.dim() != 3 or mom_cache.shape[1] != 3
                    or mom_cache.shape[0] != rows or not mom_cache.is_contiguous()):
                raise ValueError("mom_cache must be a contiguous float32 tensor [rows][3][n_mom] beside the mu cache")
            n_mom = int(mom_cache.shape[2])
        d = _lib.CampaignDesc(field.handle, float(dt), int(nsteps), int(stride), int(bool(periodic)),
                              int(cache is not None and cache.dtype == torch.float64), n,
                              *[st[k].data_ptr() for k in KEYS], al.data_ptr(),
                              cache.data_ptr() if cache is not None else None, rows, int(bool(ring)),
                              int(sort_every), deaths.data_ptr() if deaths is not None else None,
                              mom_cache.data_ptr() if mom_cache is not None else None, n_mom, pitch)
        cid = C.c_int()
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_add", ctx.handle, self.handle, C.byref(d), C.byref(cid))
        self.campaigns[cid.value] = {"field": field, "n": n, "nsteps": int(nsteps), "cache": cache, "deaths": deaths,
                                     "mom_cache": mom_cache}
        return cid.value

    def remove(self, cid: int) -> None:
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_remove", ctx.handle, self.handle, int(cid))
        self.campaigns.pop(cid, None)

    def run(self, epochs: int, use_graph: bool = True) -> None:
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_run", ctx.handle, self.handle, int(epochs), int(bool(use_graph)))

    def set_running(self, ids=None) -> None:
        """Advance only campaigns `ids` in the following epochs (None: all).
        Paused campaigns keep their slots and step counters and resume where
        they stopped, with the same trajectory."""
        ctx = _lib.torch_context(self.device.index)
        if ids is None:
            _lib.call("pt_batch_set_running", ctx.handle, self.handle, None, -1)
            return
        arr = (C.c_int * max(len(ids), 1))(*[int(i) for i in ids])
        _lib.call("pt_batch_set_running", ctx.handle, self.handle, C.cast(arr, C.c_void_p), len(ids))

    def step(self, cid: int) -> int:
        v = C.c_int64()
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_step", ctx.handle, self.handle, int(cid), C.byref(v))
        return int(v.value)

    def done(self, cid: int) -> bool:
        return self.step(cid) >= self.campaigns[cid]["nsteps"]

    def export(self, cid: int):
        import torch

        n = self.campaigns[cid]["n"]
        st = {k: torch.empty(n, dtype=torch.float64, device=self.device) for k in KEYS}
        al = torch.empty(n, dtype=torch.uint8, device=self.device)
        ctx = _lib.torch_context(self.device.index)
        _lib.call("pt_batch_export", ctx.handle, self.handle, int(cid), *[st[k].data_ptr() for k in KEYS],
                  al.data_ptr())
        return st, al

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().pt_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReferenceBatch:
    """The plain form of a batch: every campaign is pushed by the FP64
    reference-layout kernel (pt_push_advance_device), one launch per campaign
    per epoch, from its own step counter.  Same interface as Batch (add / run /
    step / remove / close), so that the campaign server can run one job stream
    through either push."""

    def __init__(self, steps_per_epoch: int = 64, device: int = 0):
        import torch

        self.K = int(steps_per_epoch)
        self.device = torch.device("cuda", device)
        self.campaigns = {}
        self._next = 0
        self._running = None  # None: all campaigns

    def add(self, field: FieldLibrary, state: dict, dt: float, nsteps: int, stride: int, periodic: bool = True,
            cache=None, alive=None, mom_cache=None, **_unused) -> int:
        """As Batch.add.  With mom_cache, the D_pp subset (particles
        0 .. n_mom-1) is pushed a second time in phase-space mode -- the FP64
        trajectory of a particle does not depend on the others -- and its
        momenta rows land in mom_cache when the campaign finishes."""
        import torch

        from .runner import DeviceEnsemble, push_params

        if field.storage not in ("ref_f64", "brick_f64"):
            raise ValueError("ReferenceBatch pushes ref_f64 or brick_f64 fields")
        # over FP64 bricks the slots are re-sorted by brick every 64 steps
        # (same results: the FP64 push of a particle does not depend on its slot)
        sort_every = 64 if field.storage == "brick_f64" else 0
        n = int(len(state["x1"]))
        al = np.ones(n, np.uint8) if alive is None else alive
        ens = DeviceEnsemble(field, state, al)
        params = push_params(dt, nsteps, stride, periodic, cache="mu" if cache is not None else "none",
                             precision="f64", steps_per_launch=self.K, sort_every=sort_every)
        sub = None
        if mom_cache is not None:
            m = int(mom_cache.shape[2])
            # a copy: DeviceEnsemble advances its state arrays in place, and a
            # prefix of the campaign's arrays would alias the main ensemble
            sub_state = {k: torch.as_tensor(np.asarray(state[k]) if not hasattr(state[k], "is_cuda") else state[k],
                                            dtype=torch.float64, device=self.device)[:m].clone() for k in KEYS}
            sub = dict(ens=DeviceEnsemble(field, sub_state, np.asarray(al)[:m].copy()),
                       params=push_params(dt, nsteps, stride, periodic, cache="phase_space", precision="f64",
                                          steps_per_launch=self.K, sort_every=sort_every),
                       ps=torch.empty((mom_cache.shape[0], 6, m), dtype=torch.float32, device=self.device),
                       out=mom_cache)
        cid = self._next
        self._next += 1
        self.campaigns[cid] = dict(ens=ens, params=params, nsteps=int(nsteps), cache=cache,
                                   rows=0 if cache is None else int(cache.shape[0]), step=0, sub=sub)
        return cid

    def run(self, epochs: int, use_graph: bool = True) -> None:
        for _ in range(int(epochs)):
            for cid, c in self.campaigns.items():
                if c["step"] >= c["nsteps"] or (self._running is not None and cid not in self._running):
                    continue
                count = min(self.K, c["nsteps"] - c["step"])
                c["ens"].advance(c["params"], c["step"], count, c["cache"], 0, c["rows"])
                sub = c["sub"]
                if sub is not None:
                    sub["ens"].advance(sub["params"], c["step"], count, sub["ps"], 0, c["rows"])
                c["step"] += count
                if sub is not None and c["step"] >= c["nsteps"]:
                    sub["out"].copy_(sub["ps"][:, 3:6, :])

    def set_running(self, ids=None) -> None:
        """As Batch.set_running: only campaigns `ids` advance (None: all)."""
        if ids is not None:
            for i in ids:
                if i not in self.campaigns:
                    raise ValueError(f"no such campaign {i}")
        self._running = None if ids is None else set(int(i) for i in ids)

    def step(self, cid: int) -> int:
        return self.campaigns[cid]["step"]

    def remove(self, cid: int) -> None:
        self.campaigns.pop(cid, None)

    def close(self):
        self.campaigns.clear()


# --------------------------------------------------------------------------
# autotuner
# --------------------------------------------------------------------------
CANDIDATES = ((64, 2), (128, 2), (32, 2), (16, 2), (64, 1), (64, 3))


def _cache_path():
    base = os.environ.get("PTB200_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "ptb200")
    os.makedirs(base, exist_ok=True)
    return os.path.join(base, "autotune.json")


def tune_key(storage: str, n_total: int, grid_n: int) -> str:
    import torch

    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return f"{name}|{storage}|n2^{int(round(math.log2(max(n_total, 1))))}|grid{grid_n}"


def autotune(campaigns, storage: str, capacity: int, epochs: int = 2, candidates=CANDIDATES, use_cache: bool = True):
    """Pick (steps_per_epoch, blocks_per_sm) for a set of campaigns.

    campaigns: list of dicts with the keyword arguments of Batch.add (field,
    state, dt, nsteps, stride).  Each candidate runs `epochs` epochs on a fresh
    batch of the same campaigns without caches; the fastest particle-step rate
    wins.  Returns (best, timings)."""
    import torch

    n_total = sum(len(c["state"]["x1"]) for c in campaigns)
    grid_n = max(c["field"].grid.nx for c in campaigns)
    key = tune_key(storage, n_total, grid_n)
    path = _cache_path()
    table = {}
    if use_cache and os.path.exists(path):
        try:
            table = json.load(open(path))
        except Exception:
            table = {}
        if key in table:
            return tuple(table[key]["best"]), table[key]["timings"]
    timings = {}
    for K, bps in candidates:
        b = Batch(capacity, max_campaigns=max(len(campaigns), 1), storage=storage, steps_per_epoch=K, sort=True,
                  blocks_per_sm=bps)
        for c in campaigns:
            b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], c.get("periodic", True))
        b.run(1)  # warm-up (graph capture)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run(epochs)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        b.close()
        timings[f"{K}x{bps}"] = n_total * K * epochs / el
    best_s = max(timings, key=timings.get)
    best = tuple(int(v) for v in best_s.split("x"))
    table[key] = {"best": list(best), "timings": timings}
    try:
        json.dump(table, open(path, "w"), indent=1)
    except Exception:
        pass
    return best, timings


# --------------------------------------------------------------------------
# sort cadence by particle speed
# --------------------------------------------------------------------------
def cells_per_step(field: FieldLibrary, state: dict, dt: float) -> float:
    """Distance the campaign's particles cover per step, in cells, from the
    speed of its first particle (a campaign is mono-energetic)."""
    pm = math.sqrt(sum(float(state[k][0]) ** 2 for k in ("p1", "p2", "p3")))
    gamma = math.sqrt(1.0 + (pm / (M_P * C_LIGHT)) ** 2)
    return cells_per_step_gamma(field, gamma, dt)


def cells_per_step_gamma(field: FieldLibrary, gamma: float, dt: float) -> float:
    """Distance a particle of Lorentz factor gamma covers per step, in cells."""
    g = field.grid
    return C_LIGHT * math.sqrt(max(1.0 - 1.0 / (gamma * gamma), 0.0)) * dt / min(g.dx, g.dy, g.dz)


def speed_class(cps: float) -> int:
    """Campaigns whose particles cover cells per step within a factor of 2
    share a class (and a tuned sort cadence)."""
    return int(math.floor(math.log2(max(cps, 1e-9))))


def sort_cadence(cps: float) -> int:
    """Default re-sort cadence, in steps, for particles covering cps cells per
    step, from the cadences tune_batch picked on a B200 at 256^3 (FP32 bricks,
    64 steps per gyroperiod): 64 steps at 1 GeV (0.1 cell per step) and 10 GeV
    (1 cell; 32-128 within 3 %), 16 steps at 100 GeV (10 cells, 54 % faster
    than 64): the particles of a warp leave each other's bricks within a few
    steps, and a sort brings them back together."""
    if cps >= 4.0:
        return 16
    if cps >= 2.0:
        return 32
    return 64


def _trial(campaigns, storage, capacity, K, bps, sort_every, steps, threads=256):
    """Particle-steps/s of `steps` steps (rounded to whole epochs) of a fresh
    batch of the campaigns, after one warm-up epoch."""
    import torch

    b = Batch(capacity, max_campaigns=max(len(campaigns), 1), storage=storage, steps_per_epoch=K, sort=True,
              blocks_per_sm=bps, threads_per_block=threads)
    for c, se in zip(campaigns, sort_every):
        b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], c.get("periodic", True), sort_every=se)
    epochs = max(1, steps // K)
    b.run(1)  # warm-up (graph capture)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run(epochs)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    b.close()
    return sum(len(c["state"]["x1"]) for c in campaigns) * K * epochs / el


def check_cadences(cadences) -> None:
    """A campaign re-sorts every (its cadence / K) epochs, where K is the
    shortest cadence picked; that is exact only when each candidate cadence is
    a multiple of every shorter one (16, 32, 64, 128 is; 16, 48, 64 is not:
    48 and 64 would give K = 48 and a 64-step class sorting every epoch)."""
    cs = sorted(set(int(c) for c in cadences))
    if not cs or cs[0] < 1:
        raise ValueError("cadences must be positive step counts")
    for i, c in enumerate(cs):
        for d in cs[:i]:
            if c % d:
                raise ValueError(f"cadence {c} is not a multiple of the shorter cadence {d}; each candidate cadence "
                                 "must be a multiple of every shorter one")


# launch shapes of the persistent push tried by tune_batch: (threads per
# block, resident blocks per SM); a thread advances 256 / threads particles of
# a tile, so (128, 2) holds the particles of (256, 1) with half the threads
LAUNCH_SHAPES = ((256, 1), (256, 2), (256, 3), (128, 2), (128, 4), (128, 6))


def tune_batch(campaigns, storage: str, capacity: int, cadences=(16, 32, 64, 128), shapes=LAUNCH_SHAPES,
               steps: int = 256, use_cache: bool = True) -> dict:
    """Launch shape and per-campaign sort cadence of a batch.

    1. Campaigns are grouped by speed class.  For each class alone, every
       cadence in `cadences` is timed as an epoch of that many steps with a
       sort before each; the fastest is the class's cadence.
    2. The batch's steps per epoch K is the shortest cadence picked; each
       campaign re-sorts every (its class's cadence / K) epochs.
    3. Launch shape of the persistent kernel -- threads per block, which sets
       the particles per thread (256 / threads per tile), and resident blocks
       per SM: each of `shapes` is timed on the whole batch with those
       cadences.
    Every trial runs `steps` steps (whole epochs) of a fresh batch without
    caches.  The result is cached in a JSON file keyed by device, storage,
    particle count, grid and speed classes.  Returns {"K", "threads_per_block",
    "particles_per_thread", "blocks_per_sm", "sort_every" (one per campaign,
    in epochs), "cadence_steps" (per class), "timings"}."""
    check_cadences(cadences)
    n_total = sum(len(c["state"]["x1"]) for c in campaigns)
    grid_n = max(c["field"].grid.nx for c in campaigns)
    cls = [speed_class(cells_per_step(c["field"], c["state"], c["dt"])) for c in campaigns]
    key = tune_key(storage, n_total, grid_n) + "|classes" + ",".join(str(v) for v in sorted(set(cls)))
    path = _cache_path()
    table = {}
    if use_cache and os.path.exists(path):
        try:
            table = json.load(open(path))
        except Exception:
            table = {}
    if key in table and "cadence_steps" in table[key] and "threads_per_block" in table[key]:
        hit = table[key]
        cad = {int(k): int(v) for k, v in hit["cadence_steps"].items()}
        K, thr = int(hit["K"]), int(hit["threads_per_block"])
        return {"K": K, "threads_per_block": thr, "particles_per_thread": 256 // thr,
                "blocks_per_sm": int(hit["blocks_per_sm"]), "sort_every": [cad[c] // K for c in cls],
                "cadence_steps": cad, "timings": hit["timings"], "cached": True}
    timings = {}
    cad = {}
    for c in sorted(set(cls)):
        sub = [campaigns[i] for i in range(len(campaigns)) if cls[i] == c]
        rates = {}
        for cs in cadences:
            rates[cs] = _trial(sub, storage, capacity, cs, 2, [1] * len(sub), steps)
            timings[f"class{c}:{cs}"] = rates[cs]
        cad[c] = max(rates, key=rates.get)
    K = min(cad.values())
    sort_every = [cad[c] // K for c in cls]
    rates = {}
    for thr, bps in shapes:
        rates[(thr, bps)] = _trial(campaigns, storage, capacity, K, bps, sort_every, steps, threads=thr)
        timings[f"all:K{K}:{thr}x{bps}"] = rates[(thr, bps)]
    thr, bps = max(rates, key=rates.get)
    table[key] = {"K": K, "threads_per_block": thr, "blocks_per_sm": bps,
                  "cadence_steps": {str(k): v for k, v in cad.items()}, "timings": timings}
    try:
        json.dump(table, open(path, "w"), indent=1)
    except Exception:
        pass
    return {"K": K, "threads_per_block": thr, "particles_per_thread": 256 // thr, "blocks_per_sm": bps,
            "sort_every": sort_every, "cadence_steps": cad, "timings": timings, "cached": False}
