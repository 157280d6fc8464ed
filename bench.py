#!/usr/bin/env python
"""Benchmark of the trajectory / transport-statistics hot path on B200.

Workload (the large single campaign at 512^3): anisotropic
Goldreich-Sridhar-like turbulence, dB/B0 = 1, u_rms = v_A = 1e-4 c
(E = -u x B), 512^3 nodes with the cell = one 1 GeV gyroradius in
B0 = 1 uG; 16,777,216 protons at 10 GeV, uniform positions, isotropic
momenta; 64 steps per reference gyroperiod (B0_ref = mean |B|), mu cache
every 8 steps.  Seeded synthetic inputs stand in for the MHD snapshots,
which do not ship with the reference.

One bench step = 64 pushes (one T_g0) of every particle with the 8 mu-cache
rows written on the device.  `value` is particle-steps/s of the FP32 push
over BF16 Morton bricks with the state resident in HBM; beside it the plain
FP64 push (reference layout, bit-exact with the reference arithmetic) on
the same particles, the D_mumu lag-pair rate on a full-length (500 T_g0,
4001 saves) campaign of 1,048,576 particles, and `e2e`: the same metric
through pt_push_run with host buffers (state upload, per-save rows to
pinned host memory, state download inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun every rank pushes its own 16,777,216 particles (weak scaling,
no collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 512³ (mixed vs FP64 push); D_μμ lag-pairs/s; job p50/p99"
UNIT = "particle-steps/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}

# Bytes the push must move per particle-step (BF16 bricks): 8 corners x 6
# components x 2 B.  Per launch each particle also reads and writes its
# state (x 24 B, p 12 B, |p|^2 8 B, id 4 B, alive 1 B) and writes one 4-byte
# mu per save row.
GATHER_BYTES = {"brick_bf16": 96, "brick_bf16x": 96, "brick_f32": 192, "ref_f64": 384}
STATE_BYTES = {"brick_bf16": 49, "brick_bf16x": 49, "brick_f32": 49, "ref_f64": 49}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--particles", type=int, default=16_777_216)
    ap.add_argument("--energy", type=float, default=10.0)
    ap.add_argument("--storage", default="brick_bf16", choices=["brick_bf16", "brick_bf16x", "brick_f32"])
    ap.add_argument("--sort-every", type=int, default=64, help="re-sort particles by brick every N pushes (0: never)")
    ap.add_argument("--variant", type=int, default=1, help="push launch shape (pt_push_params.kernel_variant)")
    ap.add_argument("--lag-particles", type=int, default=1_048_576)
    ap.add_argument("--dpp-particles", type=int, default=262_144)
    ap.add_argument("--e2e-gyroperiods", type=int, default=500,
                    help="T_g0 per pt_push_run call in the e2e leg: the whole 512^3 campaign (500 T_g0), as the "
                         "reference pushes a campaign per run_mu_cache_ensemble call")
    ap.add_argument("--skip", default="",
                    help="comma list of legs to skip: fp32b,fp64,lag,dpp,e2e,cpu,batch,serve,config1,precision")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--serve-jobs", type=int, default=100, help="jobs of the serving stream")
    ap.add_argument("--serve-cmp", type=int, default=16, help="jobs of the FP32-vs-FP64 serving comparison")
    ap.add_argument("--serve-all", action="store_true", help="also serve the stream with every job in every epoch")
    ap.add_argument("--serve-fill", type=int, default=1 << 18, help="particles the server's epochs are filled to")
    ap.add_argument("--serve-fill-sweep", default="",
                    help="comma list of epoch fills to serve the same stream with (reported as fill_sweep)")
    ap.add_argument("--precision", action="store_true",
                    help="run only the plain-vs-precision study (256^3, 3 energies) and print its JSON line")
    ap.add_argument("--precision-key-particles", type=int, default=1048576,
                    help="particles per case of the default line's precision key")
    ap.add_argument("--precision-grid", type=int, default=256)
    ap.add_argument("--precision-particles", type=int, default=1_048_576)
    ap.add_argument("--precision-gyroperiods", type=int, default=200)
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return ws, rank, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return PEAKS_FALLBACK


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_workload(args, device, rank):
    import torch

    from particle_transport_b200 import fields as F
    from particle_transport_b200.particles import energy_to_gamma, init_particles
    from particle_transport_b200.time_units import reference_Omega0

    n = args.grid
    f_uG = F.synthetic_mhd_fields(n, 2, n // 2, 1.0, 1.0, 1e-4, seed=20260423, spectrum="gs", device=device)
    fields = F.to_si(f_uG)
    del f_uG
    rg = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((n - 1) * rg, n, n, n)
    B0 = F.reference_B0_T(*fields[:3])
    g0 = energy_to_gamma(args.energy)
    Om = reference_Omega0(B0, g0, F.Q_E, F.M_P)
    dt = (2 * math.pi / 64) / Om  # 64 steps per T_g0 (resolve_trajectory_time_grid)
    state = init_particles(args.particles, grid, args.energy, seed=42 + rank)
    return fields, grid, B0, dt, state


def timed(fn, K, W, torch, per_step=True):
    for _ in range(W):
        fn(-1)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    evs[0].record()
    for k in range(K):
        fn(k)
        evs[k + 1].record()
    torch.cuda.synchronize()
    steps = [evs[k].elapsed_time(evs[k + 1]) for k in range(K)]
    return evs[0].elapsed_time(evs[K]), steps


def host_threads() -> int:
    """Host threads this process may run on (torchrun sets OMP_NUM_THREADS=1
    per rank; the CPU baselines pass this count to the oracle explicitly)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_push_rate(fields_host, grid, state, dt, seconds):
    """Oracle FP64 push (restatement of the reference's push) on all host cores."""
    from oracle import build as ob
    from oracle import oracle as o

    ob.build()
    ff = [np.asfortranarray(f.T) for f in fields_host]
    nthreads = host_threads()
    n = 4096
    sample = None
    while True:
        st = {k: np.ascontiguousarray(v[:n]).copy() for k, v in state.items()}
        t0 = time.perf_counter()
        o.push_run(ff, grid, st, np.ones(n, np.uint8), dt, 32001, 8, cache_mode=1, step_begin=0, step_count=64,
                   nthreads=nthreads)
        el = time.perf_counter() - t0
        if el * 4 >= seconds or n >= len(state["x1"]):
            sample = (n, 64, el)
            break
        n = min(len(state["x1"]), int(n * max(2.0, min(16.0, seconds / 4 / max(el, 1e-3)))))
    n, steps, el = sample
    reps = max(1, int(round(seconds / max(el, 1e-3))))
    st = {k: np.ascontiguousarray(v[:n]).copy() for k, v in state.items()}
    t0 = time.perf_counter()
    for r in range(reps):
        o.push_run(ff, grid, st, np.ones(n, np.uint8), dt, 32001, 8, cache_mode=1, step_begin=64 * r, step_count=64,
                   nthreads=nthreads)
    el = time.perf_counter() - t0
    return {"value": n * 64 * reps / el, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{n} particles x {64 * reps} FP64 steps (mu cache every 8) of the same workload, "
                      f"{el:.1f} s on {nthreads} threads"}


def cpu_lag_rate(mu_chunk, lags, edges, seconds):
    from oracle import oracle as o

    nl, nb = len(lags), len(edges) - 1
    n = 64
    while True:
        acc = {"counts": np.zeros((nl, nb), np.int64), "sum_d": np.zeros((nl, nb)), "sum_d2": np.zeros((nl, nb)),
               "w_count": np.zeros(nl, np.int64), "w_mean": np.zeros(nl), "w_m2": np.zeros(nl),
               "pair_ss": np.zeros(nl), "pair_n": np.zeros(nl, np.int64)}
        t0 = time.perf_counter()
        o.dmumu_accumulate(mu_chunk[:n], lags, edges, acc, nthreads=host_threads())
        el = time.perf_counter() - t0
        if el * 2 >= seconds or n >= mu_chunk.shape[0]:
            break
        n = min(mu_chunk.shape[0], int(n * max(2.0, min(16.0, seconds / 2 / max(el, 1e-3)))))
    pairs = int(acc["pair_n"].sum())
    return {"value": pairs / el, "unit": "lag-pairs/s", "cores": host_threads(), "kind": "port",
            "sample": f"{n} particles x {mu_chunk.shape[1]} saves x {len(lags)} lags ({pairs} pairs), {el:.1f} s"}


def cpu_dpp_rate(mom, lags, p0, seconds):
    """D_pp lag pairs/s of the oracle on host cores; mom (nsave, 3, n) float32."""
    from oracle import oracle as o

    nl = len(lags)
    n = 64
    while True:
        acc = {"counts": np.zeros(nl, np.int64), **{k: np.zeros(nl) for k in ("sum_dp", "sum_dp2", "sum_dpn",
                                                                               "sum_dpn2")}}
        sub = np.ascontiguousarray(mom[:, :, :n])
        t0 = time.perf_counter()
        o.dpp_accumulate(sub, lags, p0, acc, nthreads=host_threads())
        el = time.perf_counter() - t0
        if el * 2 >= seconds or n >= mom.shape[2]:
            break
        n = min(mom.shape[2], int(n * max(2.0, min(16.0, seconds / 2 / max(el, 1e-3)))))
    pairs = int(acc["counts"].sum())
    return {"value": pairs / el, "unit": "lag-pairs/s", "cores": host_threads(), "kind": "port",
            "sample": f"{n} particles x {mom.shape[0]} saves x {nl} lags ({pairs} pairs), {el:.1f} s"}


# ---------------------------------------------------------------------------
def run_reference(args, ws, rank):
    """Reference arm: the reference's push has no CPU path, so its CPU
    restatement (the oracle, FP64, reference operation order) is timed on all
    host threads over bounded samples of the same workload."""
    if rank != 0:
        return
    import torch

    from oracle import build as ob
    from oracle import oracle as o

    ob.build()
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    fields, grid, B0, dt, state = make_workload(args, dev, 0)
    fields_host = [f.cpu().numpy() for f in fields]
    del fields
    ff = [np.asfortranarray(f.T) for f in fields_host]
    nthreads = host_threads()
    # size one step (a sample of the particles over 64 pushes) at ~3 s
    n = min(4096, args.particles)
    while True:
        st = {k: np.ascontiguousarray(v[:n]).copy() for k, v in state.items()}
        t0 = time.perf_counter()
        o.push_run(ff, grid, st, np.ones(n, np.uint8), dt, 32001, 8, cache_mode=1, step_begin=0, step_count=64,
                   nthreads=nthreads)
        el = time.perf_counter() - t0
        if el >= 1.5 or n >= args.particles:
            break
        n = min(args.particles, int(n * max(2.0, min(16.0, 3.0 / max(el, 1e-3)))))
    st = {k: np.ascontiguousarray(v[:n]).copy() for k, v in state.items()}
    al = np.ones(n, np.uint8)
    for w in range(args.warmup):
        o.push_run(ff, grid, st, al, dt, 32001, 8, cache_mode=1, step_begin=64 * w, step_count=64,
                   nthreads=nthreads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        o.push_run(ff, grid, st, al, dt, 32001, 8, cache_mode=1, step_begin=64 * (args.warmup + k), step_count=64,
                   nthreads=nthreads)
    el = time.perf_counter() - t0
    value = n * 64 * args.steps / el
    sample = f"{n} of {args.particles} particles per step x 64 FP64 pushes (mu cache every 8)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded GS turbulence, seeded particles)",
            "config": {"workload": f"{args.grid}^3 GS turbulence, 10 GeV protons, 64 steps/T_g0, mu cache every 8",
                       "sample": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (Julia + CUDA.jl) cannot run here; its push exists only as a CUDA.jl kernel, so "
                    "this arm times the CPU restatement of its Float64 push (oracle/pt_oracle.c)"}
    print(json.dumps(line), flush=True)


def leg(name, fn, *a):
    """Run one auxiliary leg of the line (no collectives inside);
    a failure is recorded in the line as {"error": ...} with the traceback on
    stderr, so the headline and the other legs still report."""
    import traceback

    import torch

    t0 = time.perf_counter()
    try:
        out = fn(*a)
    except Exception as e:  # noqa: BLE001 -- reported, not swallowed
        traceback.print_exc()
        out = {"error": f"{type(e).__name__}: {e}"}
    torch.cuda.empty_cache()
    print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
    return out


def run_ours(args, ws, rank, local):
    import torch

    from particle_transport_b200 import _lib
    from particle_transport_b200 import runner as R
    from particle_transport_b200 import stats as S
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps

    skip = set(filter(None, args.skip.split(",")))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    fields, grid, B0, dt, state = make_workload(args, dev, rank)
    n = args.particles
    NSTEPS = 32001  # 500 T_g0 at 64 steps per T_g0
    STRIDE = 8
    K, W = args.steps, args.warmup
    launches = {"push": 0, "sort": 0}

    # ---------------- FP32 push over bricks (headline)
    fb = FieldLibrary(fields, grid, args.storage, B_ref_T=B0)
    alive = np.ones(n, np.uint8)
    ens = R.FastEnsemble(fb, state, alive)
    # the 8 mu saves of a 64-step launch land in a time-fastest cache [n][8]:
    # each particle's saves side by side (cache_pitch = 8), merged by L2 into whole sectors
    ring = torch.empty((n, 8), dtype=torch.float32, device=dev)
    # the sort cadence is driven here (same rule as pt_push_advance_fast's
    # sort_every) so that events can bracket the push launch alone
    params = R.push_params(dt, NSTEPS, STRIDE, cache="mu", precision="f32", kernel_variant=args.variant,
                           cache_pitch=8)
    step_at = [0]
    last_sort = [None]
    push_ev = []

    def fast_step(k):
        s0 = step_at[0]
        if args.sort_every and (last_sort[0] is None or s0 - last_sort[0] >= args.sort_every):
            ens.sort()
            last_sort[0] = s0
            if k >= 0:
                launches["sort"] += 4  # sort_key, sort_scan_tiles, sort_scan_top, sort_scatter
        if k >= 0:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        ens.advance(params, s0, 64, ring, s0 // STRIDE, 8)
        if k >= 0:
            e1.record()
            push_ev.append((e0, e1))
            launches["push"] += 1
        step_at[0] = s0 + 64

    dist_barrier(ws)
    with ClockSampler(local) as clk:
        total_ms, steps_ms = timed(fast_step, K, W, torch)
    total_ms = max_over_ranks(total_ms, ws, dev)
    value = ws * n * 64 * K / (total_ms / 1e3)
    clocks = clk.summary()

    # roofline of the push kernel: algorithmic bytes per launch / launch time
    peaks = load_peaks()
    bpl = n * (64 * GATHER_BYTES[args.storage] + 2 * STATE_BYTES[args.storage] + 8 * 4)
    launch_ms = float(np.mean([a.elapsed_time(b) for a, b in push_ev]))
    achieved = bpl / (launch_ms / 1e3) / 1e9
    roofline = {"kernel": "push_fast_kernel", "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": TRAFFIC.get((args.storage, args.grid, n)),
                "algorithmic_bytes_per_launch": bpl, "launch_ms": launch_ms,
                "sort_ms_per_step": float(np.mean(steps_ms)) - launch_ms}
    if rank == 0:
        print(f"[bench] headline {value:.4g} {UNIT}, push launch {launch_ms:.2f} ms, frac {roofline['frac']:.3f}",
              file=sys.stderr, flush=True)

    # ---------------- the same push over FP32 bricks (the field's second storage)
    fp32b = None
    if "fp32b" not in skip and args.storage != "brick_f32":
        f32 = FieldLibrary(fields, grid, "brick_f32", B_ref_T=B0)
        ens32 = R.FastEnsemble(f32, state, alive)
        p32 = R.push_params(dt, NSTEPS, STRIDE, cache="mu", precision="f32", sort_every=args.sort_every,
                            kernel_variant=args.variant, cache_pitch=8)
        at32 = [0]

        def f32_step(k):
            ens32.advance(p32, at32[0], 64, ring, at32[0] // STRIDE, 8)
            at32[0] += 64

        K32 = max(2, K // 2)
        ms32, _ = timed(f32_step, K32, max(3, min(W, 3)), torch)
        ms32 = max_over_ranks(ms32, ws, dev)
        fp32b = {"value": ws * n * 64 * K32 / (ms32 / 1e3), "unit": UNIT, "ms_per_step": ms32 / K32, "steps": K32,
                 "field": "brick_f32", "field_bytes": f32.device_bytes,
                 "gather_bytes_per_particle_step": GATHER_BYTES["brick_f32"]}
        ens32.close()
        del ens32, f32
        torch.cuda.empty_cache()

    # ---------------- FP64 plain push on the same particles
    fp64 = None
    if "fp64" not in skip:
        ring = torch.empty((8, n), dtype=torch.float32, device=dev)  # the FP64 push writes mu rows [8][n]
        fr = FieldLibrary(fields, grid, "ref_f64")
        dens = R.DeviceEnsemble(fr, state, alive)
        p64 = R.push_params(dt, NSTEPS, STRIDE, cache="mu", precision="f64", steps_per_launch=64)
        at = [0]

        def f64_step(k):
            dens.advance(p64, at[0], 64, ring, at[0] // STRIDE, 8)
            at[0] += 64

        K64 = max(2, K // 2)
        ms64, _ = timed(f64_step, K64, max(1, min(W, 3)), torch)
        ms64 = max_over_ranks(ms64, ws, dev)
        v64 = ws * n * 64 * K64 / (ms64 / 1e3)
        fp64 = {"value": v64, "unit": UNIT, "ms_per_step": ms64 / K64, "steps": K64, "dtype": "f64",
                "field": "reference layout, six FP64 arrays", "speedup_mixed_vs_fp64": value / v64}
        del dens, fr
        torch.cuda.empty_cache()
        # the same FP64 push over FP64 bricks: SI node values in Morton
        # bricks, slots re-sorted by brick every 64 steps; bit-identical results
        # (the cache and state of every particle; tested against the oracle)
        fb64 = FieldLibrary(fields, grid, "brick_f64")
        dens_b = R.DeviceEnsemble(fb64, state, alive)
        p64b = R.push_params(dt, NSTEPS, STRIDE, cache="mu", precision="f64", steps_per_launch=64, sort_every=64)
        at[0] = 0

        def f64b_step(k):
            dens_b.advance(p64b, at[0], 64, ring, at[0] // STRIDE, 8)
            at[0] += 64

        ms64b, _ = timed(f64b_step, K64, max(1, min(W, 3)), torch)
        ms64b = max_over_ranks(ms64b, ws, dev)
        v64b = ws * n * 64 * K64 / (ms64b / 1e3)
        fp64["bricks"] = {"value": v64b, "unit": UNIT, "ms_per_step": ms64b / K64, "steps": K64,
                          "field": "FP64 bricks (Morton 8^3, SI node values in a 32-byte and a 16-byte plane), slots re-sorted by brick "
                                   "every 64 steps (imported, sorted and scattered back within each call)",
                          "field_bytes": fb64.device_bytes, "speedup_vs_reference_layout": v64b / v64,
                          "speedup_mixed_vs_fp64_bricks": value / v64b}
        del dens_b, fb64
        torch.cuda.empty_cache()
    del ens, ring
    torch.cuda.empty_cache()

    # ---------------- D_mumu lag pairs on a full-length campaign subset
    lag = None
    if "lag" not in skip:
        nl = min(args.lag_particles, n)
        sub = {k: v[:nl] for k, v in state.items()}
        ens_l = R.FastEnsemble(fb, sub, np.ones(nl, np.uint8))
        nsave = (NSTEPS - 1) // STRIDE + 1
        pitch = (nsave + 7) // 8 * 8  # time-fastest cache [nl][pitch], each particle's saves contiguous
        cache = torch.empty((nl, pitch), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens_l.advance(R.push_params(dt, NSTEPS, STRIDE, cache="mu", precision="f32", sort_every=args.sort_every,
                                    kernel_variant=args.variant, cache_pitch=pitch), 0, NSTEPS, cache, 0, nsave)
        torch.cuda.synchronize()
        push_full_s = time.perf_counter() - t0
        lags = log_spaced_lag_steps(nsave - 1, 64)
        edges, _ = build_mu_edges_full(0.0, 1.0, 50)

        def lag_pass(_k):
            acc = S.new_dmumu_accumulators(len(lags), 50, device=dev)
            S.process_mu_chunk_dmumu(cache, lags, edges, acc["particle_counts"], acc["particle_means"],
                                     acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                                     acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                                     start_mode="sliding", bin_abs=True, layout="time_fastest", nsave=nsave)
            lag_pass.acc = acc

        lms, _ = timed(lag_pass, 2, 1, torch)
        pairs = int(lag_pass.acc["pair_counts"].sum().item())
        lag_s = lms / 2 / 1e3
        lag = {"value": ws * pairs / max_over_ranks(lag_s * 1e3, ws, dev) * 1e3, "unit": "lag-pairs/s",
               "pairs_per_pass": pairs, "ms_per_pass": lms / 2, "particles": nl, "saves": nsave,
               "lags": int(len(lags)), "mu_bins": 50, "estimator": "sliding, |mu| bins",
               "compulsory_bytes_per_pass": 4 * nl * nsave,
               "hbm_frac_of_compulsory": (4 * nl * nsave / lag_s / 1e9) / peaks["hbm_gbs"],
               "campaign_push_s": push_full_s,
               "campaign_push_rate": nl * (NSTEPS - 1) / push_full_s}
        lag["roofline"] = issue_roofline("dmumu_kernel", lag["value"] / ws, clocks, dev)
        if ws > 1:
            # the job's products: every rank's accumulators merged in rank order
            from particle_transport_b200 import shard
            merged = shard.reduce_dmumu_accumulators(lag_pass.acc)
            lag["merged"] = {"pair_counts": int(merged["pair_counts"].sum()),
                             "particle_counts": int(merged["particle_counts"].max()), "ranks": ws}
        if "cpu" not in skip and rank == 0:
            mu_host = np.ascontiguousarray(cache[:4096, :nsave].cpu().numpy())
            lag["cpu_baseline"] = cpu_lag_rate(mu_host, lags, edges, args.cpu_seconds / 2)
        del ens_l, cache
        torch.cuda.empty_cache()

    # ---------------- D_pp (64 lags) and 16 energy-snapshot histograms on a phase-space campaign subset
    dpp = None
    if "dpp" not in skip:
        from particle_transport_b200.time_units import selected_energy_snapshot_indices
        from particle_transport_b200.particles import energy_to_gamma

        npp = min(args.dpp_particles, n)
        sub = {k: v[:npp] for k, v in state.items()}
        ens_p = R.FastEnsemble(fb, sub, np.ones(npp, np.uint8))
        nsave = (NSTEPS - 1) // STRIDE + 1
        ps = torch.empty((nsave, 6, npp), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens_p.advance(R.push_params(dt, NSTEPS, STRIDE, cache="phase_space", precision="f32",
                                    sort_every=args.sort_every, kernel_variant=args.variant), 0, NSTEPS, ps, 0, nsave)
        torch.cuda.synchronize()
        ps_push_s = time.perf_counter() - t0
        del ens_p
        # phase-space D_mumu on the device: mu reconstructed (FP32, the reference's
        # default compute precision) into a device chunk and binned there, 64 log
        # lags x 50 |mu| bins; no host round trip
        lags_m = log_spaced_lag_steps(nsave - 1, 64)
        edges_m, _ = build_mu_edges_full(0.0, 1.0, 50)
        Bf = [f.float().contiguous() for f in fields[:3]]

        def ps_dmumu_pass(_k):
            acc = S.new_dmumu_accumulators(len(lags_m), 50, device=dev)
            S.process_phase_space_chunk_dmumu(ps[:, 0:3], ps[:, 3:6], *Bf, grid, lags_m, edges_m,
                                              acc["particle_counts"], acc["particle_means"], acc["particle_m2s"],
                                              acc["pair_sum_squares"], acc["pair_counts"], acc["dmumu_counts"],
                                              acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"])
            ps_dmumu_pass.acc = acc

        pms, _ = timed(ps_dmumu_pass, 2, 1, torch)
        ppairs = int(ps_dmumu_pass.acc["pair_counts"].sum().item())
        ps_dmumu = {"value": ws * ppairs / max_over_ranks(pms / 2, ws, dev) * 1e3, "unit": "lag-pairs/s",
                    "pairs_per_pass": ppairs, "ms_per_pass": pms / 2, "particles": npp, "saves": nsave,
                    "lags": int(len(lags_m)), "mu_bins": 50, "compute_precision": "f32",
                    "path": "pt_dmumu_accumulate_phase_space_device (reconstruct + bin on the device)",
                    "compulsory_bytes_per_pass": 24 * npp * nsave}
        mom = ps[:, 3:6, :].contiguous()
        del ps, Bf
        torch.cuda.empty_cache()
        lags_p = log_spaced_lag_steps(nsave - 1, 64)
        p0 = float(torch.linalg.vector_norm(mom[0, :, 0].double()).item())
        if ws > 1:
            from particle_transport_b200 import shard
            p0 = shard.broadcast_p0(p0, device=dev)  # the first particle's |p| at save 1 is rank 0's

        def dpp_pass(_k):
            acc = S.new_dpp_accumulators(len(lags_p), device=dev)
            S.process_momenta_chunk_dpp(mom, lags_p, p0, acc["counts"], acc["sum_delta_p"], acc["sum_delta_p2"],
                                        acc["sum_delta_p_norm"], acc["sum_delta_p_norm2"])
            dpp_pass.acc = acc

        dms, _ = timed(dpp_pass, 2, 1, torch)
        dpairs = int(dpp_pass.acc["counts"].sum().item())
        snaps = selected_energy_snapshot_indices(nsave, 16) - 1
        E0 = args.energy
        e_lo, e_hi = E0 / 2, E0 * 2

        def hist_pass(_k):
            hist_pass.counts = S.energy_histogram(mom, snaps, e_lo, e_hi, 256)

        hms, _ = timed(hist_pass, 3, 1, torch)
        dpp_s = dms / 2 / 1e3
        dpp = {"value": ws * dpairs / max_over_ranks(dpp_s * 1e3, ws, dev) * 1e3, "unit": "lag-pairs/s",
               "pairs_per_pass": dpairs, "ms_per_pass": dms / 2, "particles": npp, "saves": nsave,
               "lags": int(len(lags_p)), "estimator": "sliding, |p| recomputed per end in FP64",
               "compulsory_bytes_per_pass": 12 * npp * nsave,
               "hbm_frac_of_compulsory": (12 * npp * nsave / dpp_s / 1e9) / peaks["hbm_gbs"],
               "phase_space_push_s": ps_push_s, "phase_space_push_rate": npp * (NSTEPS - 1) / ps_push_s,
               "phase_space_dmumu": ps_dmumu,
               "energy_histograms": {"snapshots": int(len(snaps)), "bins": 256, "range_GeV": [e_lo, e_hi],
                                     "spacing": "log", "ms_per_pass": hms / 3,
                                     "counted": int(hist_pass.counts.sum().item()),
                                     "particles_x_snapshots": int(npp * len(snaps))}}
        dpp["roofline"] = issue_roofline("dpp_kernel", dpp["value"] / ws, clocks, dev)
        if ws > 1:
            merged = shard.reduce_dpp_accumulators(dpp_pass.acc)
            dpp["merged"] = {"counts": int(merged["counts"].sum()), "p0": p0, "ranks": ws}
        if "cpu" not in skip and rank == 0:
            dpp["cpu_baseline"] = cpu_dpp_rate(mom[:, :, :4096].cpu().numpy(), lags_p, p0, args.cpu_seconds / 2)
        del mom
        torch.cuda.empty_cache()

    # ---------------- e2e through pt_push_run with host buffers
    e2e = None
    if "e2e" not in skip:
        G = args.e2e_gyroperiods
        ns = 64 * G + 1
        host = {k: np.ascontiguousarray(v).copy() for k, v in state.items()}
        al = np.ones(n, np.uint8)
        pe = R.push_params(dt, ns, STRIDE, cache="mu", precision="f32", sort_every=args.sort_every,
                           kernel_variant=args.variant)
        rows = [0]

        def sink(i, row):
            rows[0] += 1

        def e2e_call(_k):
            R.run_push_host(fb, host, al, pe, sink)

        for _ in range(1):
            e2e_call(-1)
        dist_barrier(ws)
        t0 = time.perf_counter()
        ncall = max(1, min(3 if G <= 100 else 2, K // 3))
        for _ in range(ncall):
            e2e_call(0)
        el = time.perf_counter() - t0
        el = max_over_ranks(el * 1e3, ws, dev) / 1e3
        nsave_e = (ns - 1) // STRIDE + 1
        e2e = {"value": ws * n * (ns - 1) * ncall / el, "unit": UNIT,
               "step": "one pt_push_run call: host state in, mu rows and state out",
               "h2d_bytes_per_step": int(n * (6 * 8 + 1)),
               "d2h_bytes_per_step": int(n * (6 * 8 + 1) + nsave_e * n * 4 + 8 * ns),
               "call": f"pt_push_run over {G} T_g0 ({ns - 1} pushes, {nsave_e} mu rows) per call, host state",
               "calls": ncall, "s_per_call": el / ncall}

    # ---------------- batched campaigns and serving (their own field libraries)
    field_bytes = fb.device_bytes
    del fb
    torch.cuda.empty_cache()
    batched = leg("batched", run_batched, args, dev, rank) if "batch" not in skip else None
    serving = leg("serving", run_serving, args, dev) if ("serve" not in skip and ws == 1) else None
    config1 = leg("config1", run_config1, args, rank) if ("config1" not in skip and rank == 0) else None
    precision = leg("precision", run_precision_key, args, dev) if ("precision" not in skip and rank == 0) else None

    # ---------------- CPU baseline (oracle, host cores)
    cpu = None
    if "cpu" not in skip and rank == 0:
        fields_host = [f.cpu().numpy() for f in fields]
        cpu = cpu_push_rate(fields_host, grid, state, dt, args.cpu_seconds)
        del fields_host

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded GS turbulence and particles; no MHD snapshot ships)",
                "config": {"workload": f"{args.grid}^3 GS turbulence dB/B0=1, u_rms=1e-4 c, {n} protons/GPU at "
                                       f"{args.energy:g} GeV, 64 steps/T_g0, mu cache every 8; step = 64 pushes",
                           "field_storage": args.storage, "field_bytes": field_bytes,
                           "push": "FP32 push, FP64 positions and |p|^2", "sort_every_steps": args.sort_every,
                           "kernel_variant": args.variant,
                           "l2": "inputs larger than L2 (field and state exceed 126 MB); no flush",
                           "parallelism": f"particle-sharded replicas x{ws}"},
                "roofline": roofline, "fp32_bricks": fp32b, "fp64_push": fp64, "lag_pairs": lag, "dpp": dpp,
                "e2e": e2e,
                "cpu_baseline": cpu,
                "clocks": clocks, "gpu_launches": launches["push"] + launches["sort"], "batched": batched,
                "job_latency": ({"p50_s": serving["p50_s"], "p99_s": serving["p99_s"], "jobs": serving["jobs"]}
                                if serving and "p50_s" in serving else None),
                "serving": serving, "config1_end_to_end": config1, "precision": precision}
        print(json.dumps(line), flush=True)


# Warp instructions per lag pair of the statistics kernels: smsp__inst_executed.sum
# of one launch over the pairs it processed, from an ncu capture of the bench's
# small case (profiles/dmumu_*.md, profiles/dpp_*.md).  These kernels are
# bound by instruction issue, whose ceiling is one warp instruction per cycle
# per SM sub-partition (4 per SM).
WARP_INST_PER_PAIR = {"dmumu_kernel": 47.59e9 / 49.193e9, "dpp_kernel": 6.663e9 / 12.298e9}


def issue_roofline(kernel: str, pairs_per_s: float, clocks, device) -> dict:
    """Issue-bound roofline of a lag-statistics kernel: achieved warp
    instructions per second (pairs/s x warp instructions per pair) over the
    issue ceiling at the SM clock of the timed region."""
    import torch

    w = WARP_INST_PER_PAIR.get(kernel)
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    peak = sms * 4 * mhz * 1e6
    if w is None:
        return {"kernel": kernel, "bound": "issue", "warp_inst_per_pair": None, "peak": peak / 1e9,
                "unit": "G warp-inst/s"}
    ach = pairs_per_s * w
    return {"kernel": kernel, "bound": "issue", "warp_inst_per_pair": w, "achieved": ach / 1e9, "peak": peak / 1e9,
            "unit": "G warp-inst/s", "frac": ach / peak, "sm_mhz": mhz,
            "note": "warp instructions per pair from an ncu capture of the same kernel; peak = SMs x 4 x clock"}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one 64-step
# push_fast_kernel launch of this workload, from a 1-pass ncu capture of the
# same command; keyed by (storage, grid, particles)
TRAFFIC = {("brick_bf16", 512, 16_777_216): 6.63e9 + 1.44e9}


def run_config1(args, rank):
    """The reference's CPU-runnable configuration end to end, through the host
    API the Julia seams call: 64^3 (dB/B0 = 0.5, |k| = 2..32, E = 0), 4096
    protons at 1 GeV, 64 steps/T_g0 for 50 T_g0 (3200 pushes), mu cache every
    4 steps (801 saves) handed to the host row by row, then D_mumu on 20 log
    lags x 20 |mu| bins of the host mu cache.  The GPU path (pt_push_run FP64
    and FP32/BF16, pt_dmumu_accumulate) against the oracle on all host cores
    (the same FP64 push and binning, the reference's arithmetic)."""
    from oracle import build as ob
    from oracle import oracle as o
    from particle_transport_b200 import fields as F
    from particle_transport_b200 import runner as R
    from particle_transport_b200 import stats as S
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import energy_to_gamma, init_particles
    from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0

    ob.build()
    n, np_, spg, dur, stride = 64, 4096, 64, 50, 4
    fields = [np.ascontiguousarray(f.numpy()) for f in F.to_si(F.synthetic_mhd_fields(n, 2, 32, 0.5, 1.0, 0.0, seed=1))]
    rg = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((n - 1) * rg, n, n, n)
    B0 = F.reference_B0_T(*fields[:3])
    dt = (2 * math.pi / spg) / reference_Omega0(B0, energy_to_gamma(1.0), F.Q_E, F.M_P)
    state = init_particles(np_, grid, 1.0, seed=1)
    nsteps = spg * dur + 1
    nsave = R.n_saves(nsteps, stride)
    lags = log_spaced_lag_steps(nsave - 1, 20)
    edges, _ = build_mu_edges_full(0.0, 1.0, 20)

    def gpu(storage, precision):
        fl = FieldLibrary(fields, grid, storage, B_ref_T=B0)
        best = None
        for _ in range(3):  # the first call also sets up the context buffers
            st = {k: v.copy() for k, v in state.items()}
            t0 = time.perf_counter()
            col = R.CacheCollector(np_, nsave, "mu")
            R.run_push_host(fl, st, np.ones(np_, np.uint8),
                            R.push_params(dt, nsteps, stride, cache="mu", precision=precision,
                                          sort_every=64 if precision == "f32" else 0), col)
            acc = S.new_dmumu_accumulators(len(lags), 20)
            S.process_mu_chunk_dmumu(col.mu, lags, edges, acc["particle_counts"], acc["particle_means"],
                                     acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                                     acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                                     layout="particle_fastest")
            el = time.perf_counter() - t0
            best = el if best is None else min(best, el)
        fl.close()
        return best

    out = {"workload": "64^3, 4096 protons at 1 GeV, 3200 pushes, 801 mu saves, D_mumu 20 lags x 20 bins; "
                       "host state and host mu cache (pt_push_run + pt_dmumu_accumulate)",
           "gpu_f64_s": gpu("ref_f64", "f64"), "gpu_f32_bf16_s": gpu("brick_bf16", "f32")}
    nt = host_threads()
    st = {k: v.copy() for k, v in state.items()}
    t0 = time.perf_counter()
    mu, _ = o.push_run([np.asfortranarray(f.T) for f in fields], grid, st, np.ones(np_, np.uint8), dt, nsteps,
                       stride, cache_mode=1, nthreads=nt)
    acc = {"counts": np.zeros((len(lags), 20), np.int64), "sum_d": np.zeros((len(lags), 20)),
           "sum_d2": np.zeros((len(lags), 20)), "w_count": np.zeros(len(lags), np.int64),
           "w_mean": np.zeros(len(lags)), "w_m2": np.zeros(len(lags)), "pair_ss": np.zeros(len(lags)),
           "pair_n": np.zeros(len(lags), np.int64)}
    o.dmumu_accumulate(mu, lags, edges, acc, time_fastest=False, nthreads=nt)
    out["cpu_oracle_s"] = time.perf_counter() - t0
    out["cpu_cores"] = nt
    out["speedup_f64"] = out["cpu_oracle_s"] / out["gpu_f64_s"]
    out["speedup_f32_bf16"] = out["cpu_oracle_s"] / out["gpu_f32_bf16_s"]
    return out


def run_batched(args, dev, rank):
    """Batched campaigns: 12 campaigns (4 modes x 1/10/100 GeV) on a resident
    256^3 FP32 field library, N log-uniform in [65536, 4194304], 20-500 T_g0
    at 64 steps per T_g0 of each energy, one persistent launch per epoch
    (CUDA graph); steps per epoch, blocks per SM and each campaign's re-sort
    cadence (by particle speed) picked by the tuner; then D_mumu per
    campaign (32 log lags x 20 |mu| bins) from its full mu cache (a save
    every 32 steps)."""
    import torch

    from particle_transport_b200 import fields as F
    from particle_transport_b200 import stats as S
    from particle_transport_b200.batch import Batch, tune_batch
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import energy_to_gamma, init_particles
    from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0

    n = 256
    rg = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((n - 1) * rg, n, n, n)
    libs, B0 = {}, None
    for m in ("total", "alfven", "fast", "slow"):
        f = F.to_si(F.synthetic_mhd_fields(n, 2, n // 2, 0.5, 1.0, 1e-4, seed=77, spectrum="isotropic", modes=m,
                                           device=dev))
        if m == "total":
            B0 = F.reference_B0_T(*f[:3])
        libs[m] = FieldLibrary(f, grid, "brick_f32", B_ref_T=B0)
        del f
    torch.cuda.empty_cache()
    rng = np.random.default_rng(4 + rank)
    camps = []
    for m in libs:
        for E in (1.0, 10.0, 100.0):
            N = int(np.exp(rng.uniform(np.log(65536), np.log(4194304))))
            dur = float(rng.uniform(20, 500))
            g0 = energy_to_gamma(E)
            dt = (2 * math.pi / 64) / reference_Omega0(B0, g0, F.Q_E, F.M_P)
            camps.append(dict(field=libs[m], state=init_particles(N, grid, E, seed=len(camps) + 100 * rank), dt=dt,
                              nsteps=int(round(64 * dur)) + 1, stride=32, mode=m, E=E))
    ntot = sum(len(c["state"]["x1"]) for c in camps)
    t0 = time.perf_counter()
    tune = tune_batch(camps, "brick_f32", ntot, use_cache=False)
    tune_s = time.perf_counter() - t0
    K, bps, thr = tune["K"], tune["blocks_per_sm"], tune["threads_per_block"]
    b = Batch(ntot, max_campaigns=len(camps), storage="brick_f32", steps_per_epoch=K, blocks_per_sm=bps,
              threads_per_block=thr)
    caches = []
    for c, se in zip(camps, tune["sort_every"]):
        nsave = (c["nsteps"] - 1) // c["stride"] + 1
        c["nsave"] = nsave
        # time-fastest caches [n][pitch]: a particle's saves side by side reach DRAM as whole sectors
        caches.append(torch.empty((len(c["state"]["x1"]), (nsave + 7) // 8 * 8), dtype=torch.float32, device=dev))
        c["id"] = b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=caches[-1], sort_every=se,
                        time_fastest=True)
        c["sort_every"] = se
    epochs = max(math.ceil(c["nsteps"] / K) for c in camps)
    b.run(1)  # graph capture + first epoch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run(epochs - 1)
    e1.record()
    torch.cuda.synchronize()
    push_s = e0.elapsed_time(e1) / 1e3
    steps_timed = sum(len(c["state"]["x1"]) * max(0, c["nsteps"] - 1 - K) for c in camps)
    assert all(b.done(c["id"]) for c in camps)
    b.close()
    pairs = 0
    e0.record()
    for c, cache in zip(camps, caches):
        nsave = c["nsave"]
        lags = log_spaced_lag_steps(nsave - 1, 32)
        edges, _ = build_mu_edges_full(0.0, 1.0, 20)
        acc = S.new_dmumu_accumulators(len(lags), 20, device=dev)
        S.process_mu_chunk_dmumu(cache, lags, edges, acc["particle_counts"], acc["particle_means"],
                                 acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"], acc["dmumu_counts"],
                                 acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"], layout="time_fastest", nsave=nsave)
        c["pairs"] = acc["pair_counts"]
    e1.record()
    torch.cuda.synchronize()
    lag_s = e0.elapsed_time(e1) / 1e3
    pairs = int(sum(int(c["pairs"].sum().item()) for c in camps))
    return {"campaigns": len(camps), "particles": ntot, "epochs": epochs, "steps_per_epoch": K,
            "blocks_per_sm": bps, "threads_per_block": thr, "particles_per_thread": 256 // thr,
            "autotune": {"cadence_steps_by_speed_class": {str(k): v for k, v in tune["cadence_steps"].items()},
                         "trials": {k: round(v, 1) for k, v in tune["timings"].items()}, "seconds": tune_s},
            "value": steps_timed / push_s, "unit": UNIT, "push_s": push_s,
            "lag_pairs_per_s": pairs / lag_s, "lag_s": lag_s, "field": "256^3 FP32 bricks x 4 modes",
            "per_campaign": [{"mode": c["mode"], "E_GeV": c["E"], "n": len(c["state"]["x1"]),
                              "T_g0": (c["nsteps"] - 1) / 64, "sort_every_epochs": c["sort_every"]} for c in camps]}


def run_precision_key(args, dev):
    """The precision forms against the FP64 push, reduced from the
    plain-vs-precision configuration: 128^3 (dB/B0 = 0.5 on |k| = 2..64,
    u_rms = 1e-4 c), the total field and its alfven / fast / slow projections,
    protons at 1, 10 and 100 GeV with fixed mu0 = 0.525, 128 steps per T_g0 for
    50 T_g0, mu every 8 steps (801 saves), 32 log lags x 20 |mu| bins, D_pp
    over 131,072 particles.  For each form (FP32 push over FP32 bricks and
    over BF16 bricks) and the FP64 floors (positions moved by one FP64 ulp,
    by one FP32 ulp of the box, and an independent sample): the largest
    relative error of D_mumu(mu, tau) (cells with >= 100 pairs), <dmu^2>(tau)
    and D_pp(tau) over every variant and energy, over all cells and over the
    cells the particle count resolves to 1 % (FP64 standard error by batch
    means), the largest error in FP64 standard errors, and the energy drift
    with E = 0."""
    import torch

    from particle_transport_b200 import fields as F
    from particle_transport_b200 import precision as P

    n, npart = 128, args.precision_key_particles
    grid = F.build_uniform_grid((n - 1) * F.gyroradius_m(1.0, 1e-10), n, n, n)
    t0 = time.perf_counter()
    forms = ("f64_1ulp", "f64_f32ulp", "f64_resample", "f32", "bf16")
    prods = P.PRODUCTS
    worst = {f: {k: 0.0 for k in prods} for f in forms}
    worst_resolved = {f: {k: 0.0 for k in prods} for f in ("f32", "bf16")}
    failures = {}
    drift = {"f64": 0.0, "f32": 0.0, "bf16": 0.0}
    cases = {}
    ok = True
    for mode in ("total", "alfven", "fast", "slow"):
        fs = F.to_si(F.synthetic_mhd_fields(n, 2, n // 2, 0.5, 1.0, 1e-4, seed=5, modes=mode, device=dev))
        libs, B0 = P.build_libraries(fs, grid)
        del fs
        for E in (1.0, 10.0, 100.0):
            r = P.compare_forms(libs, B0, grid, E, npart, gyroperiods=50)
            case = f"{mode}/{E:g}GeV"
            cases[case] = {f: {k: r[f][k]["max"] for k in prods} for f in forms}
            cases[case]["resolved"] = {f: {k: r[f][k].get("max_resolved") for k in prods} for f in ("f32", "bf16")}
            cases[case]["max_z"] = {f: {k: r[f][k].get("max_z") for k in prods} for f in forms}
            bad = P.check_forms(r, ("f32", "bf16"))
            if bad:
                failures[case] = [list(map(str, b)) for b in bad]
            ok &= not bad
            for f in forms:
                for k in worst[f]:
                    worst[f][k] = max(worst[f][k], r[f][k]["max"])
            for f in worst_resolved:
                for k in prods:
                    worst_resolved[f][k] = max(worst_resolved[f][k], r[f][k].get("max_resolved", 0.0))
            for f in drift:
                drift[f] = max(drift[f], r[f]["gamma_drift_E0"])
        for lib in libs.values():
            lib.close()
        torch.cuda.empty_cache()
    return {"max_rel_err": worst, "max_rel_err_resolved": worst_resolved, "tolerance": 0.01,
            "within_tolerance": ok, "failures": failures,
            "criterion": "per cell against the FP64 push: within 1 %, or within 5 standard errors of the difference "
                         "of two runs where the FP64 statistic is not resolved to 1 % (standard errors by batch means "
                         "over 16 particle batches); the three FP64 floor runs pass the same test",
            "gamma_drift_E0_max": drift, "per_case": cases, "seconds": time.perf_counter() - t0,
            "setup": f"128^3, dB/B0=0.5, k=2..64, u_rms=1e-4 c; total/alfven/fast/slow x 1/10/100 GeV; {npart} "
                     "protons, fixed mu0=0.525, 128 steps/T_g0, 50 T_g0, mu every 8 steps; 32 lags x 20 |mu| bins "
                     "(cells >= 100 pairs); D_pp over 131072 particles from a Float64 phase-space cache; errors relative "
                     "to the FP64 push"}


def run_precision(args, dev):
    """Plain vs precision forms at 256^3 (total field, dB/B0 = 0.5, k = 2..128,
    u_rms = 1e-4 c): 1,048,576 protons per energy at 1, 10 and 100 GeV,
    fixed mu0 = 0.5 with random gyrophase, 128 steps per T_g0 for 200 T_g0
    (25,600 pushes), mu cache every 8 steps (3201 saves).  Each energy is
    pushed in FP64 over the reference layout and as the FP32 push over FP32
    and BF16 bricks; each product's error against the FP64 form is reported:
    trajectory deviation (first 65,536 particles, phase-space cache, in
    gyroradii, at 1 and 10 T_g0), |dgamma|/gamma at the end, mu at 10 T_g0,
    D_mumu(mu, tau) and <dmu^2>(tau) (32 log lags x 20 |mu| bins, cells with
    >= 100 pairs) and D_pp(tau) (same lags, all particles).  An FP64 run from
    positions moved by one ulp gives the floor set by chaotic divergence: the
    statistics of two FP64 runs differ by that much already.  Each product is
    also judged cell by cell against the FP64 statistic's own standard error
    (batch means over 16 particle batches; precision.rel_err).  mu0 = 0.5 is
    an edge of the 20 |mu| bins, so the cells a form's first saves fill can
    differ from the FP64 ones (the test of the forms injects at 0.525)."""
    import torch

    from particle_transport_b200 import fields as F
    from particle_transport_b200 import precision as P
    from particle_transport_b200 import runner as R
    from particle_transport_b200 import stats as S
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import energy_to_gamma, init_particles
    from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0

    n = args.precision_grid
    npart = args.precision_particles
    nsub = min(65536, npart)
    ps_chunk = 262144
    spg, dur, stride = 128, args.precision_gyroperiods, 8
    nsteps = spg * dur + 1
    nsave = (nsteps - 1) // stride + 1
    rg1 = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((n - 1) * rg1, n, n, n)
    L = grid.xmax - grid.xmin
    fields = F.to_si(F.synthetic_mhd_fields(n, 2, n // 2, 0.5, 1.0, 1e-4, seed=5, spectrum="isotropic", device=dev))
    B0 = F.reference_B0_T(*fields[:3])
    hostB = [f.cpu().numpy() for f in fields[:3]]
    libs = {"f64": FieldLibrary(fields, grid, "ref_f64"), "f32": FieldLibrary(fields, grid, "brick_f32", B_ref_T=B0),
            "bf16": FieldLibrary(fields, grid, "brick_bf16x", B_ref_T=B0)}
    del fields
    lags = log_spaced_lag_steps(nsave - 1, 32)
    edges, _ = build_mu_edges_full(0.0, 1.0, 20)
    tau = np.array([l * stride * 2 * math.pi / spg for l in lags])
    out = {"grid": n, "field": "total, dB/B0=0.5, k=2..128, u_rms=1e-4 c", "particles_per_energy": npart,
           "trajectory_subset": nsub, "steps_per_gyroperiod": spg, "gyroperiods": dur, "save_stride": stride,
           "saves": nsave, "lags": int(len(lags)), "mu_bins": 20, "min_count_per_cell": 100,
           "bf16_storage": "brick_bf16x", "energies": {}}

    def run(form, st, dt, cache_mode, c0, c1):
        count = c1 - c0
        sub = {k: np.ascontiguousarray(v[c0:c1]) for k, v in st.items()}
        shape = (nsave, count) if cache_mode == "mu" else (nsave, 6, count)
        cache = torch.empty(shape, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if form.startswith("f64"):
            ens = R.DeviceEnsemble(libs["f64"], sub, np.ones(count, np.uint8))
            ens.advance(R.push_params(dt, nsteps, stride, cache=cache_mode, precision="f64", steps_per_launch=64),
                        0, nsteps, cache, 0, nsave)
            torch.cuda.synchronize()
            final = {k: v.cpu().numpy() for k, v in ens.state.items()}
        else:
            ens = R.FastEnsemble(libs[form], sub, np.ones(count, np.uint8))
            ens.advance(R.push_params(dt, nsteps, stride, cache=cache_mode, precision="f32", sort_every=64,
                                      kernel_variant=1), 0, nsteps, cache, 0, nsave)
            st_out, _ = ens.export()
            torch.cuda.synchronize()
            final = {k: v.cpu().numpy() for k, v in st_out.items()}
            ens.close()
        return cache, final, time.perf_counter() - t0

    batches = 16  # independent particle batches for the FP64 statistics' standard errors
    sub = npart // batches

    def dmumu_acc(mu):
        acc = S.new_dmumu_accumulators(len(lags), 20, device=dev)
        S.process_mu_chunk_dmumu(mu, lags, edges, acc["particle_counts"], acc["particle_means"],
                                 acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                                 acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                                 layout="particle_fastest")
        return {k: v.cpu().numpy() for k, v in acc.items()}

    def dmumu(mu, with_se=False):
        a = dmumu_acc(mu)
        d = S.compute_dmumu_arrays_full(a["dmumu_counts"], a["dmumu_sum_delta"], a["dmumu_sum_delta2"], tau, tau, 100)
        se = None
        if with_se:
            parts = [dmumu_acc(mu[:, g * sub:(g + 1) * sub].contiguous()) for g in range(batches)]
            n_p = a["particle_counts"].astype(np.float64)
            with np.errstate(divide="ignore", invalid="ignore"):
                se_pm = np.sqrt(a["particle_m2s"] / (n_p - 1.0) / n_p) / np.abs(a["particle_means"])
            se = {"D": P.ratio_se([q["dmumu_sum_delta2"] for q in parts], [q["dmumu_counts"] for q in parts]),
                  "pm": se_pm}
        return d["dmumu_raw_norm"], a["particle_means"], a["dmumu_counts"], se

    def dpp_add(acc, mom, p0):
        S.process_momenta_chunk_dpp(mom, lags, p0, acc["counts"], acc["sum_delta_p"], acc["sum_delta_p2"],
                                    acc["sum_delta_p_norm"], acc["sum_delta_p_norm2"])

    def phase_space(form, st, dt, p0, with_se=False):
        """D_pp over all particles from phase-space caches of ps_chunk
        particles (add-into accumulators, p0 fixed across chunks), plus the
        positions of the first nsub particles at 1 and 10 T_g0; with_se, the
        relative standard error of each lag from the particle batches."""
        acc = S.new_dpp_accumulators(len(lags), device=dev)
        parts = []
        rows = {}
        for c0 in range(0, npart, ps_chunk):
            ps, _, _ = run(form, st, dt, "phase_space", c0, min(npart, c0 + ps_chunk))
            if p0 is None:
                p0 = float(torch.linalg.vector_norm(ps[0, 3:6, 0].double()).item())
            if c0 == 0:
                for t in (1, 10):
                    rows[t] = ps[t * spg // stride, 0:3, :nsub].double().cpu().numpy()
            mom = ps[:, 3:6, :].contiguous()
            del ps
            dpp_add(acc, mom, p0)
            if with_se:
                for b0 in range(0, mom.shape[2], sub):
                    q = S.new_dpp_accumulators(len(lags), device=dev)
                    dpp_add(q, mom[:, :, b0:b0 + sub].contiguous(), p0)
                    parts.append({k: v.cpu().numpy() for k, v in q.items()})
            del mom
        a = {k: v.cpu().numpy() for k, v in acc.items()}
        d = S.compute_dpp_arrays(a["counts"], a["sum_delta_p"], a["sum_delta_p2"], a["sum_delta_p_norm"],
                                 a["sum_delta_p_norm2"], tau, tau)
        se = P.ratio_se([q["sum_delta_p_norm2"] for q in parts], [q["counts"] for q in parts]) if with_se else None
        return d["dpp_raw_norm"], rows, p0, se

    def rel(a, b, w=None):
        m = np.isfinite(a) & np.isfinite(b) & (np.abs(b) > 0)
        r = np.abs(a[m] - b[m]) / np.abs(b[m])
        res = {"median": float(np.median(r)), "max": float(r.max()), "cells": int(m.sum())}
        if w is not None:
            res["count_weighted_mean"] = float(np.sum(r * w[m]) / np.sum(w[m]))
        return res

    def traj_dev(xa, xb, rg):
        d = xa - xb
        d -= L * np.round(d / L)  # minimum image across the periodic box
        r = np.sqrt((d * d).sum(axis=0)) / rg
        return {"median_rg": float(np.median(r)), "p99_rg": float(np.percentile(r, 99)), "max_rg": float(r.max())}

    for E in (1.0, 10.0, 100.0):
        g0 = energy_to_gamma(E)
        rgE = F.gyroradius_m(E, B0)
        dt = (2 * math.pi / spg) / reference_Omega0(B0, g0, F.Q_E, F.M_P)
        st = init_particles(npart, grid, E, seed=int(E) + 7, injection_mode="fixed_mu", mu0=0.5, B=hostB)
        # noise floor: the FP64 push from positions moved by one ulp
        st_pert = dict(st, x1=np.nextafter(st["x1"], np.inf))
        res = {}
        p0 = None
        for form in ("f64", "f64_1ulp", "f32", "bf16"):
            mu, final, secs = run(form, st_pert if form == "f64_1ulp" else st, dt, "mu", 0, npart)
            D, pmean, counts, se = dmumu(mu, with_se=form == "f64")
            mu10 = mu[10 * spg // stride].cpu().numpy()
            del mu
            torch.cuda.empty_cache()
            Dpp, rows, p0, se_pp = phase_space(form, st_pert if form == "f64_1ulp" else st, dt, p0,
                                               with_se=form == "f64")
            if se is not None:
                se["Dpp"] = se_pp
            p = np.stack([final[k] for k in ("p1", "p2", "p3")])
            gam = np.sqrt(1 + (np.linalg.norm(p, axis=0) / (F.M_P * F.C_LIGHT)) ** 2)
            res[form] = dict(D=D, pm=pmean, counts=counts, Dpp=Dpp, rows=rows, gam=gam, mu10=mu10,
                             rate=npart * (nsteps - 1) / secs, secs=secs, se=se)
            torch.cuda.empty_cache()
        ref = res["f64"]
        e = {"f64_particle_steps_per_s": ref["rate"], "f64_s": ref["secs"],
             "gamma_drift_f64_end": float(np.median(np.abs(ref["gam"] / g0 - 1)))}
        for form in ("f64_1ulp", "f32", "bf16"):
            r = res[form]
            dmu = np.abs(r["mu10"] - ref["mu10"])
            dmu = dmu[np.isfinite(dmu)]
            e[form] = {"particle_steps_per_s": r["rate"], "s": r["secs"], "speedup_vs_f64": r["rate"] / ref["rate"],
                       "trajectory_1_Tg0": traj_dev(r["rows"][1], ref["rows"][1], rgE),
                       "trajectory_10_Tg0": traj_dev(r["rows"][10], ref["rows"][10], rgE),
                       "mu_abs_err_10_Tg0": {"median": float(np.median(dmu)), "p99": float(np.percentile(dmu, 99))},
                       "gamma_rel_err_end": {"median": float(np.median(np.abs(r["gam"] / ref["gam"] - 1))),
                                             "max": float(np.max(np.abs(r["gam"] / ref["gam"] - 1)))},
                       "D_mumu_raw_norm_rel_err": rel(r["D"], ref["D"], ref["counts"].astype(np.float64)),
                       "delta_mu2_particle_mean_rel_err": rel(r["pm"], ref["pm"]),
                       "D_pp_raw_norm_rel_err": rel(r["Dpp"], ref["Dpp"]),
                       # the per-cell test of the precision forms against the FP64 sampling error
                       "against_sampling_error": {
                           "D_mumu": P.rel_err(r["D"], ref["D"], ref["se"]["D"], ref["counts"] >= 100),
                           "delta_mu2": P.rel_err(r["pm"], ref["pm"], ref["se"]["pm"]),
                           "D_pp": P.rel_err(r["Dpp"], ref["Dpp"], ref["se"]["Dpp"])}}
        out["energies"][f"{E:g}"] = e
        print(json.dumps({"precision_energy_GeV": E, **e}), flush=True)
        torch.cuda.empty_cache()
    return out


def run_serving(args, dev, rate=4.0):
    """Serving (config 5).  A Poisson stream (mean 4 jobs/s) of args.serve_jobs
    jobs drawn from the full job distribution -- 16K-8M particles, 10-300
    T_g0, 1-300 GeV, either library, any mode, isotropic or fixed-mu -- against
    resident 256^3 and 512^3 BF16-brick libraries (4 modes each), admitted
    against a 150 GB HBM budget and continuously batched: p50 / p99 job
    latency over every job and the particle-step rate over the wall clock and
    while the device is busy.
    Matched workload: the same campaigns in one Batch, all admitted at once,
    with the server's steps per epoch and sort cadences and a ring mu cache;
    its rate against the server's busy rate separates the engine's overhead
    from the workload mix.
    FP32 against FP64: the first args.serve_cmp jobs of the same stream (same
    arrivals and specs) served with the FP32 push and with the FP64 push over
    FP64 bricks (results bit-identical to the reference-layout FP64 push,
    whose rate is the fp64 leg of the headline)."""
    import torch

    from particle_transport_b200 import fields as F
    from particle_transport_b200.batch import Batch
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import init_particles_device
    from particle_transport_b200.server import CampaignServer, job_campaign, sample_jobs

    B0 = {}

    def make_libs(storage):
        """The 2 x 4 seeded field libraries in one storage (same fields for every storage)."""
        out = {}
        for n in (256, 512):
            rg = F.gyroradius_m(1.0, 1e-10)
            grid = F.build_uniform_grid((n - 1) * rg, n, n, n)
            out[str(n)] = {}
            for m in ("total", "alfven", "fast", "slow"):
                f = F.to_si(F.synthetic_mhd_fields(n, 2, n // 2, 0.5 if n == 256 else 1.0, 1.0, 1e-4, seed=91 + n,
                                                   spectrum="isotropic" if n == 256 else "gs", modes=m, device=dev))
                if m == "total":
                    B0[str(n)] = F.reference_B0_T(*f[:3])
                out[str(n)][m] = FieldLibrary(f, grid, storage, B_ref_T=B0[str(n)])
                del f
            torch.cuda.empty_cache()
        return out

    libs = make_libs("brick_bf16")

    def serve(libraries, arrivals, specs, push, schedule="srpt", fill=args.serve_fill):
        srv = CampaignServer(libraries, B0, hbm_budget_bytes=150e9, capacity=1 << 27, max_jobs=len(specs), push=push,
                             schedule=schedule, fill_particles=fill)
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        nxt = 0
        while nxt < len(specs) or not srv.idle():
            now = time.perf_counter() - t_start
            while nxt < len(specs) and arrivals[nxt] <= now:
                srv.submit(specs[nxt], arrival=t_start + arrivals[nxt])
                nxt += 1
            srv.tick()
        wall = time.perf_counter() - t_start
        lat = np.array([r.latency for r in srv.results])
        steps = sum(r.particle_steps for r in srv.results)
        busy = srv.device_busy_s()
        out = {"jobs": len(srv.results), "p50_s": float(np.percentile(lat, 50)),
               "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "max_s": float(lat.max()),
               "wall_s": wall, "particle_steps": int(steps), "aggregate_rate": steps / wall, "device_busy_s": busy,
               "busy_rate": steps / busy, "admit_host_s": srv.admit_s, "admission": dict(srv.admit_stats),
               "epochs": srv.epochs}
        srv.close()
        torch.cuda.empty_cache()
        return out

    def matched(libraries, specs, K=64):
        """The jobs' campaigns in one Batch, every one running from the first epoch."""
        ntot = sum(sp.n_particles for sp in specs)
        b = Batch(ntot, max_campaigns=len(specs), storage="brick_bf16", steps_per_epoch=K)
        rings, steps, epochs = [], 0, 0
        for sp in specs:
            fl, dt, nsteps, stride, every = job_campaign(sp, libraries, B0, K)
            st = init_particles_device(fl, sp.n_particles, sp.energy_GeV, seed=sp.seed, injection_mode=sp.injection,
                                       mu0=sp.mu0)
            rings.append(torch.empty((sp.n_particles, 8), dtype=torch.float32, device=dev))
            b.add(fl, st, dt, nsteps, stride, cache=rings[-1], ring=True, sort_every=every, time_fastest=True)
            steps += sp.n_particles * (nsteps - 1)
            epochs = max(epochs, math.ceil(nsteps / K))
            del st
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run(epochs)
        e1.record()
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
        b.close()
        del rings
        torch.cuda.empty_cache()
        return {"jobs": len(specs), "particles": ntot, "particle_steps": int(steps), "epochs": epochs,
                "seconds": secs, "rate": steps / secs, "cache": "ring of 8 saves per particle (time-fastest)"}

    arrivals, specs = sample_jobs(args.serve_jobs, rate, ["256", "512"], seed=2026)
    main = serve(libs, arrivals, specs, "f32")
    main.update({"rate_per_s": rate, "unit": UNIT, "push": "FP32 / BF16 bricks",
                 "stream": f"{args.serve_jobs} jobs, Poisson {rate}/s, 16K-8M particles, 10-300 T_g0, 1-300 GeV, "
                           "256^3 and 512^3 libraries x 4 modes, isotropic or fixed-mu",
                 "init": "on the device (pt_particles_init_device)", "hbm_budget_GB": 150,
                 "schedule": f"srpt: least work left first, epochs filled to {args.serve_fill} particles"})
    if args.serve_fill_sweep:
        main["fill_sweep"] = {}
        for fill in (int(v) for v in args.serve_fill_sweep.split(",") if v):
            r = serve(libs, arrivals, specs, "f32", fill=fill)
            main["fill_sweep"][str(fill)] = {k: r[k] for k in ("p50_s", "p99_s", "mean_s", "wall_s", "busy_rate",
                                                               "aggregate_rate", "epochs")}
    if args.serve_all:
        every = serve(libs, arrivals, specs, "f32", schedule="all")
        main["schedule_all"] = {k: every[k] for k in ("p50_s", "p99_s", "mean_s", "wall_s", "busy_rate", "epochs")}
    mt = matched(libs, specs)
    main["matched_batch"] = dict(mt, server_busy_rate_over_batch_rate=main["busy_rate"] / mt["rate"])
    k = min(args.serve_cmp, len(specs))
    cmp32 = serve(libs, arrivals[:k], specs[:k], "f32")
    del libs
    torch.cuda.empty_cache()
    libs64b = make_libs("brick_f64")  # the same fields as FP64 bricks (38 GB)
    cmp64b = serve(libs64b, arrivals[:k], specs[:k], "f64")
    del libs64b
    torch.cuda.empty_cache()
    main["fp32_vs_fp64"] = {"stream": f"the first {k} jobs of the same stream (same arrivals and specs)",
                            "fp32_bf16": cmp32,
                            "fp64_bricks": dict(cmp64b, note="the FP64 push over FP64 bricks with brick-sorted "
                                                              "slots: results bit-identical to the reference-layout "
                                                              "FP64 push"),
                            "busy_rate_ratio": cmp32["busy_rate"] / cmp64b["busy_rate"],
                            "p50_ratio": cmp64b["p50_s"] / cmp32["p50_s"]}
    return main


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, dev):
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    args = parse()
    if args.impl == "reference":
        # CPU-only arm: rank 0 alone runs and prints; other ranks exit without work
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, ws, 0)
        return
    if args.precision:
        import torch
        out = run_precision(args, torch.device("cuda", 0))
        print(json.dumps({"precision_study": out}), flush=True)
        return
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
