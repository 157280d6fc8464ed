"""Particle sharding across ranks and the end-of-job accumulator merge.

Particles never interact and the field is read-only, so a campaign shards
by contiguous particle ranges with the field replicated on every GPU; the
push and the lag statistics need no communication.  The one exchange is
the final merge of the statistics accumulators (tens of kB), plus the D_pp
normalisation p0, which belongs to the first particle and so to rank 0 and
is broadcast before the binning.  For the merge every rank all-gathers the
others' arrays and merges them in rank order -- integer
counts and FP64 sums added rank by rank, per-lag Welford triples combined
with the reference's combine_welford_stats! formula
(src/compute_delta_mu2_dmumu_full.jl:439-455) -- so every rank holds the
same, order-deterministic result.  Works over NCCL (CUDA tensors) and gloo
(CPU tensors).
"""
from __future__ import annotations

import numpy as np

DMUMU_SUM_KEYS = ("dmumu_counts", "dmumu_sum_delta", "dmumu_sum_delta2", "pair_sum_squares", "pair_counts")
DMUMU_WELFORD = ("particle_counts", "particle_means", "particle_m2s")
DPP_KEYS = ("counts", "sum_delta_p", "sum_delta_p2", "sum_delta_p_norm", "sum_delta_p_norm2")


def shard_range(n: int, rank: int, world: int):
    """Contiguous [start, stop) particle range of ``rank`` (sizes differ by at most one)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def combine_welford(gc, gm, gm2, lc, lm, lm2):
    """combine_welford_stats! on arrays (one entry per lag)."""
    gc, gm, gm2 = np.array(gc, np.int64), np.array(gm, np.float64), np.array(gm2, np.float64)
    for i in range(len(gc)):
        c = int(lc[i])
        if c <= 0:
            continue
        g = int(gc[i])
        if g == 0:
            gc[i], gm[i], gm2[i] = c, lm[i], lm2[i]
            continue
        cc = g + c
        d = float(lm[i]) - float(gm[i])
        gm[i] += d * c / cc
        gm2[i] += float(lm2[i]) + d * d * g * c / cc
        gc[i] = cc
    return gc, gm, gm2


def _gather(t, group=None):
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t.contiguous(), group=group)
    return [o.cpu().numpy() for o in out]


def reduce_dmumu_accumulators(acc: dict, group=None) -> dict:
    """Merge per-rank D_mumu / <dmu^2> accumulators (dict of numpy arrays or
    tensors, the keys of stats.new_dmumu_accumulators) into the job totals."""
    import torch

    dev = None
    for v in acc.values():
        if isinstance(v, torch.Tensor):
            dev = v.device
            break
    as_t = (lambda a: a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a), device=dev or "cpu"))
    gathered = {k: _gather(as_t(acc[k]), group) for k in DMUMU_SUM_KEYS + DMUMU_WELFORD}
    world = len(gathered["dmumu_counts"])
    out = {k: gathered[k][0].copy() for k in DMUMU_SUM_KEYS}
    for r in range(1, world):
        for k in DMUMU_SUM_KEYS:
            out[k] = out[k] + gathered[k][r]
    gc, gm, gm2 = (gathered[k][0].copy() for k in DMUMU_WELFORD)
    for r in range(1, world):
        gc, gm, gm2 = combine_welford(gc, gm, gm2, *(gathered[k][r] for k in DMUMU_WELFORD))
    out.update(particle_counts=gc, particle_means=gm, particle_m2s=gm2)
    return out


def broadcast_p0(p0: float, device="cpu", group=None) -> float:
    """The D_pp normalisation p0 = |p| of the first selected particle at the
    first save (src/compute_dpp_full.jl:483).  With contiguous particle
    ranges that particle is on rank 0; every rank takes rank 0's value, so
    the per-rank sums of dp/p0 add up to the single-pass sums.  ``device``
    is where the one-element tensor lives (a CUDA device under NCCL)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(p0)], dtype=torch.float64, device=device)
    dist.broadcast(t, src=0, group=group)
    return float(t.item())


def reduce_dpp_accumulators(acc: dict, group=None) -> dict:
    """Merge per-rank D_pp accumulators (the keys of
    stats.new_dpp_accumulators) into the job totals: counts and sums added in
    rank order."""
    import torch

    gathered = {k: _gather(acc[k] if isinstance(acc[k], torch.Tensor) else torch.as_tensor(np.asarray(acc[k])), group)
                for k in DPP_KEYS}
    out = {k: gathered[k][0].copy() for k in DPP_KEYS}
    for r in range(1, len(gathered["counts"])):
        for k in DPP_KEYS:
            out[k] = out[k] + gathered[k][r]
    return out
