"""Generate tests/golden/small_case.npz.

A second, independent restatement of the reference's Float64 path written
in scalar pure Python (Python floats are IEEE doubles; every operation is
rounded on its own, as in Julia without @fastmath):

  push  -- trilinear_sample, E = -(u x B), boris_push, wrap_periodic_coordinate
           and the advance_particles_kernel! / reconstruct_mu_step_kernel!
           save semantics (src/phase_space_gpu_runner.jl:247-391,
           src/multimode_multienergy_cache_pipeline.jl:1349-1374, 1466-1500)
  D_mumu -- mu_bin_index_full and the sliding / injection estimators
           (src/compute_delta_mu2_dmumu_full.jl:304-318, 457-654)

The script checks the restatement against the C oracle (oracle/pt_oracle.c)
-- bit for bit for the push and the integer counts, to 1e-15 for the FP64
sums -- and only then writes the fixture (inputs + outputs).  The tests then
hold both the oracle and the CUDA library to it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

Q, M, C = 1.602176634e-19, 1.67262192369e-27, 2.99792458e8


def cell(f, n):
    c = float(math.floor(f)) if math.isfinite(f) else 1.0
    return min(max(c, 1.0), float(n - 1))


def trilinear(arr, x, y, z, g):
    fx = (x - g["xmin"]) / g["dx"] + 1.0
    fy = (y - g["ymin"]) / g["dy"] + 1.0
    fz = (z - g["zmin"]) / g["dz"] + 1.0
    ci, cj, ck = cell(fx, g["nx"]), cell(fy, g["ny"]), cell(fz, g["nz"])
    tx, ty, tz = fx - ci, fy - cj, fz - ck
    i, j, k = int(ci) - 1, int(cj) - 1, int(ck) - 1
    a = lambda di, dj, dk: float(arr[k + dk, j + dj, i + di])  # noqa: E731  C-ordered (nz, ny, nx)
    c00 = a(0, 0, 0) * (1.0 - tx) + a(1, 0, 0) * tx
    c10 = a(0, 1, 0) * (1.0 - tx) + a(1, 1, 0) * tx
    c01 = a(0, 0, 1) * (1.0 - tx) + a(1, 0, 1) * tx
    c11 = a(0, 1, 1) * (1.0 - tx) + a(1, 1, 1) * tx
    c0 = c00 * (1.0 - ty) + c10 * ty
    c1 = c01 * (1.0 - ty) + c11 * ty
    return c0 * (1.0 - tz) + c1 * tz


def pitch_mu(px, py, pz, bx, by, bz):
    pn = math.sqrt(px * px + py * py + pz * pz)
    bn = math.sqrt(bx * bx + by * by + bz * bz)
    if not math.isfinite(pn) or not math.isfinite(bn) or pn == 0.0 or bn == 0.0:
        return math.nan
    mu = (px * bx + py * by + pz * bz) / (pn * bn)
    return 1.0 if mu > 1.0 else (-1.0 if mu < -1.0 else mu)


def boris(px, py, pz, x, y, z, ex, ey, ez, bx, by, bz, dt):
    half = dt / 2.0
    pmx, pmy, pmz = px + Q * ex * half, py + Q * ey * half, pz + Q * ez * half
    gm = math.sqrt(1.0 + (pmx * pmx + pmy * pmy + pmz * pmz) / ((M * M) * (C * C)))
    tx, ty, tz = Q * bx * dt / (2.0 * M * gm), Q * by * dt / (2.0 * M * gm), Q * bz * dt / (2.0 * M * gm)
    t2 = tx * tx + ty * ty + tz * tz
    sx, sy, sz = 2.0 * tx / (1.0 + t2), 2.0 * ty / (1.0 + t2), 2.0 * tz / (1.0 + t2)
    ppx, ppy, ppz = pmx + (pmy * tz - pmz * ty), pmy + (pmz * tx - pmx * tz), pmz + (pmx * ty - pmy * tx)
    qx, qy, qz = pmx + (ppy * sz - ppz * sy), pmy + (ppz * sx - ppx * sz), pmz + (ppx * sy - ppy * sx)
    nx_, ny_, nz_ = qx + Q * ex * half, qy + Q * ey * half, qz + Q * ez * half
    gn = math.sqrt(1.0 + (nx_ * nx_ + ny_ * ny_ + nz_ * nz_) / ((M * M) * (C * C)))
    return nx_, ny_, nz_, x + nx_ / (gn * M) * dt, y + ny_ / (gn * M) * dt, z + nz_ / (gn * M) * dt


def wrap(x, lo, hi):
    w = hi - lo
    return x - math.floor((x - lo) / w) * w


def push_py(fields, g, st, dt, nsteps, stride, periodic):
    n = len(st["x1"])
    nsave = (nsteps - 1) // stride + 1
    mu = np.full((nsave, n), np.nan, np.float32)
    alive_count = np.zeros(nsteps, np.int64)
    out = {k: np.array(v, copy=True) for k, v in st.items()}
    alive = np.ones(n, bool)
    for p in range(n):
        x, y, z = float(st["x1"][p]), float(st["x2"][p]), float(st["x3"][p])
        px, py, pz = float(st["p1"][p]), float(st["p2"][p]), float(st["p3"][p])
        al = True
        for s in range(nsteps):
            save = s % stride == 0
            if save:
                m = math.nan
                if al and g["xmin"] <= x <= g["xmax"] and g["ymin"] <= y <= g["ymax"] and g["zmin"] <= z <= g["zmax"]:
                    b = [trilinear(fields[c], x, y, z, g) for c in range(3)]
                    m = pitch_mu(px, py, pz, *b)
                mu[s // stride, p] = np.float32(m)
            if al and s < nsteps - 1:
                bx, by, bz, ux, uy, uz = (trilinear(fields[c], x, y, z, g) for c in range(6))
                ex, ey, ez = -(uy * bz - uz * by), -(uz * bx - ux * bz), -(ux * by - uy * bx)
                px, py, pz, x, y, z = boris(px, py, pz, x, y, z, ex, ey, ez, bx, by, bz, dt)
                if periodic:
                    x, y, z = wrap(x, g["xmin"], g["xmax"]), wrap(y, g["ymin"], g["ymax"]), wrap(z, g["zmin"], g["zmax"])
                elif not (g["xmin"] <= x <= g["xmax"] and g["ymin"] <= y <= g["ymax"] and g["zmin"] <= z <= g["zmax"]):
                    al = False
            if al:
                alive_count[s] += 1
        out["x1"][p], out["x2"][p], out["x3"][p] = x, y, z
        out["p1"][p], out["p2"][p], out["p3"][p] = px, py, pz
        alive[p] = al
    return mu, out, alive_count, alive


def bin_index(v, edges):
    if not math.isfinite(v) or v < edges[0] or v > edges[-1]:
        return 0
    b = int(np.searchsorted(edges, v, side="right"))  # searchsortedlast (1-based)
    return len(edges) - 1 if b == len(edges) else b


def dmumu_py(mu, lags, edges, injection, bin_abs):
    n, nsave = mu.shape
    nb, nl = len(edges) - 1, len(lags)
    cnt = np.zeros((nl, nb), np.int64)
    sd, sd2 = np.zeros((nl, nb)), np.zeros((nl, nb))
    pn = np.zeros(nl, np.int64)
    for li, L in enumerate(lags):
        if L >= nsave:
            continue
        last = 1 if injection else nsave - L
        for p in range(n):
            for s in range(last):
                a, b = float(mu[p, s]), float(mu[p, s + L])
                if not (math.isfinite(a) and math.isfinite(b)):
                    continue
                d = b - a
                pn[li] += 1
                bi = bin_index(abs(a) if bin_abs else a, edges)
                if 1 <= bi <= nb:
                    cnt[li, bi - 1] += 1
                    sd[li, bi - 1] += d
                    sd2[li, bi - 1] += d * d
    return cnt, sd, sd2, pn


def main():
    from helpers import copy_state, fortran_fields, random_mu_cache, small_problem, zero_dmumu
    from oracle import build as ob
    from oracle import oracle as o
    from particle_transport_b200.time_units import build_mu_edges_full

    ob.build()
    pb = small_problem(n=6, n_particles=12, energy_GeV=3.0, u_over_c=3e-4, seed=11)
    g = {k: getattr(pb.grid, k) for k in ("nx", "ny", "nz", "xmin", "ymin", "zmin", "xmax", "ymax", "zmax", "dx", "dy",
                                         "dz")}
    nsteps, stride = 81, 4
    res = {}
    for periodic in (True, False):
        mu_py, st_py, ac_py, al_py = push_py(pb.fields, g, pb.state, pb.dt, nsteps, stride, periodic)
        st_o = copy_state(pb.state)
        al_o = np.ones(12, np.uint8)
        mu_o, ac_o = o.push_run(fortran_fields(pb.fields), pb.grid, st_o, al_o, pb.dt, nsteps, stride,
                                periodic=periodic, cache_mode=1)
        assert np.array_equal(mu_py, mu_o, equal_nan=True), "mu cache: Python and C restatements differ"
        for k in st_py:
            assert np.array_equal(st_py[k], st_o[k]), f"final {k}: Python and C restatements differ"
        assert np.array_equal(ac_py, ac_o) and np.array_equal(al_py.astype(np.uint8), al_o)
        tag = "periodic" if periodic else "open"
        res[f"mu_{tag}"] = mu_o
        res[f"alive_count_{tag}"] = ac_o
        for k in st_o:
            res[f"final_{k}_{tag}"] = st_o[k]
    mu = random_mu_cache(9, 37, seed=5, nan_frac=0.05)
    mu[0, 3] = 0.5  # exactly on an edge
    mu[1, 0] = 1.0
    mu[2, 0] = -1.0
    lags = np.array([1, 2, 5, 17, 36, 37], np.int64)
    edges, _ = build_mu_edges_full(0.0, 1.0, 8)
    for inj in (False, True):
        cnt, sd, sd2, pn = dmumu_py(mu, lags, edges, inj, True)
        acc = zero_dmumu(len(lags), 8)
        o.dmumu_accumulate(mu, lags, edges, acc, injection=inj, nthreads=1)
        assert np.array_equal(cnt, acc["counts"]) and np.array_equal(pn, acc["pair_n"])
        assert np.allclose(sd, acc["sum_d"], rtol=1e-15, atol=1e-17) and np.allclose(sd2, acc["sum_d2"], rtol=1e-15)
        tag = "injection" if inj else "sliding"
        for k, v in acc.items():
            res[f"dmumu_{tag}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "small_case.npz"), fields=np.stack(pb.fields), state_x1=pb.state["x1"],
                        state_x2=pb.state["x2"], state_x3=pb.state["x3"], state_p1=pb.state["p1"],
                        state_p2=pb.state["p2"], state_p3=pb.state["p3"], dt=pb.dt, nsteps=nsteps, stride=stride,
                        grid=np.array([g[k] for k in ("xmin", "ymin", "zmin", "xmax", "ymax", "zmax", "dx", "dy", "dz")]),
                        grid_n=np.array([g["nx"], g["ny"], g["nz"]]), mu_cache=mu, lags=lags, edges=edges, **res)
    print("wrote", os.path.join(HERE, "small_case.npz"))


if __name__ == "__main__":
    main()
