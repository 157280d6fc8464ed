/*
 * CPU ORACLE -- test infrastructure only.
 *
 * This file is a plain-C restatement of the reference's Float64 algorithms on
 * the trajectory / transport-statistics path.  It is the checker for the CUDA
 * library: only the tests, the smoke check and bench.py's CPU-baseline leg
 * load it.  The product never links or calls it.
 *
 * Parity status: the reference is Julia (CUDA.jl kernels + threaded CPU
 * loops) and cannot run here (no julia binary); the push exists in the
 * reference only as a CUDA.jl kernel.  The reference's own tests pin only
 * the time/lag grid host logic (test/runtests.jl), which the host package
 * restates and checks.  The arithmetic below is therefore pinned by analytic
 * known-answer tests (uniform-B rotation angle 2*atan(|t|), |p| and gamma
 * conservation, hand-built mu caches with closed-form bin counts, pair-visit
 * counts) and NOT by reference outputs: "parity unpinned" against the running
 * reference.
 *
 * Operation order is literal: every expression below follows the reference
 * expression tree (Julia evaluates a*b*c as (a*b)*c, x^2 as x*x and does not
 * contract into FMA), and this file is compiled with -ffp-contract=off so
 * that the results are bit-identical to a Julia Float64 run on IEEE hardware.
 *
 * Citations are src/<file>.jl:<line> in the reference project.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/phase_space_gpu_runner.jl:8-12 */
#define OR_C_LIGHT 2.99792458e8
#define OR_Q_E 1.602176634e-19
#define OR_M_P 1.67262192369e-27

typedef struct {
    int64_t nx, ny, nz;
    double xmin, ymin, zmin;
    double xmax, ymax, zmax;
    double dx, dy, dz;
} or_grid;

/* clamp(floor(Int, f), 1, n - 1), returned as the Float64 value of the index.
 * Julia's floor(Int, f) throws for NaN; here NaN maps to the lower clamp. */
static inline double or_cell(double f, int64_t n)
{
    double c = floor(f);
    double hi = (double)(n - 1);
    if (!(c >= 1.0)) c = 1.0;
    if (c > hi) c = hi;
    return c;
}

/* trilinear_sample: src/phase_space_gpu_runner.jl:247-276 (identical copy at
 * src/compute_delta_mu2_curve.jl:62-91).  arr is column-major, x fastest. */
double or_trilinear(const double* arr, double x, double y, double z, const or_grid* g)
{
    double fx = (x - g->xmin) / g->dx + 1.0;
    double fy = (y - g->ymin) / g->dy + 1.0;
    double fz = (z - g->zmin) / g->dz + 1.0;
    double ci = or_cell(fx, g->nx), cj = or_cell(fy, g->ny), ck = or_cell(fz, g->nz);
    double tx = fx - ci, ty = fy - cj, tz = fz - ck;
    int64_t i0 = (int64_t)ci - 1, j0 = (int64_t)cj - 1, k0 = (int64_t)ck - 1;
    int64_t sx = 1, sy = g->nx, sz = g->nx * g->ny;
    const double* b = arr + i0 + sy * j0 + sz * k0;
    double c000 = b[0], c100 = b[sx], c010 = b[sy], c110 = b[sx + sy];
    double c001 = b[sz], c101 = b[sx + sz], c011 = b[sy + sz], c111 = b[sx + sy + sz];
    double c00 = c000 * (1.0 - tx) + c100 * tx;
    double c10 = c010 * (1.0 - tx) + c110 * tx;
    double c01 = c001 * (1.0 - tx) + c101 * tx;
    double c11 = c011 * (1.0 - tx) + c111 * tx;
    double c0 = c00 * (1.0 - ty) + c10 * ty;
    double c1 = c01 * (1.0 - ty) + c11 * ty;
    return c0 * (1.0 - tz) + c1 * tz;
}

/* Float32 instance of the same function, used by the phase-space mu
 * reconstruction at compute_precision = Float32
 * (src/compute_delta_mu2_curve.jl:62-91, 186-225). */
float or_trilinear_f32(const float* arr, float x, float y, float z, float xmin, float ymin, float zmin,
                       float dx, float dy, float dz, int64_t nx, int64_t ny, int64_t nz)
{
    float fx = (x - xmin) / dx + 1.0f;
    float fy = (y - ymin) / dy + 1.0f;
    float fz = (z - zmin) / dz + 1.0f;
    double ci = or_cell((double)fx, nx), cj = or_cell((double)fy, ny), ck = or_cell((double)fz, nz);
    float tx = fx - (float)ci, ty = fy - (float)cj, tz = fz - (float)ck;
    int64_t i0 = (int64_t)ci - 1, j0 = (int64_t)cj - 1, k0 = (int64_t)ck - 1;
    int64_t sx = 1, sy = nx, sz = nx * ny;
    const float* b = arr + i0 + sy * j0 + sz * k0;
    float c000 = b[0], c100 = b[sx], c010 = b[sy], c110 = b[sx + sy];
    float c001 = b[sz], c101 = b[sx + sz], c011 = b[sy + sz], c111 = b[sx + sy + sz];
    float c00 = c000 * (1.0f - tx) + c100 * tx;
    float c10 = c010 * (1.0f - tx) + c110 * tx;
    float c01 = c001 * (1.0f - tx) + c101 * tx;
    float c11 = c011 * (1.0f - tx) + c111 * tx;
    float c0 = c00 * (1.0f - ty) + c10 * ty;
    float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

/* pitch_mu_from_pB: src/compute_delta_mu2_curve.jl:93-110 */
double or_pitch_mu(double px, double py, double pz, double bx, double by, double bz)
{
    double pn = sqrt(px * px + py * py + pz * pz);
    double bn = sqrt(bx * bx + by * by + bz * bz);
    if (!isfinite(pn) || !isfinite(bn) || pn == 0.0 || bn == 0.0) return NAN;
    double mu = (px * bx + py * by + pz * bz) / (pn * bn);
    return mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
}

float or_pitch_mu_f32(float px, float py, float pz, float bx, float by, float bz)
{
    float pn = sqrtf(px * px + py * py + pz * pz);
    float bn = sqrtf(bx * bx + by * by + bz * bz);
    if (!isfinite(pn) || !isfinite(bn) || pn == 0.0f || bn == 0.0f) return NAN;
    float mu = (px * bx + py * by + pz * bz) / (pn * bn);
    return mu > 1.0f ? 1.0f : (mu < -1.0f ? -1.0f : mu);
}

/* boris_push: src/phase_space_gpu_runner.jl:282-323 (qm is the charge q). */
static inline void or_boris(double* px, double* py, double* pz, double* x, double* y, double* z,
                            double ex, double ey, double ez, double bx, double by, double bz, double dt)
{
    const double half = dt / 2.0;
    const double qm = OR_Q_E, mp = OR_M_P, cl = OR_C_LIGHT;
    double pmx = *px + qm * ex * half;
    double pmy = *py + qm * ey * half;
    double pmz = *pz + qm * ez * half;
    double gamma_minus = sqrt(1.0 + (pmx * pmx + pmy * pmy + pmz * pmz) / ((mp * mp) * (cl * cl)));
    double tx = qm * bx * dt / (2.0 * mp * gamma_minus);
    double ty = qm * by * dt / (2.0 * mp * gamma_minus);
    double tz = qm * bz * dt / (2.0 * mp * gamma_minus);
    double t2 = tx * tx + ty * ty + tz * tz;
    double sx = 2.0 * tx / (1.0 + t2);
    double sy = 2.0 * ty / (1.0 + t2);
    double sz = 2.0 * tz / (1.0 + t2);
    /* cross3: src/phase_space_gpu_runner.jl:278-280 */
    double ppx = pmx + (pmy * tz - pmz * ty);
    double ppy = pmy + (pmz * tx - pmx * tz);
    double ppz = pmz + (pmx * ty - pmy * tx);
    double ppx2 = pmx + (ppy * sz - ppz * sy);
    double ppy2 = pmy + (ppz * sx - ppx * sz);
    double ppz2 = pmz + (ppx * sy - ppy * sx);
    double pxn = ppx2 + qm * ex * half;
    double pyn = ppy2 + qm * ey * half;
    double pzn = ppz2 + qm * ez * half;
    double gamma_new = sqrt(1.0 + (pxn * pxn + pyn * pyn + pzn * pzn) / ((mp * mp) * (cl * cl)));
    double vxn = pxn / (gamma_new * mp);
    double vyn = pyn / (gamma_new * mp);
    double vzn = pzn / (gamma_new * mp);
    *px = pxn; *py = pyn; *pz = pzn;
    *x = *x + vxn * dt; *y = *y + vyn * dt; *z = *z + vzn * dt;
}

/* wrap_periodic_coordinate: src/phase_space_gpu_runner.jl:325-328 */
static inline double or_wrap(double x, double xmin, double xmax)
{
    double width = xmax - xmin;
    return x - floor((x - xmin) / width) * width;
}

/* mu at the pre-push state: reconstruct_mu_step_kernel!,
 * src/multimode_multienergy_cache_pipeline.jl:1349-1374 */
static inline double or_mu_at(const double* const* f, const or_grid* g, double xx, double yy, double zz,
                              double px, double py, double pz)
{
    if (isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) return NAN;
    if (!(g->xmin <= xx && xx <= g->xmax && g->ymin <= yy && yy <= g->ymax && g->zmin <= zz && zz <= g->zmax))
        return NAN;
    double bx = or_trilinear(f[0], xx, yy, zz, g);
    double by = or_trilinear(f[1], xx, yy, zz, g);
    double bz = or_trilinear(f[2], xx, yy, zz, g);
    return or_pitch_mu(px, py, pz, bx, by, bz);
}

/*
 * Host step loop + advance_particles_kernel! for steps [step_begin,
 * step_begin + step_count) of an ensemble of nsteps samples (0-based step s
 * is reference step si = s + 1):
 *   src/phase_space_gpu_runner.jl:330-391 (kernel), 561-591 (loop);
 *   src/multimode_multienergy_cache_pipeline.jl:1466-1500 (mu-cache loop).
 * At s % stride == 0 the pre-push state is recorded into save row s / stride:
 *   cache_mode 1: mu_out[row * n + p] (float if out_f64 == 0 else double)
 *   cache_mode 2: pos_out / mom_out[(row * 3 + c) * n + p]
 * alive_count[s] receives the number of live particles after the push of step s
 * (sum(dalive) at src/phase_space_gpu_runner.jl:576).
 * fields: Bx, By, Bz, ux, uy, uz in SI units, column-major, x fastest.
 */
void or_push_run(const double* const* f, const or_grid* g, double* x1, double* x2, double* x3, double* p1,
                 double* p2, double* p3, uint8_t* alive, int64_t n, double dt, int64_t nsteps, int64_t step_begin,
                 int64_t step_count, int64_t stride, int periodic, int cache_mode, int out_f64, void* mu_out,
                 void* pos_out, void* mom_out, int64_t* alive_count, int nthreads)
{
    int64_t s_end = step_begin + step_count;
    /* death step per particle (-1: alive at the end, -2: dead on entry) */
    int64_t* died = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < n; ++p) {
        double xx = x1[p], yy = x2[p], zz = x3[p], px = p1[p], py = p2[p], pz = p3[p];
        int al = alive[p] != 0;
        died[p] = al ? -1 : -2;
        for (int64_t s = step_begin; s < s_end; ++s) {
            double sx_ = NAN, sy_ = NAN, sz_ = NAN, spx = NAN, spy = NAN, spz = NAN;
            if (al) {
                sx_ = xx; sy_ = yy; sz_ = zz; spx = px; spy = py; spz = pz;
                if (s < nsteps - 1) {
                    double bx = or_trilinear(f[0], xx, yy, zz, g);
                    double by = or_trilinear(f[1], xx, yy, zz, g);
                    double bz = or_trilinear(f[2], xx, yy, zz, g);
                    double vfx = or_trilinear(f[3], xx, yy, zz, g);
                    double vfy = or_trilinear(f[4], xx, yy, zz, g);
                    double vfz = or_trilinear(f[5], xx, yy, zz, g);
                    double ex = -(vfy * bz - vfz * by);
                    double ey = -(vfz * bx - vfx * bz);
                    double ez = -(vfx * by - vfy * bx);
                    or_boris(&px, &py, &pz, &xx, &yy, &zz, ex, ey, ez, bx, by, bz, dt);
                    if (periodic) {
                        xx = or_wrap(xx, g->xmin, g->xmax);
                        yy = or_wrap(yy, g->ymin, g->ymax);
                        zz = or_wrap(zz, g->zmin, g->zmax);
                    } else if (xx < g->xmin || xx > g->xmax || yy < g->ymin || yy > g->ymax || zz < g->zmin ||
                               zz > g->zmax) {
                        al = 0;
                        died[p] = s;
                    }
                }
            }
            if (s % stride == 0) {
                int64_t row = s / stride;
                if (cache_mode == 1) {
                    double mu = or_mu_at(f, g, sx_, sy_, sz_, spx, spy, spz);
                    if (out_f64) ((double*)mu_out)[row * n + p] = mu;
                    else ((float*)mu_out)[row * n + p] = (float)mu;
                } else if (cache_mode == 2) {
                    double v[6] = {sx_, sy_, sz_, spx, spy, spz};
                    for (int c = 0; c < 3; ++c) {
                        int64_t idx = (row * 3 + c) * n + p;
                        if (out_f64) {
                            ((double*)pos_out)[idx] = v[c];
                            ((double*)mom_out)[idx] = v[3 + c];
                        } else {
                            ((float*)pos_out)[idx] = (float)v[c];
                            ((float*)mom_out)[idx] = (float)v[3 + c];
                        }
                    }
                }
            }
        }
        x1[p] = xx; x2[p] = yy; x3[p] = zz; p1[p] = px; p2[p] = py; p3[p] = pz;
        alive[p] = (uint8_t)al;
    }
    if (alive_count) {
        int64_t live0 = 0;
        for (int64_t s = step_begin; s < s_end; ++s) alive_count[s] = 0;
        for (int64_t p = 0; p < n; ++p) {
            if (died[p] == -2) continue;
            live0 += 1;
            if (died[p] >= 0) alive_count[died[p]] -= 1;
        }
        int64_t run = live0;
        for (int64_t s = step_begin; s < s_end; ++s) {
            run += alive_count[s];
            alive_count[s] = run;
        }
    }
    free(died);
}

/*
 * Phase-space mu reconstruction (reconstruct_mu_chunk_cpu / _gpu,
 * src/compute_delta_mu2_curve.jl:112-225).  positions / momenta are the
 * cache layout Julia (chunk, 3, nsave): element [p, c, s] at (s*3 + c)*chunk + p.
 * mu_out is Julia (nsave, chunk): element [s, p] at p*nsave + s.
 * Fields and grid scalars are given in the compute precision.
 */
void or_reconstruct_mu_f64(const double* pos, const double* mom, int64_t chunk, int64_t nsave,
                           const double* const* bfield, const or_grid* g, double* mu_out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < chunk; ++p)
        for (int64_t s = 0; s < nsave; ++s) {
            const double* P = pos + s * 3 * chunk + p;
            const double* M = mom + s * 3 * chunk + p;
            mu_out[p * nsave + s] = or_mu_at(bfield, g, P[0], P[chunk], P[2 * chunk], M[0], M[chunk], M[2 * chunk]);
        }
}

void or_reconstruct_mu_f32(const float* pos, const float* mom, int64_t chunk, int64_t nsave,
                           const float* const* bfield, int64_t nx, int64_t ny, int64_t nz, const float* lims,
                           float* mu_out, int nthreads)
{
    /* lims: xmin ymin zmin xmax ymax zmax dx dy dz, already rounded to Float32 */
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < chunk; ++p)
        for (int64_t s = 0; s < nsave; ++s) {
            const float* P = pos + s * 3 * chunk + p;
            const float* M = mom + s * 3 * chunk + p;
            float xx = P[0], yy = P[chunk], zz = P[2 * chunk];
            float px = M[0], py = M[chunk], pz = M[2 * chunk];
            float v = NAN;
            if (!(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) &&
                lims[0] <= xx && xx <= lims[3] && lims[1] <= yy && yy <= lims[4] && lims[2] <= zz && zz <= lims[5]) {
                float bx = or_trilinear_f32(bfield[0], xx, yy, zz, lims[0], lims[1], lims[2], lims[6], lims[7], lims[8], nx, ny, nz);
                float by = or_trilinear_f32(bfield[1], xx, yy, zz, lims[0], lims[1], lims[2], lims[6], lims[7], lims[8], nx, ny, nz);
                float bz = or_trilinear_f32(bfield[2], xx, yy, zz, lims[0], lims[1], lims[2], lims[6], lims[7], lims[8], nx, ny, nz);
                v = or_pitch_mu_f32(px, py, pz, bx, by, bz);
            }
            mu_out[p * nsave + s] = v;
        }
}

/* mu_bin_value + mu_bin_index_full: src/compute_delta_mu2_dmumu_full.jl:304-318.
 * Returns a 1-based bin in [1, n_bins] or 0 (skip). */
int or_mu_bin_index(double v, const double* edges, int n_bins)
{
    if (!isfinite(v)) return 0;
    if (v < edges[0] || v > edges[n_bins]) return 0;
    /* searchsortedlast: last 1-based i with edges[i] <= v */
    int lo = 0, hi = n_bins + 1; /* count of edges <= v lies in [lo, hi] */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (edges[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    int b = lo;
    if (b == n_bins + 1) return n_bins;
    return b < 1 ? 0 : b;
}

/* combine_welford_stats!: src/compute_delta_mu2_dmumu_full.jl:439-455 */
void or_combine_welford(int64_t* counts, double* means, double* m2s, int64_t lag, int64_t local_count,
                        double local_mean, double local_m2)
{
    if (local_count <= 0) return;
    int64_t global_count = counts[lag];
    if (global_count == 0) {
        counts[lag] = local_count;
        means[lag] = local_mean;
        m2s[lag] = local_m2;
        return;
    }
    int64_t combined = global_count + local_count;
    double delta = local_mean - means[lag];
    means[lag] += delta * (double)local_count / (double)combined;
    m2s[lag] += local_m2 + delta * delta * (double)global_count * (double)local_count / (double)combined;
    counts[lag] = combined;
}

/*
 * process_mu_chunk_dmumu_cpu! and its two estimators:
 *   sliding   src/compute_delta_mu2_dmumu_full.jl:457-560
 *   injection src/compute_delta_mu2_dmumu_full.jl:562-654
 * mu element (particle p, save s) is mu[p * sp + s * ss] (Julia mu_chunk
 * (nsave, chunk) has sp = nsave, ss = 1).  Accumulators are add-into; the
 * (bin, lag) arrays are Julia (n_bins, n_lags): element [b, l] at l*n_bins + b.
 * Threads keep private accumulators merged in thread order, as the reference
 * does per Threads.threadid().
 */
/* mu of (particle p, save s): a Float32 chunk (the cache default) or a
 * Float64 chunk (compute_precision = Float64 in the phase-space path); the
 * reference reads Float64(mu_chunk[s, p]) either way (dmumu:509-510). */
static inline double or_mu_at_index(const float* mu32, const double* mu64, int64_t i)
{
    return mu32 ? (double)mu32[i] : mu64[i];
}

static void or_dmumu_core(const float* mu, const double* mu64, int64_t chunk, int64_t nsave, int64_t sp,
                          int64_t ss, const int64_t* lag_steps, int n_lags, const double* edges, int n_bins,
                          int injection, int bin_abs, int64_t* counts, double* sum_d, double* sum_d2,
                          int64_t* w_count, double* w_mean, double* w_m2, double* pair_ss, int64_t* pair_n,
                          int nthreads)
{
    int nt = 1;
#ifdef _OPENMP
    nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    int64_t* lc = (int64_t*)calloc((size_t)nt * n_bins, sizeof(int64_t));
    double* ld = (double*)calloc((size_t)nt * n_bins, sizeof(double));
    double* ld2 = (double*)calloc((size_t)nt * n_bins, sizeof(double));
    int64_t* tpc = (int64_t*)calloc((size_t)nt, sizeof(int64_t));
    double* tpm = (double*)calloc((size_t)nt, sizeof(double));
    double* tpm2 = (double*)calloc((size_t)nt, sizeof(double));
    double* tss = (double*)calloc((size_t)nt, sizeof(double));
    int64_t* tpn = (int64_t*)calloc((size_t)nt, sizeof(int64_t));

    for (int li = 0; li < n_lags; ++li) {
        int64_t lag = lag_steps[li];
        if (lag >= nsave) continue;
        int64_t last_start = injection ? 1 : nsave - lag;
        memset(lc, 0, sizeof(int64_t) * nt * n_bins);
        memset(ld, 0, sizeof(double) * nt * n_bins);
        memset(ld2, 0, sizeof(double) * nt * n_bins);
        memset(tpc, 0, sizeof(int64_t) * nt);
        memset(tpm, 0, sizeof(double) * nt);
        memset(tpm2, 0, sizeof(double) * nt);
        memset(tss, 0, sizeof(double) * nt);
        memset(tpn, 0, sizeof(int64_t) * nt);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
        for (int64_t p = 0; p < chunk; ++p) {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            double particle_sumsq = 0.0;
            int64_t valid = 0;
            for (int64_t s = 0; s < last_start; ++s) {
                double a = or_mu_at_index(mu, mu64, p * sp + s * ss);
                double b = or_mu_at_index(mu, mu64, p * sp + (s + lag) * ss);
                if (!(isfinite(a) && isfinite(b))) continue;
                double dm = b - a;
                double dm2 = dm * dm;
                particle_sumsq += dm2;
                valid += 1;
                int bi = or_mu_bin_index(bin_abs ? fabs(a) : a, edges, n_bins);
                if (bi >= 1 && bi <= n_bins) {
                    lc[(int64_t)t * n_bins + bi - 1] += 1;
                    ld[(int64_t)t * n_bins + bi - 1] += dm;
                    ld2[(int64_t)t * n_bins + bi - 1] += dm2;
                }
            }
            if (valid > 0) {
                /* sliding: per-particle mean of dmu^2; injection: dmu^2 itself */
                double value = injection ? particle_sumsq : particle_sumsq / (double)valid;
                tpc[t] += 1;
                double delta = value - tpm[t];
                tpm[t] += delta / (double)tpc[t];
                double delta2 = value - tpm[t];
                tpm2[t] += delta * delta2;
                tss[t] += particle_sumsq;
                tpn[t] += valid;
            }
        }
        for (int t = 0; t < nt; ++t) {
            for (int b = 0; b < n_bins; ++b) {
                counts[(int64_t)li * n_bins + b] += lc[(int64_t)t * n_bins + b];
                sum_d[(int64_t)li * n_bins + b] += ld[(int64_t)t * n_bins + b];
                sum_d2[(int64_t)li * n_bins + b] += ld2[(int64_t)t * n_bins + b];
            }
            or_combine_welford(w_count, w_mean, w_m2, li, tpc[t], tpm[t], tpm2[t]);
            pair_ss[li] += tss[t];
            pair_n[li] += tpn[t];
        }
    }
    free(lc); free(ld); free(ld2); free(tpc); free(tpm); free(tpm2); free(tss); free(tpn);
}

void or_dmumu_accumulate(const float* mu, int64_t chunk, int64_t nsave, int64_t sp, int64_t ss,
                         const int64_t* lag_steps, int n_lags, const double* edges, int n_bins, int injection,
                         int bin_abs, int64_t* counts, double* sum_d, double* sum_d2, int64_t* w_count,
                         double* w_mean, double* w_m2, double* pair_ss, int64_t* pair_n, int nthreads)
{
    or_dmumu_core(mu, NULL, chunk, nsave, sp, ss, lag_steps, n_lags, edges, n_bins, injection, bin_abs, counts,
                  sum_d, sum_d2, w_count, w_mean, w_m2, pair_ss, pair_n, nthreads);
}

void or_dmumu_accumulate_f64(const double* mu, int64_t chunk, int64_t nsave, int64_t sp, int64_t ss,
                             const int64_t* lag_steps, int n_lags, const double* edges, int n_bins, int injection,
                             int bin_abs, int64_t* counts, double* sum_d, double* sum_d2, int64_t* w_count,
                             double* w_mean, double* w_m2, double* pair_ss, int64_t* pair_n, int nthreads)
{
    or_dmumu_core(NULL, mu, chunk, nsave, sp, ss, lag_steps, n_lags, edges, n_bins, injection, bin_abs, counts,
                  sum_d, sum_d2, w_count, w_mean, w_m2, pair_ss, pair_n, nthreads);
}

/* momentum_magnitude: src/compute_dpp_full.jl:232-234 */
static inline double or_pmag(float px, float py, float pz)
{
    double x = (double)px, y = (double)py, z = (double)pz;
    return sqrt(x * x + y * y + z * z);
}

/*
 * process_momenta_chunk_dpp_cpu!: src/compute_dpp_full.jl:247-288.
 * momenta is the cache layout Julia (chunk, 3, nsave): [p, c, s] at
 * (s*3 + c)*chunk + p.  Accumulators [n_lags] are add-into.
 */
void or_dpp_accumulate(const float* mom, int64_t chunk, int64_t nsave, const int64_t* lag_steps, int n_lags,
                       double p0, int64_t* counts, double* sdp, double* sdp2, double* sdn, double* sdn2, int nthreads)
{
    int nt = 1;
#ifdef _OPENMP
    nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    int64_t* lc = (int64_t*)calloc((size_t)nt, sizeof(int64_t));
    double* acc = (double*)calloc((size_t)nt * 4, sizeof(double));
    for (int li = 0; li < n_lags; ++li) {
        int64_t lag = lag_steps[li];
        if (lag >= nsave) continue;
        int64_t last_start = nsave - lag;
        memset(lc, 0, sizeof(int64_t) * nt);
        memset(acc, 0, sizeof(double) * nt * 4);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
        for (int64_t p = 0; p < chunk; ++p) {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            for (int64_t s = 0; s < last_start; ++s) {
                const float* a = mom + s * 3 * chunk + p;
                const float* b = mom + (s + lag) * 3 * chunk + p;
                double ps = or_pmag(a[0], a[chunk], a[2 * chunk]);
                double pe = or_pmag(b[0], b[chunk], b[2 * chunk]);
                if (!(isfinite(ps) && isfinite(pe))) continue;
                double d = pe - ps;
                double dn = d / p0;
                lc[t] += 1;
                acc[t * 4 + 0] += d;
                acc[t * 4 + 1] += d * d;
                acc[t * 4 + 2] += dn;
                acc[t * 4 + 3] += dn * dn;
            }
        }
        int64_t c = 0;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int t = 0; t < nt; ++t) {
            c += lc[t];
            a0 += acc[t * 4 + 0]; a1 += acc[t * 4 + 1]; a2 += acc[t * 4 + 2]; a3 += acc[t * 4 + 3];
        }
        counts[li] += c; sdp[li] += a0; sdp2[li] += a1; sdn[li] += a2; sdn2[li] += a3;
    }
    free(lc); free(acc);
}

/* kinetic_energy_gev_from_pmag + fill_energy_snapshots!:
 * src/compute_dpp_full.jl:236-240, 290-299.  snap_steps are 0-based save
 * indices; out is Julia (n_snap, n_total): [j, q] at q*n_snap + j, written for
 * q = particle_offset + p (0-based). */
double or_kinetic_energy_gev(double pmag)
{
    if (!isfinite(pmag)) return NAN;
    const double gev_to_j = 1.0e9 * 1.602176634e-19;
    double r = pmag / (OR_M_P * OR_C_LIGHT);
    double gamma = sqrt(1.0 + r * r);
    return (gamma - 1.0) * OR_M_P * (OR_C_LIGHT * OR_C_LIGHT) / gev_to_j;
}

void or_energy_snapshots(const float* mom, int64_t chunk, int64_t nsave, const int64_t* snap_steps, int n_snap,
                         int64_t particle_offset, double* out)
{
    (void)nsave;
    for (int j = 0; j < n_snap; ++j) {
        int64_t s = snap_steps[j];
        for (int64_t p = 0; p < chunk; ++p) {
            const float* a = mom + s * 3 * chunk + p;
            out[(particle_offset + p) * n_snap + j] = or_kinetic_energy_gev(or_pmag(a[0], a[chunk], a[2 * chunk]));
        }
    }
}

/* ------------------------------------------------------------------------
 * Derived product arrays: the formulas that turn the accumulators into the
 * numbers the reference writes into its HDF5 products and tables.
 * --------------------------------------------------------------------- */

/* Julia's max(0.0, x) for Float64: NaN propagates (C's fmax would drop it). */
static inline double or_jl_max0(double x)
{
    if (isnan(x)) return x;
    return x > 0.0 ? x : 0.0;
}

/* compute_dmumu_arrays_full: src/compute_delta_mu2_dmumu_full.jl:706-744.
 * counts/sum_d/sum_d2 are Julia (n_bins, n_lags) arrays, bins fastest.  out
 * holds seven arrays of that shape one after another: mean_delta,
 * mean_delta2, drift_norm, dmumu_raw_norm, dmumu_centered_norm,
 * dmumu_raw_per_s, dmumu_centered_per_s.  Cells with count < min_count stay
 * NaN (fill(NaN, ...)). */
void or_dmumu_arrays_full(const int64_t* counts, const double* sum_d, const double* sum_d2, const double* tau_s,
                          const double* tau_norm, int n_lags, int n_bins, int64_t min_count, double* out)
{
    const int64_t cells = (int64_t)n_lags * n_bins;
    for (int64_t i = 0; i < 7 * cells; ++i) out[i] = NAN;
    for (int l = 0; l < n_lags; ++l) {
        const double normalized_lag = tau_norm[l];
        const double physical_lag = tau_s[l];
        for (int b = 0; b < n_bins; ++b) {
            const int64_t c = (int64_t)l * n_bins + b;
            const int64_t count = counts[c];
            if (!(count >= min_count)) continue;
            const double delta_mean = sum_d[c] / (double)count;
            const double delta2_mean = sum_d2[c] / (double)count;
            const double centered = or_jl_max0(delta2_mean - delta_mean * delta_mean);
            out[0 * cells + c] = delta_mean;
            out[1 * cells + c] = delta2_mean;
            out[2 * cells + c] = delta_mean / normalized_lag;
            out[3 * cells + c] = delta2_mean / (2.0 * normalized_lag);
            out[4 * cells + c] = centered / (2.0 * normalized_lag);
            out[5 * cells + c] = delta2_mean / (2.0 * physical_lag);
            out[6 * cells + c] = centered / (2.0 * physical_lag);
        }
    }
}

/* average_over_tau_full: src/compute_delta_mu2_dmumu_full.jl:746-776.
 * values/counts are Julia (n_bins, n_lags); out_unweighted and
 * out_count_weighted have n_bins entries (NaN where no lag qualifies). */
void or_average_over_tau_full(const double* values, const int64_t* counts, int n_lags, int n_bins,
                              int64_t min_count, double* out_unweighted, double* out_count_weighted)
{
    for (int b = 0; b < n_bins; ++b) {
        double value_sum = 0.0, weighted_sum = 0.0;
        int64_t valid_lags = 0, total_weight = 0;
        for (int l = 0; l < n_lags; ++l) {
            const double value = values[(int64_t)l * n_bins + b];
            const int64_t count = counts[(int64_t)l * n_bins + b];
            if (isfinite(value) && count >= min_count) {
                value_sum += value;
                valid_lags += 1;
                weighted_sum += value * (double)count;
                total_weight += count;
            }
        }
        out_unweighted[b] = valid_lags > 0 ? value_sum / (double)valid_lags : NAN;
        out_count_weighted[b] = total_weight > 0 ? weighted_sum / (double)total_weight : NAN;
    }
}

/* sem_from_stats: src/compute_delta_mu2_curve.jl:387-393. */
double or_sem_from_stats(int64_t count, double m2)
{
    if (count <= 1) return NAN;
    const double variance = m2 / (double)(count - 1);
    return sqrt(variance / (double)count);
}

/* The computed columns of build_output_dataframe:
 * src/compute_delta_mu2_curve.jl:409-429.  lag_steps are offsets into the
 * sample times t_s / t_norm (0-based here: t[lag] - t[0] is Julia's
 * t[lag + 1] - t[1]).  out holds six n_lags arrays: tau_s, tau_norm,
 * tau_gyroperiods (tOmega0_to_gyroperiods, src/time_units.jl:8),
 * delta_mu2_particle_std, delta_mu2_particle_sem, delta_mu2_pair_mean. */
void or_output_table(const int64_t* lag_steps, int n_lags, const double* t_s, const double* t_norm,
                     const int64_t* particle_counts, const double* particle_m2s, const double* pair_sum_squares,
                     const int64_t* pair_counts, double* out)
{
    const double two_pi = 2.0 * 3.141592653589793;
    for (int l = 0; l < n_lags; ++l) {
        const int64_t lag = lag_steps[l];
        const double tau_norm = t_norm[lag] - t_norm[0];
        const int64_t count = particle_counts[l];
        out[0 * n_lags + l] = t_s[lag] - t_s[0];
        out[1 * n_lags + l] = tau_norm;
        out[2 * n_lags + l] = tau_norm / two_pi;
        out[3 * n_lags + l] = count <= 1 ? NAN : sqrt(particle_m2s[l] / (double)(count - 1));
        out[4 * n_lags + l] = or_sem_from_stats(count, particle_m2s[l]);
        out[5 * n_lags + l] = pair_counts[l] == 0 ? NAN : pair_sum_squares[l] / (double)pair_counts[l];
    }
}

/* compute_dpp_arrays: src/compute_dpp_full.jl:301-330.  Inputs are the five
 * per-lag accumulators; out holds eight n_lags arrays: mean_delta_p,
 * mean_delta_p2, mean_delta_p_norm, mean_delta_p_norm2, dpp_raw_per_s,
 * dpp_centered_per_s, dpp_raw_norm, dpp_centered_norm (NaN where count = 0). */
void or_dpp_arrays(const int64_t* counts, const double* sum_dp, const double* sum_dp2, const double* sum_dpn,
                   const double* sum_dpn2, const double* tau_s, const double* tau_norm, int n_lags, double* out)
{
    for (int64_t i = 0; i < 8 * (int64_t)n_lags; ++i) out[i] = NAN;
    for (int l = 0; l < n_lags; ++l) {
        const int64_t count = counts[l];
        if (!(count > 0)) continue;
        const double delta_mean = sum_dp[l] / (double)count;
        const double delta2_mean = sum_dp2[l] / (double)count;
        const double norm_mean = sum_dpn[l] / (double)count;
        const double norm2_mean = sum_dpn2[l] / (double)count;
        const double centered = or_jl_max0(delta2_mean - delta_mean * delta_mean);
        const double centered_norm = or_jl_max0(norm2_mean - norm_mean * norm_mean);
        out[0 * n_lags + l] = delta_mean;
        out[1 * n_lags + l] = delta2_mean;
        out[2 * n_lags + l] = norm_mean;
        out[3 * n_lags + l] = norm2_mean;
        out[4 * n_lags + l] = delta2_mean / (2.0 * tau_s[l]);
        out[5 * n_lags + l] = centered / (2.0 * tau_s[l]);
        out[6 * n_lags + l] = norm2_mean / (2.0 * tau_norm[l]);
        out[7 * n_lags + l] = centered_norm / (2.0 * tau_norm[l]);
    }
}

/* ------------------------------------------------------------------------
 * Particle initialisation: init_particles / rand_unit_vector /
 * fixed_mu_unit_vector (src/phase_space_gpu_runner.jl:51-66, 170-245) over
 * the counter-based stream of the device initialiser: draw d of particle i
 * is the SplitMix64 output of counter 8 i + d + 1 under key mix64(seed)
 * (Steele, Lea, Flood 2014), as (h >> 11) * 2^-53.  Draws 0-2 position,
 * draw 3 z (isotropic) or phi (fixed mu), draw 4 phi (isotropic).
 * Returns the number of particles where fixed-mu injection met a zero or
 * non-finite |B| (their momenta are NaN).
 * --------------------------------------------------------------------- */
static inline uint64_t or_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double or_draw(uint64_t key, int64_t i, int d)
{
    uint64_t c = (uint64_t)i * 8u + (uint64_t)d + 1u;
    return (double)(or_mix64(key + c * 0x9E3779B97F4A7C15ull) >> 11) * 0x1.0p-53;
}

int64_t or_init_particles(int64_t n, uint64_t seed, double energy_GeV, int fixed_mu, int random_pos, double mu0,
                          const double* position, const double* const* bfield, const or_grid* g, double* x1,
                          double* x2, double* x3, double* p1, double* p2, double* p3)
{
    const double two_pi = 6.283185307179586; /* Float64(2 * pi) */
    const double gev_to_j = 1e9 * 1.602176634e-19;
    double kinetic = energy_GeV * gev_to_j;
    double gamma0 = kinetic / (OR_M_P * (OR_C_LIGHT * OR_C_LIGHT)) + 1.0;
    double v0 = OR_C_LIGHT * sqrt(1.0 - 1.0 / (gamma0 * gamma0));
    double pscale = gamma0 * OR_M_P * v0;
    double perp = sqrt(fmax(0.0, 1.0 - mu0 * mu0));
    double lo[3] = {g->xmin, g->ymin, g->zmin}, len[3], fixed[3];
    double hi[3] = {g->xmax, g->ymax, g->zmax};
    uint64_t key = or_mix64(seed);
    int64_t bad = 0;
    for (int d = 0; d < 3; ++d) {
        len[d] = hi[d] - lo[d];
        fixed[d] = lo[d] + position[d] * (hi[d] - lo[d]);
    }
    for (int64_t i = 0; i < n; ++i) {
        double x[3], ux, uy, uz;
        for (int d = 0; d < 3; ++d) x[d] = random_pos ? or_draw(key, i, d) * len[d] + lo[d] : fixed[d];
        if (fixed_mu) {
            double bx = or_trilinear(bfield[0], x[0], x[1], x[2], g);
            double by = or_trilinear(bfield[1], x[0], x[1], x[2], g);
            double bz = or_trilinear(bfield[2], x[0], x[1], x[2], g);
            double bn = sqrt(bx * bx + by * by + bz * bz);
            if (!isfinite(bn) || bn == 0.0) {
                ++bad;
                ux = uy = uz = NAN;
            } else {
                double bhx = bx / bn, bhy = by / bn, bhz = bz / bn, e1x, e1y, e1z;
                if (fabs(bhx) < 0.9) {
                    e1x = 0.0; e1y = bhz; e1z = -bhy;
                } else {
                    e1x = -bhz; e1y = 0.0; e1z = bhx;
                }
                double e1n = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
                e1x = e1x / e1n; e1y = e1y / e1n; e1z = e1z / e1n;
                double e2x = bhy * e1z - bhz * e1y;
                double e2y = bhz * e1x - bhx * e1z;
                double e2z = bhx * e1y - bhy * e1x;
                double phi = two_pi * or_draw(key, i, 3);
                double cphi = cos(phi), sphi = sin(phi);
                ux = mu0 * bhx + perp * (cphi * e1x + sphi * e2x);
                uy = mu0 * bhy + perp * (cphi * e1y + sphi * e2y);
                uz = mu0 * bhz + perp * (cphi * e1z + sphi * e2z);
            }
        } else {
            double z = 2.0 * or_draw(key, i, 3) - 1.0;
            double phi = two_pi * or_draw(key, i, 4);
            double r = sqrt(fmax(0.0, 1.0 - z * z));
            ux = r * cos(phi);
            uy = r * sin(phi);
            uz = z;
        }
        x1[i] = x[0]; x2[i] = x[1]; x3[i] = x[2];
        p1[i] = pscale * ux; p2[i] = pscale * uy; p3[i] = pscale * uz;
    }
    return bad;
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
