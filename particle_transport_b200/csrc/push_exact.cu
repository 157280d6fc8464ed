// Plain (parity) form of the push and the phase-space mu reconstruction.
//
// This translation unit is compiled with --fmad=false: every expression keeps
// the reference's evaluation order (Julia: a*b*c == (a*b)*c, x^2 == x*x, no
// FMA contraction), division and sqrt are IEEE round-to-nearest, so the FP64
// results are bit-identical to a Float64 run of the reference on the same
// inputs.
#include "pt_internal.cuh"

namespace pt {
namespace {

// clamp(floor(Int, f), 1, n - 1) as a double (NaN -> 1).
// src/phase_space_gpu_runner.jl:252-254
template <typename R>
__device__ __forceinline__ double cell_index(R f, int64_t n)
{
    double c = floor((double)f);
    double hi = (double)(n - 1);
    if (!(c >= 1.0)) c = 1.0;
    if (c > hi) c = hi;
    return c;
}

// Cell location of one position, shared by all components sampled there.
template <typename R>
struct Cell {
    int64_t base;  // 0-based linear index of corner (i0, j0, k0)
    R tx, ty, tz;
};

template <typename R>
__device__ __forceinline__ Cell<R> locate(R x, R y, R z, R xmin, R ymin, R zmin, R dx, R dy, R dz, int64_t nx,
                                          int64_t ny, int64_t nz)
{
    // trilinear_sample, src/phase_space_gpu_runner.jl:247-258
    R fx = (x - xmin) / dx + R(1);
    R fy = (y - ymin) / dy + R(1);
    R fz = (z - zmin) / dz + R(1);
    double ci = cell_index(fx, nx), cj = cell_index(fy, ny), ck = cell_index(fz, nz);
    Cell<R> c;
    c.tx = fx - (R)ci;
    c.ty = fy - (R)cj;
    c.tz = fz - (R)ck;
    c.base = ((int64_t)ci - 1) + nx * (((int64_t)cj - 1) + ny * ((int64_t)ck - 1));
    return c;
}

// src/phase_space_gpu_runner.jl:260-275
template <typename R>
__device__ __forceinline__ R sample(const R* __restrict__ arr, const Cell<R>& c, int64_t sy, int64_t sz)
{
    const R* b = arr + c.base;
    R c000 = __ldg(b), c100 = __ldg(b + 1), c010 = __ldg(b + sy), c110 = __ldg(b + 1 + sy);
    R c001 = __ldg(b + sz), c101 = __ldg(b + 1 + sz), c011 = __ldg(b + sy + sz), c111 = __ldg(b + 1 + sy + sz);
    R c00 = c000 * (R(1) - c.tx) + c100 * c.tx;
    R c10 = c010 * (R(1) - c.tx) + c110 * c.tx;
    R c01 = c001 * (R(1) - c.tx) + c101 * c.tx;
    R c11 = c011 * (R(1) - c.tx) + c111 * c.tx;
    R c0 = c00 * (R(1) - c.ty) + c10 * c.ty;
    R c1 = c01 * (R(1) - c.ty) + c11 * c.ty;
    return c0 * (R(1) - c.tz) + c1 * c.tz;
}

// pitch_mu_from_pB, src/compute_delta_mu2_curve.jl:93-110
template <typename R>
__device__ __forceinline__ R pitch_mu(R px, R py, R pz, R bx, R by, R bz)
{
    R pn = sqrt(px * px + py * py + pz * pz);
    R bn = sqrt(bx * bx + by * by + bz * bz);
    if (!isfinite(pn) || !isfinite(bn) || pn == R(0) || bn == R(0)) return R(NAN);
    R mu = (px * bx + py * by + pz * bz) / (pn * bn);
    return mu > R(1) ? R(1) : (mu < R(-1) ? R(-1) : mu);
}

__device__ __forceinline__ double wrap(double x, double xmin, double xmax)
{
    // src/phase_space_gpu_runner.jl:325-328
    double width = xmax - xmin;
    return x - floor((x - xmin) / width) * width;
}

// One thread = one particle, step_count steps with the state in registers.
// advance_particles_kernel! (src/phase_space_gpu_runner.jl:330-391) with
// boris_push (:282-323) and, at save steps, reconstruct_mu_step_kernel!
// (src/multimode_multienergy_cache_pipeline.jl:1349-1374) on the pre-push
// state, reusing the B sample of the push.
__global__ void __launch_bounds__(256) push_ref_kernel(PushArgsRef a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const pt_grid g = a.g;
    const int64_t sy = g.nx, sz = g.nx * g.ny;
    double xx = a.x[0][p], yy = a.x[1][p], zz = a.x[2][p];
    double px = a.p[0][p], py = a.p[1][p], pz = a.p[2][p];
    bool al = a.alive[p] != 0;

    const double qm = Q_E, mp = M_P, cl = C_LIGHT;
    const double dt = a.dt;
    const double half = dt / 2.0;
    const double mc2 = (mp * mp) * (cl * cl);

    const int64_t s_end = a.step_begin + a.step_count;
    int64_t next_save = ((a.step_begin + a.stride - 1) / a.stride) * a.stride;
    for (int64_t s = a.step_begin; s < s_end; ++s) {
        const bool do_push = s < a.nsteps - 1;
        bool is_save = false;
        int64_t row = 0;
        if (s == next_save) {
            row = s / a.stride;
            next_save += a.stride;
            is_save = a.cache_mode != PT_CACHE_NONE && row >= a.row_base && row < a.row_base + a.rows;
        }
        double bx = 0, by = 0, bz = 0;
        Cell<double> c{};
        const bool need_mu = is_save && a.cache_mode == PT_CACHE_MU;
        if (al && (do_push || need_mu)) {
            c = locate<double>(xx, yy, zz, g.xmin, g.ymin, g.zmin, g.dx, g.dy, g.dz, g.nx, g.ny, g.nz);
            bx = sample(a.f[0], c, sy, sz);
            by = sample(a.f[1], c, sy, sz);
            bz = sample(a.f[2], c, sy, sz);
        }
        if (is_save) {
            const int64_t r = row - a.row_base;
            if (a.cache_mode == PT_CACHE_MU) {
                double mu = NAN;
                if (al && !(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) &&
                    g.xmin <= xx && xx <= g.xmax && g.ymin <= yy && yy <= g.ymax && g.zmin <= zz && zz <= g.zmax)
                    mu = pitch_mu<double>(px, py, pz, bx, by, bz);
                if (a.cache_f64) ((double*)a.cache)[r * a.n + p] = mu;
                else ((float*)a.cache)[r * a.n + p] = (float)mu;
            } else {
                double v[6] = {xx, yy, zz, px, py, pz};
                for (int k = 0; k < 6; ++k) {
                    double w = al ? v[k] : (double)NAN;
                    int64_t idx = (r * 6 + k) * a.n + p;
                    if (a.cache_f64) ((double*)a.cache)[idx] = w;
                    else ((float*)a.cache)[idx] = (float)w;
                }
            }
        }
        if (al && do_push) {
            double vfx = sample(a.f[3], c, sy, sz);
            double vfy = sample(a.f[4], c, sy, sz);
            double vfz = sample(a.f[5], c, sy, sz);
            // E = -(u x B): src/phase_space_gpu_runner.jl:365-368
            double ex = -(vfy * bz - vfz * by);
            double ey = -(vfz * bx - vfx * bz);
            double ez = -(vfx * by - vfy * bx);
            // boris_push
            double pmx = px + qm * ex * half;
            double pmy = py + qm * ey * half;
            double pmz = pz + qm * ez * half;
            double gamma_minus = sqrt(1.0 + (pmx * pmx + pmy * pmy + pmz * pmz) / mc2);
            double tx = qm * bx * dt / (2.0 * mp * gamma_minus);
            double ty = qm * by * dt / (2.0 * mp * gamma_minus);
            double tz = qm * bz * dt / (2.0 * mp * gamma_minus);
            double t2 = tx * tx + ty * ty + tz * tz;
            double sxx = 2.0 * tx / (1.0 + t2);
            double syy = 2.0 * ty / (1.0 + t2);
            double szz = 2.0 * tz / (1.0 + t2);
            double ppx = pmx + (pmy * tz - pmz * ty);
            double ppy = pmy + (pmz * tx - pmx * tz);
            double ppz = pmz + (pmx * ty - pmy * tx);
            double ppx2 = pmx + (ppy * szz - ppz * syy);
            double ppy2 = pmy + (ppz * sxx - ppx * szz);
            double ppz2 = pmz + (ppx * syy - ppy * sxx);
            double pxn = ppx2 + qm * ex * half;
            double pyn = ppy2 + qm * ey * half;
            double pzn = ppz2 + qm * ez * half;
            double gamma_new = sqrt(1.0 + (pxn * pxn + pyn * pyn + pzn * pzn) / mc2);
            double vxn = pxn / (gamma_new * mp);
            double vyn = pyn / (gamma_new * mp);
            double vzn = pzn / (gamma_new * mp);
            px = pxn; py = pyn; pz = pzn;
            xx = xx + vxn * dt; yy = yy + vyn * dt; zz = zz + vzn * dt;
            if (a.periodic) {
                xx = wrap(xx, g.xmin, g.xmax);
                yy = wrap(yy, g.ymin, g.ymax);
                zz = wrap(zz, g.zmin, g.zmax);
            } else if (xx < g.xmin || xx > g.xmax || yy < g.ymin || yy > g.ymax || zz < g.zmin || zz > g.zmax) {
                al = false;
                if (a.deaths) atomicAdd((unsigned long long*)&a.deaths[s], 1ull);
            }
        }
    }
    a.x[0][p] = xx; a.x[1][p] = yy; a.x[2][p] = zz;
    a.p[0][p] = px; a.p[1][p] = py; a.p[2][p] = pz;
    a.alive[p] = al ? 1 : 0;
}

// reconstruct_mu_kernel!, src/compute_delta_mu2_curve.jl:151-184, at the
// compute precision R.  Thread index runs particle-fastest so that the
// phase-space reads coalesce; mu_out is Julia (nsave, chunk) = [p][s].
template <typename R>
__global__ void __launch_bounds__(256) reconstruct_mu_kernel(const R* __restrict__ pos, const R* __restrict__ mom,
                                                             int64_t chunk, int64_t nsave, const R* __restrict__ bx,
                                                             const R* __restrict__ by, const R* __restrict__ bz,
                                                             pt_grid g, R* __restrict__ mu_out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= chunk * nsave) return;
    const int64_t p = t % chunk, s = t / chunk;
    const R xmin = (R)g.xmin, ymin = (R)g.ymin, zmin = (R)g.zmin;
    const R xmax = (R)g.xmax, ymax = (R)g.ymax, zmax = (R)g.zmax;
    const R dx = (R)g.dx, dy = (R)g.dy, dz = (R)g.dz;
    const R* P = pos + s * 3 * chunk + p;
    const R* M = mom + s * 3 * chunk + p;
    R xx = P[0], yy = P[chunk], zz = P[2 * chunk];
    R px = M[0], py = M[chunk], pz = M[2 * chunk];
    R v = R(NAN);
    if (!(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) && xmin <= xx &&
        xx <= xmax && ymin <= yy && yy <= ymax && zmin <= zz && zz <= zmax) {
        Cell<R> c = locate<R>(xx, yy, zz, xmin, ymin, zmin, dx, dy, dz, g.nx, g.ny, g.nz);
        const int64_t sy = g.nx, sz = g.nx * g.ny;
        R b0 = sample(bx, c, sy, sz), b1 = sample(by, c, sy, sz), b2 = sample(bz, c, sy, sz);
        v = pitch_mu<R>(px, py, pz, b0, b1, b2);
    }
    mu_out[p * nsave + s] = v;
}

}  // namespace

int launch_push_ref(const PushArgsRef& a, cudaStream_t s)
{
    if (a.n <= 0 || a.step_count <= 0) return PT_OK;
    const int threads = 256;
    const int64_t blocks = (a.n + threads - 1) / threads;
    push_ref_kernel<<<(unsigned)blocks, threads, 0, s>>>(a);
    PT_CHECK_LAUNCH("push_ref_kernel");
    return PT_OK;
}

int launch_reconstruct_mu(const void* pos, const void* mom, int64_t chunk, int64_t nsave, const void* const b[3],
                          const pt_grid& g, int f64, void* mu_out, cudaStream_t s)
{
    const int64_t total = chunk * nsave;
    if (total <= 0) return PT_OK;
    const int threads = 256;
    const int64_t blocks = (total + threads - 1) / threads;
    if (f64)
        reconstruct_mu_kernel<double><<<(unsigned)blocks, threads, 0, s>>>(
            (const double*)pos, (const double*)mom, chunk, nsave, (const double*)b[0], (const double*)b[1],
            (const double*)b[2], g, (double*)mu_out);
    else
        reconstruct_mu_kernel<float><<<(unsigned)blocks, threads, 0, s>>>(
            (const float*)pos, (const float*)mom, chunk, nsave, (const float*)b[0], (const float*)b[1],
            (const float*)b[2], g, (float*)mu_out);
    PT_CHECK_LAUNCH("reconstruct_mu_kernel");
    return PT_OK;
}

}  // namespace pt
