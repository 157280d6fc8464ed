// Plain (parity) form of the push and the phase-space mu reconstruction.
//
// This translation unit is compiled with --fmad=false: every expression keeps
// the reference's evaluation order (Julia: a*b*c == (a*b)*c, x^2 == x*x, no
// FMA contraction), division and sqrt are IEEE round-to-nearest, so the FP64
// results are bit-identical to a Float64 run of the reference on the same
// inputs.
#include "exact_mu.cuh"
#include "pt_internal.cuh"

namespace pt {
namespace {

using namespace exact;

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
    const R* P = pos + s * 3 * chunk + p;
    const R* M = mom + s * 3 * chunk + p;
    const R* B[3] = {bx, by, bz};
    mu_out[p * nsave + s] = phase_space_mu<R>(P[0], P[chunk], P[2 * chunk], M[0], M[chunk], M[2 * chunk], B, g);
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
