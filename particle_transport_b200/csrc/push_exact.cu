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

// Cache write of one save row at the pre-push state (column q of row r):
// the mu row (reconstruct_mu_step_kernel!,
// src/multimode_multienergy_cache_pipeline.jl:1349-1374, reusing the B
// sample of the push) or the phase-space row.
__device__ __forceinline__ void exact_save(const pt_grid& g, int cache_mode, int cache_f64, void* cache, int64_t ncol,
                                           int64_t r, int64_t q, bool al, double xx, double yy, double zz, double px,
                                           double py, double pz, double bx, double by, double bz)
{
    if (cache_mode == PT_CACHE_MU) {
        double mu = NAN;
        if (al && !(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) && g.xmin <= xx &&
            xx <= g.xmax && g.ymin <= yy && yy <= g.ymax && g.zmin <= zz && zz <= g.zmax)
            mu = pitch_mu<double>(px, py, pz, bx, by, bz);
        if (cache_f64) ((double*)cache)[r * ncol + q] = mu;
        else ((float*)cache)[r * ncol + q] = (float)mu;
    } else {
        double v[6] = {xx, yy, zz, px, py, pz};
        for (int k = 0; k < 6; ++k) {
            double w = al ? v[k] : (double)NAN;
            int64_t idx = (r * 6 + k) * ncol + q;
            if (cache_f64) ((double*)cache)[idx] = w;
            else ((float*)cache)[idx] = (float)w;
        }
    }
}

// boris_push (src/phase_space_gpu_runner.jl:282-323) with E = -(u x B)
// (:365-368), the drift and the boundary (:370-387), in place.
__device__ __forceinline__ void exact_push_step(double& xx, double& yy, double& zz, double& px, double& py,
                                                double& pz, bool& al, double bx, double by, double bz, double vfx,
                                                double vfy, double vfz, const pt_grid& g, double dt, int periodic,
                                                int64_t* deaths, int64_t s)
{
    const double qm = Q_E, mp = M_P, cl = C_LIGHT;
    const double half = dt / 2.0;
    const double mc2 = (mp * mp) * (cl * cl);
    double ex = -(vfy * bz - vfz * by);
    double ey = -(vfz * bx - vfx * bz);
    double ez = -(vfx * by - vfy * bx);
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
    if (periodic) {
        xx = wrap(xx, g.xmin, g.xmax);
        yy = wrap(yy, g.ymin, g.ymax);
        zz = wrap(zz, g.zmin, g.zmax);
    } else if (xx < g.xmin || xx > g.xmax || yy < g.ymin || yy > g.ymax || zz < g.zmin || zz > g.zmax) {
        al = false;
        if (deaths) atomicAdd((unsigned long long*)&deaths[s], 1ull);
    }
}

// One thread = one particle, step_count steps with the state in registers.
// advance_particles_kernel! (src/phase_space_gpu_runner.jl:330-391): at a
// save step the pre-push state is cached, then the particle is pushed.
__global__ void __launch_bounds__(256) push_ref_kernel(PushArgsRef a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const pt_grid g = a.g;
    const int64_t sy = g.nx, sz = g.nx * g.ny;
    double xx = a.x[0][p], yy = a.x[1][p], zz = a.x[2][p];
    double px = a.p[0][p], py = a.p[1][p], pz = a.p[2][p];
    bool al = a.alive[p] != 0;
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
        if (is_save)
            exact_save(g, a.cache_mode, a.cache_f64, a.cache, a.n, row - a.row_base, p, al, xx, yy, zz, px, py, pz,
                       bx, by, bz);
        if (al && do_push) {
            const double vfx = sample(a.f[3], c, sy, sz);
            const double vfy = sample(a.f[4], c, sy, sz);
            const double vfz = sample(a.f[5], c, sy, sz);
            exact_push_step(xx, yy, zz, px, py, pz, al, bx, by, bz, vfx, vfy, vfz, g, a.dt, a.periodic, a.deaths, s);
        }
    }
    a.x[0][p] = xx; a.x[1][p] = yy; a.x[2][p] = zz;
    a.p[0][p] = px; a.p[1][p] = py; a.p[2][p] = pz;
    a.alive[p] = al ? 1 : 0;
}

// Head record (Bx, By, Bz, ux) of an FP64 node: one 256-bit read-only load
// (32-byte aligned).
__device__ __forceinline__ double4 ld_node_head(const double* r)
{
    uint32_t w[8];
    asm volatile("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(r));
    return make_double4(__hiloint2double((int)w[1], (int)w[0]), __hiloint2double((int)w[3], (int)w[2]),
                        __hiloint2double((int)w[5], (int)w[4]), __hiloint2double((int)w[7], (int)w[6]));
}

// push_ref_kernel over a BRICK_F64 field: the 8 corners of the cell are
// node records (ox[i] + oy[j] + oz[k] in the Morton brick order) in a head
// plane (Bx, By, Bz, ux) and a tail plane (uy, uz); each
// component is interpolated by the lerps of sample() in the same order, so
// every value equals the reference-layout kernel's.  Slots may be in brick
// order; the cache column of slot p is pid[p].
__global__ void __launch_bounds__(256) push_exact_brick_kernel(PushArgsExactBrick a)
{
    extern __shared__ uint32_t s_offs[];
    const pt_grid g = a.g;
    const int nx = (int)g.nx, ny = (int)g.ny, nz = (int)g.nz;
    for (int i = threadIdx.x; i < nx + ny + nz; i += blockDim.x) s_offs[i] = a.offs[i];
    __syncthreads();
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const uint32_t* ox = s_offs;
    const uint32_t* oy = s_offs + nx;
    const uint32_t* oz = s_offs + nx + ny;
    const double* N = (const double*)a.nodes;
    const double2* T = (const double2*)a.tail;
    const int64_t q = a.pid ? (int64_t)a.pid[p] : p;
    double xx = a.x[0][p], yy = a.x[1][p], zz = a.x[2][p];
    double px = a.p[0][p], py = a.p[1][p], pz = a.p[2][p];
    bool al = a.alive[p] != 0;
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
        double bx = 0, by = 0, bz = 0, vfx = 0, vfy = 0, vfz = 0;
        const bool need_mu = is_save && a.cache_mode == PT_CACHE_MU;
        if (al && (do_push || need_mu)) {
            const Cell3<double> c = locate3<double>(xx, yy, zz, g.xmin, g.ymin, g.zmin, g.dx, g.dy, g.dz, g.nx, g.ny,
                                                    g.nz);
            const uint32_t x0 = ox[c.i], x1 = ox[c.i + 1], y0 = oy[c.j], y1 = oy[c.j + 1], z0 = oz[c.k],
                           z1 = oz[c.k + 1];
            const uint32_t nd[8] = {x0 + y0 + z0, x1 + y0 + z0, x0 + y1 + z0, x1 + y1 + z0,
                                    x0 + y0 + z1, x1 + y0 + z1, x0 + y1 + z1, x1 + y1 + z1};
            double4 h[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) h[k] = ld_node_head(N + 4 * (size_t)nd[k]);
            bx = lerp8(h[0].x, h[1].x, h[2].x, h[3].x, h[4].x, h[5].x, h[6].x, h[7].x, c.t);
            by = lerp8(h[0].y, h[1].y, h[2].y, h[3].y, h[4].y, h[5].y, h[6].y, h[7].y, c.t);
            bz = lerp8(h[0].z, h[1].z, h[2].z, h[3].z, h[4].z, h[5].z, h[6].z, h[7].z, c.t);
            if (do_push) {
                double2 u[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) u[k] = __ldg(T + nd[k]);
                vfx = lerp8(h[0].w, h[1].w, h[2].w, h[3].w, h[4].w, h[5].w, h[6].w, h[7].w, c.t);
                vfy = lerp8(u[0].x, u[1].x, u[2].x, u[3].x, u[4].x, u[5].x, u[6].x, u[7].x, c.t);
                vfz = lerp8(u[0].y, u[1].y, u[2].y, u[3].y, u[4].y, u[5].y, u[6].y, u[7].y, c.t);
            }
        }
        if (is_save)
            exact_save(g, a.cache_mode, a.cache_f64, a.cache, a.n, row - a.row_base, q, al, xx, yy, zz, px, py, pz,
                       bx, by, bz);
        if (al && do_push)
            exact_push_step(xx, yy, zz, px, py, pz, al, bx, by, bz, vfx, vfy, vfz, g, a.dt, a.periodic, a.deaths, s);
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

int launch_push_exact_brick(const PushArgsExactBrick& a, cudaStream_t s)
{
    if (a.n <= 0 || a.step_count <= 0) return PT_OK;
    const int threads = 256;
    const int64_t blocks = (a.n + threads - 1) / threads;
    const size_t smem = sizeof(uint32_t) * (size_t)(a.g.nx + a.g.ny + a.g.nz);
    if (smem > 48 * 1024)
        PT_CUDA(cudaFuncSetAttribute(push_exact_brick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    push_exact_brick_kernel<<<(unsigned)blocks, threads, smem, s>>>(a);
    PT_CHECK_LAUNCH("push_exact_brick_kernel");
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
