// Mixed-precision form of the push (the reference's advance_particles_kernel!,
// src/phase_space_gpu_runner.jl:330-391, restated in nondimensional units).
//
// Units: positions in cells, x~ = (x - xmin)/dx (carried in FP64);
// momentum p~ = p/(m c) in FP32 with |p~|^2 carried in FP64; B~ = B/B_ref and
// u~ = u/c stored in Morton-ordered 8^3 bricks with the six components of a
// node interleaved (BF16: one 16-byte load per corner; FP32: two).
// With h = q B_ref dt/(2m) the Boris step of boris_push (:282-323) becomes
//   eps = -(u~ x h B~)           (= q E dt/(2 m c))
//   p-  = p~ + eps,   g- = sqrt(1 + |p-|^2)
//   t   = h B~ / g-,  s = 2 t/(1 + t.t)
//   p+  = p- + (p- + p- x t) x s,  rescaled to |p+| = |p-| (the rotation is
//         norm-preserving; the scale is taken from the FP64 |p|^2)
//   p~' = p+ + eps,   x~ += p~' (c dt/dx) / g'
// and |p|^2 is advanced in FP64 by the two E kicks only, so with E = 0 the
// particle energy is conserved to FP64 rounding.
#include "pt_internal.cuh"

namespace pt {
namespace {

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

struct Corners {
    uint32_t idx[8];
    float w[8];
};

// Corner node indices and trilinear weights of the cell holding (x, y, z)
// (cell units).  Cell = clamp(floor(x), 0, n-2) as in trilinear_sample
// (src/phase_space_gpu_runner.jl:247-258, 0-based).
__device__ __forceinline__ Corners locate_brick(double x, double y, double z, const uint32_t* ox, const uint32_t* oy,
                                                const uint32_t* oz, int nx, int ny, int nz)
{
    int ix = (int)floor(x), iy = (int)floor(y), iz = (int)floor(z);
    ix = min(max(ix, 0), nx - 2);
    iy = min(max(iy, 0), ny - 2);
    iz = min(max(iz, 0), nz - 2);
    float tx = (float)(x - (double)ix), ty = (float)(y - (double)iy), tz = (float)(z - (double)iz);
    uint32_t x0 = ox[ix], x1 = ox[ix + 1], y0 = oy[iy], y1 = oy[iy + 1], z0 = oz[iz], z1 = oz[iz + 1];
    Corners c;
    c.idx[0] = x0 + y0 + z0; c.idx[1] = x1 + y0 + z0; c.idx[2] = x0 + y1 + z0; c.idx[3] = x1 + y1 + z0;
    c.idx[4] = x0 + y0 + z1; c.idx[5] = x1 + y0 + z1; c.idx[6] = x0 + y1 + z1; c.idx[7] = x1 + y1 + z1;
    float ux = 1.0f - tx, uy = 1.0f - ty, uz = 1.0f - tz;
    float a00 = ux * uy, a10 = tx * uy, a01 = ux * ty, a11 = tx * ty;
    c.w[0] = a00 * uz; c.w[1] = a10 * uz; c.w[2] = a01 * uz; c.w[3] = a11 * uz;
    c.w[4] = a00 * tz; c.w[5] = a10 * tz; c.w[6] = a01 * tz; c.w[7] = a11 * tz;
    return c;
}

// 32-byte read-only load (sm_100 256-bit vector load; the address is 32-byte aligned)
__device__ __forceinline__ void ldg256(const void* p, uint32_t w[8])
{
    asm volatile("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(p));
}

__device__ __forceinline__ void acc_bf16x3(float f[6], float w, uint32_t a, uint32_t b, uint32_t c)
{
    f[0] = fmaf(w, bf_lo(a), f[0]);
    f[1] = fmaf(w, bf_hi(a), f[1]);
    f[2] = fmaf(w, bf_lo(b), f[2]);
    f[3] = fmaf(w, bf_hi(b), f[3]);
    f[4] = fmaf(w, bf_lo(c), f[4]);
    f[5] = fmaf(w, bf_hi(c), f[5]);
}

// Interpolate the six components at a cell: 8 weighted corners.
//  LAYOUT_BF16        16-byte node (Bx,By | Bz,ux | uy,uz | pad), 8 x 16-byte loads
//  LAYOUT_F32         32-byte node (Bx,By,Bz,ux,uy,uz,pad,pad), 8 x 32-byte loads
//  LAYOUT_BF16_XPAIR  32-byte record = node (i) + node (i+1), 4 x 32-byte loads
// TEXC (BF16 only): the odd corners -- TEXC of them -- are fetched through the
// texture path (tex1Dfetch on the same records), the others with LDG: the two
// L1TEX data pipes share the gathers.  Same values, same summation order.
template <int LAYOUT, int TEXC = 0>
__device__ __forceinline__ void gather6(const void* __restrict__ nodes, cudaTextureObject_t tex, const Corners& c,
                                        float f[6])
{
    // adds the weighted corners to f (which holds 0, or the BF16 forms' mean field)
    if (LAYOUT == LAYOUT_F32) {
        const char* N = (const char*)nodes;
        uint32_t v[8][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) ldg256(N + 32 * (size_t)c.idx[q], v[q]);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float w = c.w[q];
#pragma unroll
            for (int k = 0; k < 6; ++k) f[k] = fmaf(w, __uint_as_float(v[q][k]), f[k]);
        }
        return;
    }
    if (LAYOUT == LAYOUT_BF16_XPAIR) {
        const char* N = (const char*)nodes;
        uint32_t v[4][8];
#pragma unroll
        for (int q = 0; q < 4; ++q) ldg256(N + 32 * (size_t)c.idx[2 * q], v[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            acc_bf16x3(f, c.w[2 * q], v[q][0], v[q][1], v[q][2]);
            acc_bf16x3(f, c.w[2 * q + 1], v[q][3], v[q][4], v[q][5]);
        }
        return;
    }
    {
        const uint4* N = (const uint4*)nodes;
        uint4 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const bool via_tex = TEXC == 8 || (TEXC == 4 && (q & 1));
            if (via_tex) v[q] = tex1Dfetch<uint4>(tex, (int)c.idx[q]);
            else v[q] = __ldg(N + c.idx[q]);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float w = c.w[q];
            f[0] = fmaf(w, bf_lo(v[q].x), f[0]);
            f[1] = fmaf(w, bf_hi(v[q].x), f[1]);
            f[2] = fmaf(w, bf_lo(v[q].y), f[2]);
            f[3] = fmaf(w, bf_hi(v[q].y), f[3]);
            f[4] = fmaf(w, bf_lo(v[q].z), f[4]);
            f[5] = fmaf(w, bf_hi(v[q].z), f[5]);
        }
    }
}

__device__ __forceinline__ float mu_f32(float px, float py, float pz, float bx, float by, float bz)
{
    // pitch_mu_from_pB, src/compute_delta_mu2_curve.jl:101-110 (FP32)
    float pn = sqrtf(px * px + py * py + pz * pz);
    float bn = sqrtf(bx * bx + by * by + bz * bz);
    if (!isfinite(pn) || !isfinite(bn) || pn == 0.0f || bn == 0.0f) return NAN;
    float mu = (px * bx + py * by + pz * bz) / (pn * bn);
    return fminf(1.0f, fmaxf(-1.0f, mu));
}

__device__ __forceinline__ double wrap_cells(double x, double w)
{
    // wrap_periodic_coordinate (src/phase_space_gpu_runner.jl:325-328) in cell units
    if (x < 0.0 || x >= w) x -= floor(x / w) * w;
    return x;
}

// K steps of one particle held in registers.  State is (x, y, z) in cells
// (FP64), p/(mc) (FP32) and |p/(mc)|^2 (FP64); pid indexes the cache row.
// Cache rows of a.n_cache particles: row r at (r - a.row_base) or, with
// a.ring, at (r % a.rows).
template <int LAYOUT, int TEXC = 0>
__device__ __forceinline__ void advance_particle(double& x, double& y, double& z, float& px, float& py, float& pz,
                                                 double& P2, bool& al, const int64_t pid, const PushArgsFast& a,
                                                 const uint32_t* ox, const uint32_t* oy, const uint32_t* oz,
                                                 const int64_t s_begin, const int64_t s_end)
{
    const int nx = (int)a.fld.nx, ny = (int)a.fld.ny, nz = (int)a.fld.nz;
    const float hB = a.hB;
    const int64_t n = a.n_cache;
    {
        int64_t next_save = ((s_begin + a.stride - 1) / a.stride) * a.stride;
        for (int64_t s = s_begin; s < s_end; ++s) {
            const bool do_push = s < a.nsteps - 1;
            bool is_save = false;
            int64_t row = 0;
            if (s == next_save) {
                row = s / a.stride;
                next_save += a.stride;
                is_save = a.cache_mode != PT_CACHE_NONE &&
                          (a.ring || (row >= a.row_base && row < a.row_base + a.rows));
            }
            float f[6] = {0, 0, 0, 0, 0, 0};
            if (al && (do_push || (is_save && a.cache_mode == PT_CACHE_MU))) {
                Corners c = locate_brick(x, y, z, ox, oy, oz, nx, ny, nz);
                if (LAYOUT == LAYOUT_BF16 || LAYOUT == LAYOUT_BF16_XPAIR) {
                    // the BF16 nodes hold B - <B>: the weights sum to 1, so the
                    // mean enters once, as the start of the weighted sum
                    f[0] = a.fld.boff[0];
                    f[1] = a.fld.boff[1];
                    f[2] = a.fld.boff[2];
                }
                gather6<LAYOUT, TEXC>(a.fld.nodes, a.fld.tex, c, f);
            }
            if (is_save) {
                const int64_t r = a.ring ? row % a.rows : row - a.row_base;
                if (a.cache_mode == PT_CACHE_MU) {
                    float mu = NAN;
                    if (al && x >= 0.0 && x <= a.wx && y >= 0.0 && y <= a.wy && z >= 0.0 && z <= a.wz)
                        mu = mu_f32(px, py, pz, f[0], f[1], f[2]);
                    // rows: save r of every particle in one row; time-fastest
                    // (pitch > 0): a particle's saves side by side, so the 8
                    // saves of a launch, written by this thread while it holds
                    // the particle (~0.1 ms of a 64-step launch at 16.7M
                    // particles), merge in L2 into one whole DRAM sector
                    const int64_t at = a.pitch > 0 ? pid * a.pitch + r : r * n + pid;
                    if (a.cache_f64) ((double*)a.cache)[at] = (double)mu;
                    else ((float*)a.cache)[at] = mu;
                    if (pid < a.n_mom) {
                        // momenta of the D_pp subset, as the phase-space writer stores them
                        const double pm = sqrt(P2) / sqrt((double)px * px + (double)py * py + (double)pz * pz) *
                                          (M_P * C_LIGHT);
                        float* M = a.mom_cache + r * 3 * a.n_mom + pid;
                        M[0] = al ? (float)((double)px * pm) : NAN;
                        M[a.n_mom] = al ? (float)((double)py * pm) : NAN;
                        M[2 * a.n_mom] = al ? (float)((double)pz * pm) : NAN;
                    }
                } else {
                    double v[6];
                    const double pm = sqrt(P2) / sqrt((double)px * px + (double)py * py + (double)pz * pz) *
                                      (M_P * C_LIGHT);
                    v[0] = a.xmin[0] + x * a.dxs[0];
                    v[1] = a.xmin[1] + y * a.dxs[1];
                    v[2] = a.xmin[2] + z * a.dxs[2];
                    v[3] = (double)px * pm; v[4] = (double)py * pm; v[5] = (double)pz * pm;
                    for (int k = 0; k < 6; ++k) {
                        double w = al ? v[k] : (double)NAN;
                        int64_t idx = (r * 6 + k) * n + pid;
                        if (a.cache_f64) ((double*)a.cache)[idx] = w;
                        else ((float*)a.cache)[idx] = (float)w;
                    }
                }
            }
            if (al && do_push) {
                const float bx = hB * f[0], by = hB * f[1], bz = hB * f[2];
                const float ux = f[3], uy = f[4], uz = f[5];
                // eps = -(u x hB) = q E dt / (2 m c)
                const float ex = -(uy * bz - uz * by);
                const float ey = -(uz * bx - ux * bz);
                const float ez = -(ux * by - uy * bx);
                const float pmx = px + ex, pmy = py + ey, pmz = pz + ez;
                const float e2 = ex * ex + ey * ey + ez * ez;
                const double P2m = P2 + (double)(2.0f * (px * ex + py * ey + pz * ez) + e2);
                const float gm = sqrtf(1.0f + (float)P2m);
                const float ig = 1.0f / gm;
                const float tx = bx * ig, ty = by * ig, tz = bz * ig;
                const float t2 = tx * tx + ty * ty + tz * tz;
                const float sf = 2.0f / (1.0f + t2);
                const float sx = sf * tx, sy = sf * ty, sz = sf * tz;
                const float qx = pmx + (pmy * tz - pmz * ty);
                const float qy = pmy + (pmz * tx - pmx * tz);
                const float qz = pmz + (pmx * ty - pmy * tx);
                float rx = pmx + (qy * sz - qz * sy);
                float ry = pmy + (qz * sx - qx * sz);
                float rz = pmz + (qx * sy - qy * sx);
                // norm-preserving rotation: pin |p+|^2 to the FP64 |p-|^2
                const float r2 = rx * rx + ry * ry + rz * rz;
                const float sc = sqrtf((float)P2m) * rsqrtf(r2);
                rx *= sc; ry *= sc; rz *= sc;
                px = rx + ex; py = ry + ey; pz = rz + ez;
                P2 = P2m + (double)(2.0f * (rx * ex + ry * ey + rz * ez) + e2);
                const float ign = rsqrtf(1.0f + (float)P2);
                x += (double)(px * (a.vfac[0] * ign));
                y += (double)(py * (a.vfac[1] * ign));
                z += (double)(pz * (a.vfac[2] * ign));
                if (a.periodic) {
                    x = wrap_cells(x, a.wx);
                    y = wrap_cells(y, a.wy);
                    z = wrap_cells(z, a.wz);
                } else if (x < 0.0 || x > a.wx || y < 0.0 || y > a.wy || z < 0.0 || z > a.wz) {
                    al = false;
                    if (a.deaths) atomicAdd((unsigned long long*)&a.deaths[s], 1ull);
                }
            }
        }
    }
}

template <int LAYOUT, int BLOCK, int MINB, int TEXC = 0>
__global__ void __launch_bounds__(BLOCK, MINB) push_fast_kernel(PushArgsFast a)
{
    extern __shared__ uint32_t s_offs[];
    const int nx = (int)a.fld.nx, ny = (int)a.fld.ny, nz = (int)a.fld.nz;
    for (int i = threadIdx.x; i < nx + ny + nz; i += blockDim.x) s_offs[i] = a.fld.offs[i];
    __syncthreads();
    const uint32_t* ox = s_offs;
    const uint32_t* oy = s_offs + nx;
    const uint32_t* oz = s_offs + nx + ny;
    const int64_t s_end = a.step_begin + a.step_count;
    const int64_t n = a.n;
    for (int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; slot < n;
         slot += (int64_t)gridDim.x * blockDim.x) {
        double x = a.x[slot], y = a.x[n + slot], z = a.x[2 * n + slot];
        float px = a.p[slot], py = a.p[n + slot], pz = a.p[2 * n + slot];
        double P2 = a.p2[slot];
        bool al = a.alive[slot] != 0;
        advance_particle<LAYOUT, TEXC>(x, y, z, px, py, pz, P2, al, a.pid[slot], a, ox, oy, oz, a.step_begin, s_end);
        a.x[slot] = x; a.x[n + slot] = y; a.x[2 * n + slot] = z;
        a.p[slot] = px; a.p[n + slot] = py; a.p[2 * n + slot] = pz;
        a.p2[slot] = P2;
        a.alive[slot] = al ? 1 : 0;
    }
}

// ------------------------------------------------------------ field bricks
__global__ void brick_convert_kernel(const double* __restrict__ bx, const double* __restrict__ by,
                                     const double* __restrict__ bz, const double* __restrict__ ux,
                                     const double* __restrict__ uy, const double* __restrict__ uz, int64_t nx,
                                     int64_t ny, int64_t nz, double inv_b, double inv_c, int layout, void* nodes,
                                     const uint32_t* __restrict__ offs, int64_t n_nodes, float o0, float o1, float o2)
{
    const int64_t total = nx * ny * nz;
    // B / B_ref less the stored mean-field offset (0 but for the BF16 forms)
    auto comps = [&](int64_t t, float v[6]) {
        v[0] = (float)(bx[t] * inv_b - (double)o0);
        v[1] = (float)(by[t] * inv_b - (double)o1);
        v[2] = (float)(bz[t] * inv_b - (double)o2);
        v[3] = (float)(ux[t] * inv_c); v[4] = (float)(uy[t] * inv_c); v[5] = (float)(uz[t] * inv_c);
    };
    auto pack3 = [](const float v[6], uint32_t w[3]) {
        for (int q = 0; q < 3; ++q) {
            const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(v[2 * q]));
            const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(v[2 * q + 1]));
            w[q] = lo | (hi << 16);
        }
    };
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t % nx, j = (t / nx) % ny, k = t / (nx * ny);
        const uint32_t node = offs[i] + offs[nx + j] + offs[nx + ny + k];
        if (layout == LAYOUT_F64) {
            // SI values as they are (the FP64 push reads them unchanged): the
            // head plane (Bx, By, Bz, ux), then the tail plane (uy, uz)
            ((double4*)nodes)[node] = make_double4(bx[t], by[t], bz[t], ux[t]);
            ((double2*)((double4*)nodes + n_nodes))[node] = make_double2(uy[t], uz[t]);
            continue;
        }
        float v[6];
        comps(t, v);
        if (layout == LAYOUT_BF16) {
            uint32_t w[3];
            pack3(v, w);
            ((uint4*)nodes)[node] = make_uint4(w[0], w[1], w[2], 0u);
        } else if (layout == LAYOUT_BF16_XPAIR) {
            uint32_t w[3], w2[3] = {0u, 0u, 0u};
            pack3(v, w);
            if (i + 1 < nx) {
                float v2[6];
                comps(t + 1, v2);
                pack3(v2, w2);
            }
            uint4* N = (uint4*)nodes;
            N[2 * (size_t)node] = make_uint4(w[0], w[1], w[2], w2[0]);
            N[2 * (size_t)node + 1] = make_uint4(w2[1], w2[2], 0u, 0u);
        } else {
            float4* N = (float4*)nodes;
            N[2 * (size_t)node] = make_float4(v[0], v[1], v[2], v[3]);
            N[2 * (size_t)node + 1] = make_float4(v[4], v[5], 0.0f, 0.0f);
        }
    }
}

// ------------------------------------------------------------ state import / export
__global__ void fast_import_kernel(const double* __restrict__ x1, const double* __restrict__ x2,
                                   const double* __restrict__ x3, const double* __restrict__ p1,
                                   const double* __restrict__ p2, const double* __restrict__ p3,
                                   const uint8_t* __restrict__ alive, int64_t n, double xmin, double ymin,
                                   double zmin, double dx, double dy, double dz, double* xo, float* po, double* p2o,
                                   int32_t* pid, uint8_t* ao)
{
    const double inv_mc = 1.0 / (M_P * C_LIGHT);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        xo[i] = (x1[i] - xmin) / dx;
        xo[n + i] = (x2[i] - ymin) / dy;
        xo[2 * n + i] = (x3[i] - zmin) / dz;
        const double qx = p1[i] * inv_mc, qy = p2[i] * inv_mc, qz = p3[i] * inv_mc;
        po[i] = (float)qx; po[n + i] = (float)qy; po[2 * n + i] = (float)qz;
        p2o[i] = qx * qx + qy * qy + qz * qz;
        pid[i] = (int32_t)i;
        ao[i] = alive[i];
    }
}

__global__ void fast_export_kernel(const double* __restrict__ xs, const float* __restrict__ ps,
                                   const double* __restrict__ p2s, const int32_t* __restrict__ pid,
                                   const uint8_t* __restrict__ as, int64_t n, double xmin, double ymin, double zmin,
                                   double dx, double dy, double dz, double* x1, double* x2, double* x3, double* p1,
                                   double* p2, double* p3, uint8_t* alive)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = pid[i];
        x1[q] = xmin + xs[i] * dx;
        x2[q] = ymin + xs[n + i] * dy;
        x3[q] = zmin + xs[2 * n + i] * dz;
        const double px = ps[i], py = ps[n + i], pz = ps[2 * n + i];
        const double sc = sqrt(p2s[i] / (px * px + py * py + pz * pz)) * (M_P * C_LIGHT);
        p1[q] = px * sc; p2[q] = py * sc; p3[q] = pz * sc;
        alive[q] = as[i];
    }
}

// ------------------------------------------------------------ brick sort
// One-digit radix (counting) sort of the particle slots by the brick that
// holds their cell; dead particles go to a final bucket.
// Histogram and scatter aggregate equal keys within a warp (__match_any_sync)
// so that runs of particles in one brick -- the common case once sorted --
// cost one atomic per warp instead of one per particle.  blockDim must be a
// multiple of 32 (every lane of a warp runs the same loop trips).
// sort bucket of a particle: the brick of its cell, dead_key when dead
__device__ __forceinline__ uint32_t brick_key(double x, double y, double z, uint8_t alive,
                                              const uint32_t* __restrict__ offs, int nx, int ny, int nz,
                                              uint32_t dead_key)
{
    if (!alive) return dead_key;
    const int ix = min(max((int)floor(x), 0), nx - 2);
    const int iy = min(max((int)floor(y), 0), ny - 2);
    const int iz = min(max((int)floor(z), 0), nz - 2);
    return (offs[ix] + offs[nx + iy] + offs[nx + ny + iz]) >> 9;
}

__global__ void sort_key_kernel(const double* __restrict__ xs, const uint8_t* __restrict__ as, int64_t n,
                                const uint32_t* __restrict__ offs, int nx, int ny, int nz, uint32_t dead_key,
                                uint32_t* __restrict__ hist)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t key =
            valid ? brick_key(xs[i], xs[n + i], xs[2 * n + i], as[i], offs, nx, ny, nz, dead_key) : dead_key;
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned same = __match_any_sync(act, key);
            if ((same & lt) == 0) atomicAdd(&hist[key], (uint32_t)__popc(same));
        }
    }
}

// Exclusive scan of hist[0..m) in two levels: sort_scan_tiles_kernel writes
// each 2048-bucket tile's in-tile exclusive prefix to cursor and the tile's
// total to tile_off; sort_scan_top_kernel turns tile_off into the tiles'
// exclusive offsets.  The scatter adds tile_off[key / 2048] to the cursor.
constexpr int kScanTile = (int)kSortScanTile;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane)
{
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
    }
    return v;
}

// m_dev, when not null, holds the bucket count (read on the device: the batch
// sort runs inside CUDA graphs while its bucket count changes)
__global__ void __launch_bounds__(1024) sort_scan_tiles_kernel(const uint32_t* __restrict__ hist,
                                                               uint32_t* __restrict__ cursor,
                                                               uint32_t* __restrict__ tile_off, int64_t m,
                                                               const int64_t* __restrict__ m_dev)
{
    __shared__ uint32_t wsum[32];
    if (m_dev) m = *m_dev;
    if ((int64_t)blockIdx.x * kScanTile >= m) return;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t i0 = (int64_t)blockIdx.x * kScanTile + 2 * t;
    const uint32_t a = i0 < m ? hist[i0] : 0u;
    const uint32_t b = i0 + 1 < m ? hist[i0 + 1] : 0u;
    const uint32_t own = a + b;
    const uint32_t incl = warp_incl_scan(own, lane);
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        const uint32_t v = wsum[lane];
        const uint32_t vi = warp_incl_scan(v, lane);
        wsum[lane] = vi - v;
        if (lane == 31) tile_off[blockIdx.x] = vi;
    }
    __syncthreads();
    const uint32_t excl = wsum[w] + incl - own;
    if (i0 < m) cursor[i0] = excl;
    if (i0 + 1 < m) cursor[i0 + 1] = excl + a;
}

__global__ void __launch_bounds__(1024) sort_scan_top_kernel(uint32_t* tile_off, int64_t tiles,
                                                             const int64_t* __restrict__ m_dev)
{
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (m_dev) tiles = (*m_dev + kScanTile - 1) / kScanTile;
    if (t == 0) carry = 0u;
    __syncthreads();
    for (int64_t base = 0; base < tiles; base += 1024) {
        const int64_t i = base + t;
        const uint32_t v = i < tiles ? tile_off[i] : 0u;
        const uint32_t incl = warp_incl_scan(v, lane);
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            const uint32_t x = wsum[lane];
            wsum[lane] = warp_incl_scan(x, lane) - x;
        }
        __syncthreads();
        const uint32_t excl = carry + wsum[w] + incl - v;
        __syncthreads();  // every thread has read carry
        if (i < tiles) tile_off[i] = excl;
        if (t == 1023) carry = excl + v;
        __syncthreads();
    }
}

// Block-local scatter.  A CTA takes a block of slots, sorts their (key, thread)
// pairs (bitonic: partners within a warp by shuffle, across warps through
// shared memory), reserves one cursor range per run of equal keys -- one
// atomic per run instead of one per warp and key -- and writes the particles
// in key order, so that a run's particles go to consecutive slots from
// consecutive threads.  The particle data is staged in shared memory by
// thread and read back by sorted position.
// Blocks of 512 slots for the single-state sorts (measured: 1.05 ms per
// 16.7M particles against 1.14 ms with 256); the batch scatter keeps one
// 256-particle tile per block.
constexpr int kScatterBlock = 512;
constexpr uint32_t kPastEnd = 0xFFFFFFFFu;  // key of a thread without a particle: sorts last, written nowhere

template <int B>
struct RunScratch {
    unsigned long long v[B];
    uint32_t key[B], base[B];
    int wmax[B / 32];
};
// the FP32-push state of a block's particles
template <int B>
struct ScatterStage {
    double x[3][B], p2[B];
    float p[3][B];
    int32_t pid[B];
    uint8_t alive[B];
    RunScratch<B> run;
};
// the FP64 SI state of a block's particles
template <int B>
struct ExactStage {
    double v[6][B];
    int32_t pid[B];
    uint8_t alive[B];
    RunScratch<B> run;
};

struct BlockRun {
    int src;      // thread whose particle leaves from this sorted position
    int64_t dest; // its slot relative to the bucket's cursor base; -1: nothing to write
};

// Called by every thread of the block, with its key (kPastEnd without a
// particle); its barriers also publish the staged particle data.
template <int B>
__device__ __forceinline__ BlockRun block_runs(uint32_t key, uint32_t* cursor, const uint32_t* __restrict__ tile_off,
                                               RunScratch<B>& sh)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    unsigned long long v = ((unsigned long long)key << 32) | (unsigned)t;
    for (int k = 2; k <= B; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            unsigned long long o;
            if (j >= 32) {
                sh.v[t] = v;
                __syncthreads();
                o = sh.v[t ^ j];
                __syncthreads();
            } else {
                o = __shfl_xor_sync(0xffffffffu, v, j);
            }
            const bool up = (t & k) == 0, lower = (t & j) == 0;
            v = (lower == up) ? (v < o ? v : o) : (v > o ? v : o);
        }
    }
    const uint32_t k_t = (uint32_t)(v >> 32);
    sh.key[t] = k_t;
    __syncthreads();
    const bool head = t == 0 || sh.key[t - 1] != k_t;
    const bool tail = t == B - 1 || sh.key[t + 1] != k_t;
    // start of this position's run: inclusive max-scan of (head ? t : 0)
    int rs = head ? t : 0;
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, rs, d);
        if (lane >= d) rs = max(rs, y);
    }
    if (lane == 31) sh.wmax[w] = rs;
    __syncthreads();
    for (int q = 0; q < w; ++q) rs = max(rs, sh.wmax[q]);
    if (tail && k_t != kPastEnd)
        sh.base[rs] = atomicAdd(&cursor[k_t], (uint32_t)(t - rs + 1)) + tile_off[k_t / kScanTile];
    __syncthreads();
    BlockRun r;
    r.src = (int)(v & 0xFFFFFFFFu);
    r.dest = k_t == kPastEnd ? -1 : (int64_t)sh.base[rs] + (t - rs);
    return r;
}

__global__ void __launch_bounds__(kScatterBlock) sort_scatter_block_kernel(
    uint32_t* cursor, const uint32_t* __restrict__ tile_off, int64_t n, const uint32_t* __restrict__ offs, int nx,
    int ny, int nz, uint32_t dead_key, const double* __restrict__ xs, const float* __restrict__ ps,
    const double* __restrict__ p2s, const int32_t* __restrict__ pids, const uint8_t* __restrict__ as,
    double* __restrict__ xd, float* __restrict__ pd, double* __restrict__ p2d, int32_t* __restrict__ pidd,
    uint8_t* __restrict__ ad)
{
    __shared__ ScatterStage<kScatterBlock> sh;
    const int t = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kScatterBlock + t;
    uint32_t key = kPastEnd;
    if (i < n) {
        const double x0 = xs[i], x1 = xs[n + i], x2 = xs[2 * n + i];
        const uint8_t al = as[i];
        sh.x[0][t] = x0; sh.x[1][t] = x1; sh.x[2][t] = x2;
        sh.p[0][t] = ps[i]; sh.p[1][t] = ps[n + i]; sh.p[2][t] = ps[2 * n + i];
        sh.p2[t] = p2s[i];
        sh.pid[t] = pids[i];
        sh.alive[t] = al;
        key = brick_key(x0, x1, x2, al, offs, nx, ny, nz, dead_key);
    }
    const BlockRun r = block_runs(key, cursor, tile_off, sh.run);
    if (r.dest < 0) return;
    const int64_t d = r.dest;
    const int q = r.src;
    xd[d] = sh.x[0][q]; xd[n + d] = sh.x[1][q]; xd[2 * n + d] = sh.x[2][q];
    pd[d] = sh.p[0][q]; pd[n + d] = sh.p[1][q]; pd[2 * n + d] = sh.p[2][q];
    p2d[d] = sh.p2[q];
    pidd[d] = sh.pid[q];
    ad[d] = sh.alive[q];
}

// ---- brick sort of an FP64 SI state (the FP64 push over BRICK_F64 fields):
// xs = [6][n] (x1, x2, x3, p1, p2, p3), pid, alive.  The bucket is the
// brick of the cell holding the position; it only orders the slots.
__device__ __forceinline__ uint32_t exact_brick_key(const double* __restrict__ xs, int64_t n, int64_t i, uint8_t al,
                                                    double x0, double y0, double z0, double idx, double idy,
                                                    double idz, const uint32_t* __restrict__ offs, int nx, int ny,
                                                    int nz, uint32_t dead_key)
{
    return brick_key((xs[i] - x0) * idx, (xs[n + i] - y0) * idy, (xs[2 * n + i] - z0) * idz, al, offs, nx, ny, nz,
                     dead_key);
}

__global__ void exact_key_kernel(const double* __restrict__ xs, const uint8_t* __restrict__ as, int64_t n, double x0,
                                 double y0, double z0, double idx, double idy, double idz,
                                 const uint32_t* __restrict__ offs, int nx, int ny, int nz, uint32_t dead_key,
                                 uint32_t* __restrict__ hist)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key =
        valid ? exact_brick_key(xs, n, i, as[i], x0, y0, z0, idx, idy, idz, offs, nx, ny, nz, dead_key) : dead_key;
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (valid) {
        const unsigned same = __match_any_sync(act, key);
        if ((same & lt) == 0) atomicAdd(&hist[key], (uint32_t)__popc(same));
    }
}

__global__ void __launch_bounds__(kScatterBlock) exact_scatter_kernel(
    uint32_t* cursor, const uint32_t* __restrict__ tile_off, int64_t n, double x0, double y0, double z0, double idx,
    double idy, double idz, const uint32_t* __restrict__ offs, int nx, int ny, int nz, uint32_t dead_key,
    const double* __restrict__ xs, const int32_t* __restrict__ pids, const uint8_t* __restrict__ as,
    double* __restrict__ xd, int32_t* __restrict__ pidd, uint8_t* __restrict__ ad)
{
    // block-local runs as in sort_scatter_block_kernel
    __shared__ ExactStage<kScatterBlock> sh;
    const int t = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kScatterBlock + t;
    uint32_t key = kPastEnd;
    if (i < n) {
#pragma unroll
        for (int k = 0; k < 6; ++k) sh.v[k][t] = xs[k * n + i];
        const uint8_t al = as[i];
        sh.pid[t] = pids[i];
        sh.alive[t] = al;
        key = exact_brick_key(xs, n, i, al, x0, y0, z0, idx, idy, idz, offs, nx, ny, nz, dead_key);
    }
    const BlockRun r = block_runs(key, cursor, tile_off, sh.run);
    if (r.dest < 0) return;
    const int64_t d = r.dest;
#pragma unroll
    for (int k = 0; k < 6; ++k) xd[k * n + d] = sh.v[k][r.src];
    pidd[d] = sh.pid[r.src];
    ad[d] = sh.alive[r.src];
}

__global__ void exact_import_kernel(const double* __restrict__ s0, const double* __restrict__ s1,
                                    const double* __restrict__ s2, const double* __restrict__ s3,
                                    const double* __restrict__ s4, const double* __restrict__ s5,
                                    const uint8_t* __restrict__ alive, int64_t n, double* __restrict__ xs,
                                    int32_t* __restrict__ pids, uint8_t* __restrict__ as)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        xs[i] = s0[i]; xs[n + i] = s1[i]; xs[2 * n + i] = s2[i];
        xs[3 * n + i] = s3[i]; xs[4 * n + i] = s4[i]; xs[5 * n + i] = s5[i];
        pids[i] = (int32_t)i;
        as[i] = alive[i];
    }
}

__global__ void exact_export_kernel(const double* __restrict__ xs, const int32_t* __restrict__ pids,
                                    const uint8_t* __restrict__ as, int64_t n, double* __restrict__ d0,
                                    double* __restrict__ d1, double* __restrict__ d2, double* __restrict__ d3,
                                    double* __restrict__ d4, double* __restrict__ d5, uint8_t* __restrict__ alive)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = pids[i];
        d0[q] = xs[i]; d1[q] = xs[n + i]; d2[q] = xs[2 * n + i];
        d3[q] = xs[3 * n + i]; d4[q] = xs[4 * n + i]; d5[q] = xs[5 * n + i];
        alive[q] = as[i];
    }
}

int grid_for(int64_t n, int threads, int num_sms)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms * 16;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

// Persistent launch: (SM count) x (resident blocks per SM, optionally capped).
// The gather is cache-bound, so fewer resident warps can win (less L1 churn).
template <int LAYOUT, int BLOCK, int MINB, int TEXC = 0>
int launch_push_fast_shape(const PushArgsFast& a, cudaStream_t s, int cap_per_sm = 0)
{
    const size_t smem = sizeof(uint32_t) * (size_t)(a.fld.nx + a.fld.ny + a.fld.nz);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto kfn = push_fast_kernel<LAYOUT, BLOCK, MINB, TEXC>;
    if (smem > 48 * 1024) PT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, BLOCK, smem);
    per_sm = std::max(per_sm, 1);
    if (cap_per_sm > 0) per_sm = std::min(per_sm, cap_per_sm);
    const int64_t blocks = std::min<int64_t>((a.n + BLOCK - 1) / BLOCK, (int64_t)sms * per_sm);
    kfn<<<(unsigned)blocks, BLOCK, smem, s>>>(a);
    PT_CHECK_LAUNCH("push_fast_kernel");
    return PT_OK;
}

template <int LAYOUT>
int launch_push_fast_t(const PushArgsFast& a, cudaStream_t s)
{
    switch (a.variant) {
    case 2: return launch_push_fast_shape<LAYOUT,256, 4>(a, s);
    case 3: return launch_push_fast_shape<LAYOUT,128, 8>(a, s);
    case 4: return launch_push_fast_shape<LAYOUT,512, 2>(a, s);
    case 5: return launch_push_fast_shape<LAYOUT,256, 1>(a, s, 1);
    case 6: return launch_push_fast_shape<LAYOUT,512, 1>(a, s, 1);
    case 7: return launch_push_fast_shape<LAYOUT,128, 1>(a, s, 3);
    case 8: return launch_push_fast_shape<LAYOUT,128, 1>(a, s, 2);
    case 9:   // 256 x occupancy, half of the corners through the texture path
        if (LAYOUT == LAYOUT_BF16 && a.fld.tex) return launch_push_fast_shape<LAYOUT, 256, 1, 4>(a, s);
        return launch_push_fast_shape<LAYOUT, 256, 1>(a, s);
    case 10:  // 256 x occupancy, every corner through the texture path
        if (LAYOUT == LAYOUT_BF16 && a.fld.tex) return launch_push_fast_shape<LAYOUT, 256, 1, 8>(a, s);
        return launch_push_fast_shape<LAYOUT, 256, 1>(a, s);
    case 11:  // 512 x 1, half of the corners through the texture path
        if (LAYOUT == LAYOUT_BF16 && a.fld.tex) return launch_push_fast_shape<LAYOUT, 512, 1, 4>(a, s, 1);
        return launch_push_fast_shape<LAYOUT, 512, 1>(a, s, 1);
    case 0:
    case 1:
    default: return launch_push_fast_shape<LAYOUT,256, 1>(a, s);
    }
}

int launch_push_fast(const PushArgsFast& a, cudaStream_t s)
{
    if (a.n <= 0 || a.step_count <= 0) return PT_OK;
    switch (a.fld.layout) {
    case LAYOUT_F32: return launch_push_fast_t<LAYOUT_F32>(a, s);
    case LAYOUT_BF16_XPAIR: return launch_push_fast_t<LAYOUT_BF16_XPAIR>(a, s);
    default: return launch_push_fast_t<LAYOUT_BF16>(a, s);
    }
}

int launch_brick_convert(const double* const comps[6], const pt_grid& g, double B_ref, int layout, void* nodes,
                         const uint32_t* offs, int64_t n_nodes, const float boff[3], cudaStream_t s)
{
    const int64_t total = g.nx * g.ny * g.nz;
    const int threads = 256;
    int blocks = (int)std::min<int64_t>((total + threads - 1) / threads, 148 * 32);
    brick_convert_kernel<<<blocks, threads, 0, s>>>(comps[0], comps[1], comps[2], comps[3], comps[4], comps[5],
                                                    g.nx, g.ny, g.nz, 1.0 / B_ref, 1.0 / C_LIGHT, layout, nodes, offs,
                                                    n_nodes, boff[0], boff[1], boff[2]);
    PT_CHECK_LAUNCH("brick_convert_kernel");
    return PT_OK;
}

// One thread per particle: its `rows` saves (contiguous, one 32-byte record
// at pitch 8) out to `rows` coalesced rows.
__global__ void tf_to_rows_kernel(const float* __restrict__ tf, int64_t n, int pitch, int rows,
                                  float* __restrict__ out)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const float* rec = tf + p * pitch;
        for (int r = 0; r < rows; ++r) out[(int64_t)r * n + p] = rec[r];
    }
}

int launch_tf_to_rows(const float* tf, int64_t n, int pitch, int rows, float* out, cudaStream_t s)
{
    if (n <= 0 || rows <= 0) return PT_OK;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)148 * 64);
    tf_to_rows_kernel<<<blocks, 256, 0, s>>>(tf, n, pitch, rows, out);
    PT_CHECK_LAUNCH("tf_to_rows_kernel");
    return PT_OK;
}

// Sums and counts of the finite values of Bx, By, Bz: kMeanBlocks blocks
// each add a contiguous range (a strided sum per thread, then a tree over the
// block), and one thread adds the block sums in block order -- a fixed order,
// so the same bits each time.  A non-finite node is left out of the mean
// (it stays non-finite in the bricks, where only its own cells see it).
constexpr int kMeanBlocks = 256, kMeanThreads = 256;
__global__ void __launch_bounds__(kMeanThreads) component_sum_kernel(const double* __restrict__ bx,
                                                                     const double* __restrict__ by,
                                                                     const double* __restrict__ bz, int64_t nn,
                                                                     double* __restrict__ partial)
{
    __shared__ double sh[6][kMeanThreads];
    const int64_t per = (nn + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * per, hi = min(nn, lo + per);
    double s[3] = {0.0, 0.0, 0.0}, k[3] = {0.0, 0.0, 0.0};
    for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        const double v[3] = {bx[t], by[t], bz[t]};
        for (int c = 0; c < 3; ++c)
            if (isfinite(v[c])) {
                s[c] += v[c];
                k[c] += 1.0;
            }
    }
    for (int c = 0; c < 3; ++c) {
        sh[c][threadIdx.x] = s[c];
        sh[3 + c][threadIdx.x] = k[c];
    }
    __syncthreads();
    for (int w = kMeanThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; ++c) partial[6 * blockIdx.x + c] = sh[c][0];
}

__global__ void partial_sum_kernel(const double* __restrict__ partial, int blocks, double* __restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < blocks; ++b)
        for (int c = 0; c < 6; ++c) s[c] += partial[6 * b + c];
    for (int c = 0; c < 6; ++c) out[c] = s[c];
}

int field_means(pt_ctx* ctx, const double* const comps[6], int64_t nn, double mean[3], cudaStream_t s)
{
    (void)ctx;
    if (nn <= 0) return fail(PT_ERR_ARG, "empty field");
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * (6 * kMeanBlocks + 6));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PT_ERR_OOM, "field mean scratch allocation failed");
    }
    component_sum_kernel<<<kMeanBlocks, kMeanThreads, 0, s>>>(comps[0], comps[1], comps[2], nn, d);
    partial_sum_kernel<<<1, 32, 0, s>>>(d, kMeanBlocks, d + 6 * kMeanBlocks);
    double sums[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(sums, d + 6 * kMeanBlocks, sizeof(sums), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "field means");
    for (int c = 0; c < 3; ++c) mean[c] = sums[3 + c] > 0.0 ? sums[c] / sums[3 + c] : 0.0;
    return PT_OK;
}

int launch_fast_import(pt_fast_state* st, const pt_field* f, const double* x1, const double* x2, const double* x3,
                       const double* p1, const double* p2, const double* p3, const uint8_t* alive, cudaStream_t s)
{
    const pt_grid& g = f->grid;
    fast_import_kernel<<<grid_for(st->n, 256, st->ctx->num_sms), 256, 0, s>>>(
        x1, x2, x3, p1, p2, p3, alive, st->n, g.xmin, g.ymin, g.zmin, g.dx, g.dy, g.dz, st->x, st->p, st->p2,
        st->pid, st->alive);
    PT_CHECK_LAUNCH("fast_import_kernel");
    return PT_OK;
}

int launch_fast_export(const pt_fast_state* st, const pt_field* f, double* x1, double* x2, double* x3, double* p1,
                       double* p2, double* p3, uint8_t* alive, cudaStream_t s)
{
    const pt_grid& g = f->grid;
    fast_export_kernel<<<grid_for(st->n, 256, st->ctx->num_sms), 256, 0, s>>>(
        st->x, st->p, st->p2, st->pid, st->alive, st->n, g.xmin, g.ymin, g.zmin, g.dx, g.dy, g.dz, x1, x2, x3, p1,
        p2, p3, alive);
    PT_CHECK_LAUNCH("fast_export_kernel");
    return PT_OK;
}

int fast_sort(pt_ctx* ctx, pt_fast_state* st, const pt_field* f, cudaStream_t s)
{
    const int64_t n = st->n;
    if (n <= 1) return PT_OK;
    const uint32_t nb = (uint32_t)((f->n_nodes + 511) / 512);
    const int64_t m = (int64_t)nb + 1;  // + dead bucket
    // scratch: hist[m], cursor[m], tile offsets; the scatter goes to the
    // state's second buffer set, which then becomes the current one
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const int64_t tiles = (m + kScanTile - 1) / kScanTile;
    const size_t o_hist = take(sizeof(uint32_t) * m), o_cur = take(sizeof(uint32_t) * m),
                 o_tiles = take(sizeof(uint32_t) * tiles);
    if (st->sort_tmp_bytes < off) {
        if (st->sort_tmp) cudaFree(st->sort_tmp);
        st->sort_tmp = nullptr;
        st->sort_tmp_bytes = 0;
        cudaError_t e = cudaMalloc(&st->sort_tmp, off);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PT_ERR_OOM, "sort scratch allocation failed");
        }
        st->sort_tmp_bytes = off;
    }
    if (!st->x_alt) {
        cudaError_t e = cudaMalloc((void**)&st->x_alt, sizeof(double) * 3 * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&st->p_alt, sizeof(float) * 3 * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&st->p2_alt, sizeof(double) * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&st->pid_alt, sizeof(int32_t) * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&st->alive_alt, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PT_ERR_OOM, "sort state buffers allocation failed");
        }
    }
    char* base = (char*)st->sort_tmp;
    uint32_t* hist = (uint32_t*)(base + o_hist);
    uint32_t* cur = (uint32_t*)(base + o_cur);
    uint32_t* tile_off = (uint32_t*)(base + o_tiles);
    PT_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * m, s));
    // one particle per thread: the key and scatter loops are chains of
    // dependent memory operations, so more of them in flight is what counts
    const int gb = (int)std::min<int64_t>((n + 255) / 256, INT32_MAX);
    const int nx = (int)f->grid.nx, ny = (int)f->grid.ny, nz = (int)f->grid.nz;
    sort_key_kernel<<<gb, 256, 0, s>>>(st->x, st->alive, n, f->offs, nx, ny, nz, nb, hist);
    PT_CHECK_LAUNCH("sort_key_kernel");
    sort_scan_tiles_kernel<<<(unsigned)tiles, 1024, 0, s>>>(hist, cur, tile_off, m, nullptr);
    PT_CHECK_LAUNCH("sort_scan_tiles_kernel");
    sort_scan_top_kernel<<<1, 1024, 0, s>>>(tile_off, tiles, nullptr);
    PT_CHECK_LAUNCH("sort_scan_top_kernel");
    sort_scatter_block_kernel<<<(unsigned)((n + kScatterBlock - 1) / kScatterBlock), kScatterBlock, 0, s>>>(
        cur, tile_off, n, f->offs, nx, ny, nz, nb, st->x, st->p, st->p2, st->pid, st->alive, st->x_alt, st->p_alt,
        st->p2_alt, st->pid_alt, st->alive_alt);
    PT_CHECK_LAUNCH("sort_scatter_block_kernel");
    std::swap(st->x, st->x_alt);
    std::swap(st->p, st->p_alt);
    std::swap(st->p2, st->p2_alt);
    std::swap(st->pid, st->pid_alt);
    std::swap(st->alive, st->alive_alt);
    return PT_OK;
}

int launch_exact_sort(const double* xs, const int32_t* pids, const uint8_t* as, int64_t n, const pt_field* f,
                      double* xd, int32_t* pidd, uint8_t* ad, uint32_t* hist, uint32_t* cursor, int num_sms,
                      cudaStream_t s)
{
    if (n <= 0) return PT_OK;
    const pt_grid& g = f->grid;
    const uint32_t nb = (uint32_t)((f->n_nodes + 511) / 512);
    const int64_t m = (int64_t)nb + 1;  // + dead bucket
    const int64_t tiles = sort_scan_tiles(m);
    uint32_t* tile_off = cursor + m;
    PT_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * m, s));
    const int gb = (int)std::min<int64_t>((n + 255) / 256, INT32_MAX);
    const int nx = (int)g.nx, ny = (int)g.ny, nz = (int)g.nz;
    const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
    exact_key_kernel<<<gb, 256, 0, s>>>(xs, as, n, g.xmin, g.ymin, g.zmin, idx, idy, idz, f->offs, nx, ny, nz, nb,
                                        hist);
    PT_CHECK_LAUNCH("exact_key_kernel");
    sort_scan_tiles_kernel<<<(unsigned)tiles, 1024, 0, s>>>(hist, cursor, tile_off, m, nullptr);
    PT_CHECK_LAUNCH("sort_scan_tiles_kernel");
    sort_scan_top_kernel<<<1, 1024, 0, s>>>(tile_off, tiles, nullptr);
    PT_CHECK_LAUNCH("sort_scan_top_kernel");
    exact_scatter_kernel<<<(unsigned)((n + kScatterBlock - 1) / kScatterBlock), kScatterBlock, 0, s>>>(
        cursor, tile_off, n, g.xmin, g.ymin, g.zmin, idx, idy, idz, f->offs, nx, ny, nz, nb, xs, pids, as, xd, pidd,
        ad);
    PT_CHECK_LAUNCH("exact_scatter_kernel");
    (void)num_sms;
    return PT_OK;
}

int launch_exact_import(double* const src[6], const uint8_t* alive, int64_t n, double* xs, int32_t* pids,
                        uint8_t* as, int num_sms, cudaStream_t s)
{
    if (n <= 0) return PT_OK;
    exact_import_kernel<<<grid_for(n, 256, num_sms), 256, 0, s>>>(src[0], src[1], src[2], src[3], src[4], src[5],
                                                                 alive, n, xs, pids, as);
    PT_CHECK_LAUNCH("exact_import_kernel");
    return PT_OK;
}

int launch_exact_export(const double* xs, const int32_t* pids, const uint8_t* as, int64_t n, double* const dst[6],
                        uint8_t* alive, int num_sms, cudaStream_t s)
{
    if (n <= 0) return PT_OK;
    exact_export_kernel<<<grid_for(n, 256, num_sms), 256, 0, s>>>(xs, pids, as, n, dst[0], dst[1], dst[2], dst[3],
                                                                 dst[4], dst[5], alive);
    PT_CHECK_LAUNCH("exact_export_kernel");
    return PT_OK;
}

// ------------------------------------------------------------ batches
namespace {

// One persistent kernel for every campaign of a batch: each CTA pulls
// 256-particle tiles from the tile table (atomic counter), loads the tile's
// campaign constants and field offset tables into shared memory when the
// campaign changes, and runs K steps of its particles from the campaign's
// device-resident step counter.  The per-particle arithmetic is
// advance_particle, so a particle's trajectory is the same alone or batched.
// BLOCK threads per CTA: thread i advances particles i, i + BLOCK, ... of each
// kBatchTile-particle tile it claims, one after another.
template <int LAYOUT, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) push_batch_kernel(BatchLaunch L)
{
    extern __shared__ uint32_t s_offs[];
    __shared__ PushArgsFast s_a;
    __shared__ int s_tile, s_camp, s_buf;
    __shared__ const uint32_t* s_loaded;
    __shared__ long long s_begin, s_end;
    if (threadIdx.x == 0) {
        s_camp = -1;
        s_loaded = nullptr;
    }
    const int n_tiles = *L.n_tiles;
    const int64_t cap = L.st[0].cap;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = atomicAdd(L.tile_counter, 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= n_tiles) break;
        const BatchTile T = L.tiles[t];
        if (T.campaign != s_camp) {
            const BatchCampaignDev* C = L.camps + T.campaign;
            constexpr int words = (int)(sizeof(PushArgsFast) / sizeof(uint32_t));
            for (int i = threadIdx.x; i < words; i += blockDim.x)
                reinterpret_cast<uint32_t*>(&s_a)[i] = reinterpret_cast<const uint32_t*>(&C->a)[i];
            if (threadIdx.x == 0) {
                s_begin = C->step;
                s_end = min(C->step + C->K, C->a.nsteps);
                // a campaign re-sorted in this epoch now sits in its other buffer
                s_buf = (L.sorted && batch_sort_due(*C)) ? 1 - C->par : C->par;
            }
            __syncthreads();
            if (threadIdx.x == 0) s_camp = T.campaign;
            if (s_a.fld.offs != s_loaded) {
                const int tot = (int)(s_a.fld.nx + s_a.fld.ny + s_a.fld.nz);
                for (int i = threadIdx.x; i < tot; i += blockDim.x) s_offs[i] = s_a.fld.offs[i];
            }
            __syncthreads();
            if (threadIdx.x == 0) s_loaded = s_a.fld.offs;
        }
        const int64_t sb = s_begin, se = s_end;
        if (sb >= se) continue;
        for (int q = threadIdx.x; q < T.count; q += BLOCK) {
            const uint32_t* ox = s_offs;
            const uint32_t* oy = s_offs + s_a.fld.nx;
            const uint32_t* oz = s_offs + s_a.fld.nx + s_a.fld.ny;
            const BatchStateDev st = s_buf ? L.st[1] : L.st[0];
            const int64_t slot = T.begin + q;
            double x = st.x[slot], y = st.x[cap + slot], z = st.x[2 * cap + slot];
            float px = st.p[slot], py = st.p[cap + slot], pz = st.p[2 * cap + slot];
            double P2 = st.p2[slot];
            bool al = st.alive[slot] != 0;
            advance_particle<LAYOUT>(x, y, z, px, py, pz, P2, al, st.pid[slot], s_a, ox, oy, oz, sb, se);
            st.x[slot] = x; st.x[cap + slot] = y; st.x[2 * cap + slot] = z;
            st.p[slot] = px; st.p[cap + slot] = py; st.p[2 * cap + slot] = pz;
            st.p2[slot] = P2;
            st.alive[slot] = al ? 1 : 0;
        }
    }
}

__global__ void batch_epoch_end_kernel(BatchCampaignDev* camps, int n, int* tile_counter, int sorted)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n && camps[c].active && camps[c].running) {
        BatchCampaignDev& C = camps[c];
        if (sorted && batch_sort_due(C)) C.par ^= 1;
        C.epochs += 1;
        C.step = min(C.step + C.K, C.a.nsteps);
    }
    if (c == 0) *tile_counter = 0;
}

// Install a new campaign table uploaded by the host while keeping the fields
// the epochs advance on the device (step, epochs, buffer parity) of every
// campaign already in the batch -- the host's copies of them are stale;
// `fresh`, a campaign just added, takes the table's (0, 0, buffer 0).
__global__ void batch_apply_kernel(BatchCampaignDev* camps, const BatchCampaignDev* __restrict__ staged, int n,
                                   int fresh)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    BatchCampaignDev v = staged[c];
    const BatchCampaignDev& old = camps[c];
    if (c != fresh && v.active && old.active) {
        v.step = old.step;
        v.epochs = old.epochs;
        v.par = old.par;
    }
    camps[c] = v;
}

__global__ void zero_counted_kernel(uint32_t* a, const int64_t* m)
{
    const int64_t mm = *m;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < mm; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = 0u;
}

// Sort key of every particle of a campaign due for a re-sort -- the slots
// the tile table covers, one block per tile: the campaign's first bucket +
// the brick of the particle's cell (the campaign's dead bucket for dead
// particles).  Free slots and paused campaigns hold no tiles, and campaigns
// not due skip their tiles, so the cost follows the particles sorted, not
// the arena's capacity.
__global__ void __launch_bounds__(kBatchTile) batch_key_kernel(const BatchCampaignDev* __restrict__ camps,
                                                               const BatchTile* __restrict__ tiles,
                                                               const int* __restrict__ n_tiles, BatchStateDev st0,
                                                               BatchStateDev st1, uint32_t* __restrict__ keys,
                                                               uint32_t* __restrict__ hist)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t cap = st0.cap;
    const int nt = *n_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const BatchTile T = tiles[t];
        const BatchCampaignDev& C = camps[T.campaign];
        if (!batch_sort_due(C)) continue;  // uniform over the block
        const BatchStateDev st = C.par ? st1 : st0;
        const bool valid = (int)threadIdx.x < T.count;
        const int64_t i = T.begin + threadIdx.x;
        uint32_t key = 0;
        if (valid) {
            key = (uint32_t)(C.key_base + C.n_bricks);
            if (st.alive[i]) {
                const int nx = (int)C.a.fld.nx, ny = (int)C.a.fld.ny, nz = (int)C.a.fld.nz;
                const uint32_t* offs = C.a.fld.offs;
                int ix = min(max((int)floor(st.x[i]), 0), nx - 2);
                int iy = min(max((int)floor(st.x[cap + i]), 0), ny - 2);
                int iz = min(max((int)floor(st.x[2 * cap + i]), 0), nz - 2);
                key = (uint32_t)C.key_base + ((offs[ix] + offs[nx + iy] + offs[nx + ny + iz]) >> 9);
            }
            keys[i] = key;
        }
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned same = __match_any_sync(act, key);
            if ((same & lt) == 0) atomicAdd(&hist[key], (uint32_t)__popc(same));
        }
    }
}

// Sort position of each due campaign's first bucket, read before the
// scatter's cursor atomics move it: a campaign's particles land at
// slot0 + (sort position - dense_base) in its other buffer.
__global__ void batch_base_kernel(BatchCampaignDev* camps, int n, const uint32_t* __restrict__ cursor,
                                  const uint32_t* __restrict__ tile_off)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || !batch_sort_due(camps[c])) return;
    const int64_t k = camps[c].key_base;
    camps[c].dense_base = (int64_t)cursor[k] + tile_off[k / kScanTile];
}

__global__ void __launch_bounds__(kBatchTile) batch_scatter_kernel(const uint32_t* __restrict__ keys, uint32_t* cursor,
                                                                   const uint32_t* __restrict__ tile_off,
                                                                   const BatchCampaignDev* __restrict__ camps,
                                                                   const BatchTile* __restrict__ tiles,
                                                                   const int* __restrict__ n_tiles,
                                                                   BatchStateDev st0, BatchStateDev st1)
{
    // one tile per block at a time, scattered as in sort_scatter_block_kernel
    __shared__ ScatterStage<kBatchTile> sh;
    const int64_t cap = st0.cap;
    const int nt = *n_tiles;
    const int t = threadIdx.x;
    for (int tl = blockIdx.x; tl < nt; tl += gridDim.x) {
        const BatchTile T = tiles[tl];
        const BatchCampaignDev& C = camps[T.campaign];
        if (!batch_sort_due(C)) continue;  // uniform over the block
        const BatchStateDev from = C.par ? st1 : st0, to = C.par ? st0 : st1;
        uint32_t key = kPastEnd;
        if (t < T.count) {
            const int64_t i = T.begin + t;
            key = keys[i];
            sh.x[0][t] = from.x[i]; sh.x[1][t] = from.x[cap + i]; sh.x[2][t] = from.x[2 * cap + i];
            sh.p[0][t] = from.p[i]; sh.p[1][t] = from.p[cap + i]; sh.p[2][t] = from.p[2 * cap + i];
            sh.p2[t] = from.p2[i];
            sh.pid[t] = from.pid[i];
            sh.alive[t] = from.alive[i];
        }
        const BlockRun r = block_runs(key, cursor, tile_off, sh.run);
        if (r.dest >= 0) {
            const int64_t d = r.dest + C.slot0 - C.dense_base;
            const int q = r.src;
            to.x[d] = sh.x[0][q]; to.x[cap + d] = sh.x[1][q]; to.x[2 * cap + d] = sh.x[2][q];
            to.p[d] = sh.p[0][q]; to.p[cap + d] = sh.p[1][q]; to.p[2 * cap + d] = sh.p[2][q];
            to.p2[d] = sh.p2[q];
            to.pid[d] = sh.pid[q];
            to.alive[d] = sh.alive[q];
        }
        __syncthreads();  // the next tile's staging overwrites sh
    }
}

// SI state of one campaign <-> arena slots [slot0, slot0 + n); same formulas
// as fast_import_kernel / fast_export_kernel.
__global__ void batch_import_kernel(BatchStateDev st, int64_t slot0, int64_t n, const double* __restrict__ x1,
                                    const double* __restrict__ x2, const double* __restrict__ x3,
                                    const double* __restrict__ p1, const double* __restrict__ p2,
                                    const double* __restrict__ p3, const uint8_t* __restrict__ alive, double xmin,
                                    double ymin, double zmin, double dx, double dy, double dz)
{
    const double inv_mc = 1.0 / (M_P * C_LIGHT);
    const int64_t cap = st.cap;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = slot0 + i;
        st.x[s] = (x1[i] - xmin) / dx;
        st.x[cap + s] = (x2[i] - ymin) / dy;
        st.x[2 * cap + s] = (x3[i] - zmin) / dz;
        const double qx = p1[i] * inv_mc, qy = p2[i] * inv_mc, qz = p3[i] * inv_mc;
        st.p[s] = (float)qx; st.p[cap + s] = (float)qy; st.p[2 * cap + s] = (float)qz;
        st.p2[s] = qx * qx + qy * qy + qz * qz;
        st.pid[s] = (int32_t)i;
        st.alive[s] = alive[i];
    }
}

__global__ void batch_export_kernel(BatchStateDev st0, BatchStateDev st1, const BatchCampaignDev* __restrict__ camps,
                                    int id, int64_t slot0, int64_t n, double xmin, double ymin, double zmin,
                                    double dx, double dy, double dz, double* x1, double* x2, double* x3, double* p1,
                                    double* p2, double* p3, uint8_t* alive)
{
    const BatchStateDev st = camps[id].par ? st1 : st0;
    const int64_t cap = st.cap;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = slot0 + i;
        const int64_t q = st.pid[s];
        x1[q] = xmin + st.x[s] * dx;
        x2[q] = ymin + st.x[cap + s] * dy;
        x3[q] = zmin + st.x[2 * cap + s] * dz;
        const double px = st.p[s], py = st.p[cap + s], pz = st.p[2 * cap + s];
        const double sc = sqrt(st.p2[s] / (px * px + py * py + pz * pz)) * (M_P * C_LIGHT);
        p1[q] = px * sc; p2[q] = py * sc; p3[q] = pz * sc;
        alive[q] = st.alive[s];
    }
}

}  // namespace

template <int BLOCK>
void* push_batch_fn(int layout)
{
    return layout == LAYOUT_F32 ? (void*)push_batch_kernel<LAYOUT_F32, BLOCK>
           : (layout == LAYOUT_BF16_XPAIR ? (void*)push_batch_kernel<LAYOUT_BF16_XPAIR, BLOCK>
                                          : (void*)push_batch_kernel<LAYOUT_BF16, BLOCK>);
}

int launch_push_batch(const BatchLaunch& L, cudaStream_t s)
{
    const size_t smem = sizeof(uint32_t) * (size_t)std::max(L.smem_words, 1);
    void* kfn = L.threads == 64 ? push_batch_fn<64>(L.layout)
                : (L.threads == 128 ? push_batch_fn<128>(L.layout) : push_batch_fn<kBatchTile>(L.layout));
    const int threads = L.threads == 64 || L.threads == 128 ? L.threads : kBatchTile;
    if (smem > 48 * 1024) PT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BatchLaunch arg = L;
    void* args[] = {&arg};
    PT_CUDA(cudaLaunchKernel(kfn, dim3(L.grid), dim3(threads), args, smem, s));
    PT_CHECK_LAUNCH("push_batch_kernel");
    return PT_OK;
}

int launch_batch_apply(BatchCampaignDev* camps, const BatchCampaignDev* staged, int n_camps, int fresh,
                       cudaStream_t s)
{
    batch_apply_kernel<<<(std::max(n_camps, 1) + 127) / 128, 128, 0, s>>>(camps, staged, n_camps, fresh);
    PT_CHECK_LAUNCH("batch_apply_kernel");
    return PT_OK;
}

int launch_batch_epoch_end(BatchCampaignDev* camps, int n_camps, int* tile_counter, int sorted, cudaStream_t s)
{
    batch_epoch_end_kernel<<<(std::max(n_camps, 1) + 127) / 128, 128, 0, s>>>(camps, n_camps, tile_counter, sorted);
    PT_CHECK_LAUNCH("batch_epoch_end_kernel");
    return PT_OK;
}

int launch_batch_sort(BatchCampaignDev* camps, int n_camps, const BatchTile* tiles, const int* n_tiles, int grid,
                      BatchStateDev st0, BatchStateDev st1, uint32_t* keys, uint32_t* hist, uint32_t* cursor,
                      const int64_t* d_m, int64_t max_buckets, int num_sms, cudaStream_t s)
{
    const int zb = (int)std::min<int64_t>((max_buckets + 255) / 256, (int64_t)num_sms * 8);
    zero_counted_kernel<<<std::max(zb, 1), 256, 0, s>>>(hist, d_m);
    PT_CHECK_LAUNCH("zero_counted_kernel");
    const int gb = std::max(grid, 1);  // one block per tile of the table (tile-stride beyond)
    batch_key_kernel<<<gb, kBatchTile, 0, s>>>(camps, tiles, n_tiles, st0, st1, keys, hist);
    PT_CHECK_LAUNCH("batch_key_kernel");
    uint32_t* tile_off = cursor + max_buckets;
    const int64_t max_tiles = sort_scan_tiles(max_buckets);
    sort_scan_tiles_kernel<<<(unsigned)std::max<int64_t>(max_tiles, 1), 1024, 0, s>>>(hist, cursor, tile_off,
                                                                                    max_buckets, d_m);
    PT_CHECK_LAUNCH("sort_scan_tiles_kernel");
    sort_scan_top_kernel<<<1, 1024, 0, s>>>(tile_off, max_tiles, d_m);
    PT_CHECK_LAUNCH("sort_scan_top_kernel");
    batch_base_kernel<<<(std::max(n_camps, 1) + 127) / 128, 128, 0, s>>>(camps, n_camps, cursor, tile_off);
    PT_CHECK_LAUNCH("batch_base_kernel");
    batch_scatter_kernel<<<gb, kBatchTile, 0, s>>>(keys, cursor, tile_off, camps, tiles, n_tiles, st0, st1);
    PT_CHECK_LAUNCH("batch_scatter_kernel");
    return PT_OK;
}

int launch_batch_import(BatchStateDev st, int64_t slot0, int64_t n, const pt_field* f, const double* x1,
                        const double* x2, const double* x3, const double* p1, const double* p2, const double* p3,
                        const uint8_t* alive, int num_sms, cudaStream_t s)
{
    if (n <= 0) return PT_OK;
    const pt_grid& g = f->grid;
    batch_import_kernel<<<grid_for(n, 256, num_sms), 256, 0, s>>>(st, slot0, n, x1, x2, x3, p1, p2, p3, alive,
                                                                 g.xmin, g.ymin, g.zmin, g.dx, g.dy, g.dz);
    PT_CHECK_LAUNCH("batch_import_kernel");
    return PT_OK;
}

int launch_batch_export(BatchStateDev st0, BatchStateDev st1, const BatchCampaignDev* camps, int id, int64_t slot0,
                        int64_t n, const pt_field* f, double* x1, double* x2, double* x3, double* p1, double* p2,
                        double* p3, uint8_t* alive, int num_sms, cudaStream_t s)
{
    if (n <= 0) return PT_OK;
    const pt_grid& g = f->grid;
    batch_export_kernel<<<grid_for(n, 256, num_sms), 256, 0, s>>>(st0, st1, camps, id, slot0, n, g.xmin, g.ymin,
                                                                 g.zmin, g.dx, g.dy, g.dz, x1, x2, x3, p1, p2, p3,
                                                                 alive);
    PT_CHECK_LAUNCH("batch_export_kernel");
    return PT_OK;
}

}  // namespace pt
