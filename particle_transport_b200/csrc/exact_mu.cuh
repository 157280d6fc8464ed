// Exact (reference-rounding) mu of a phase-space sample, shared by the
// phase-space mu reconstruction and the fused phase-space D_mumu binning.
//
// Every translation unit that includes this header is compiled with
// --fmad=false: the expressions keep the reference's evaluation order
// (a*b*c == (a*b)*c, no FMA contraction) and IEEE division / sqrt, so mu is
// bit-identical to the reference's reconstruction at the same precision.
#pragma once

#include "pt_internal.cuh"

namespace pt {
namespace exact {

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

// locate() with the cell's 0-based node indices instead of its linear base
template <typename R>
struct Cell3 {
    int i, j, k;
    Cell<R> t;  // tx, ty, tz (base unused)
};

template <typename R>
__device__ __forceinline__ Cell3<R> locate3(R x, R y, R z, R xmin, R ymin, R zmin, R dx, R dy, R dz, int64_t nx,
                                            int64_t ny, int64_t nz)
{
    R fx = (x - xmin) / dx + R(1);
    R fy = (y - ymin) / dy + R(1);
    R fz = (z - zmin) / dz + R(1);
    double ci = cell_index(fx, nx), cj = cell_index(fy, ny), ck = cell_index(fz, nz);
    Cell3<R> c;
    c.t.tx = fx - (R)ci;
    c.t.ty = fy - (R)cj;
    c.t.tz = fz - (R)ck;
    c.t.base = 0;
    c.i = (int)ci - 1;
    c.j = (int)cj - 1;
    c.k = (int)ck - 1;
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

// reconstruct_mu_kernel! body (src/compute_delta_mu2_curve.jl:151-184) at
// the compute precision R: NaN for NaN inputs or a position outside the box.
template <typename R>
__device__ __forceinline__ R phase_space_mu(R xx, R yy, R zz, R px, R py, R pz, const R* const B[3], const pt_grid& g)
{
    const R xmin = (R)g.xmin, ymin = (R)g.ymin, zmin = (R)g.zmin;
    const R xmax = (R)g.xmax, ymax = (R)g.ymax, zmax = (R)g.zmax;
    const R dx = (R)g.dx, dy = (R)g.dy, dz = (R)g.dz;
    R v = R(NAN);
    if (!(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) && xmin <= xx &&
        xx <= xmax && ymin <= yy && yy <= ymax && zmin <= zz && zz <= zmax) {
        Cell<R> c = locate<R>(xx, yy, zz, xmin, ymin, zmin, dx, dy, dz, g.nx, g.ny, g.nz);
        const int64_t sy = g.nx, sz = g.nx * g.ny;
        R b0 = sample(B[0], c, sy, sz), b1 = sample(B[1], c, sy, sz), b2 = sample(B[2], c, sy, sz);
        v = pitch_mu<R>(px, py, pz, b0, b1, b2);
    }
    return v;
}

// B of one node as one record (Bx, By, Bz, pad): the 8 corners of a cell are
// 8 vector loads instead of 24 scalar ones.  The values and the arithmetic are
// those of sample() on the three separate arrays, component by component.
template <typename R>
struct alignas(4 * sizeof(R)) Vec4 {
    R x, y, z, w;
};

template <typename R>
__device__ __forceinline__ Vec4<R> load_vec4(const Vec4<R>* p)
{
    if constexpr (sizeof(R) == 4) {
        const float4 v = __ldg((const float4*)p);
        return Vec4<R>{v.x, v.y, v.z, v.w};
    } else {
        const double2 a = __ldg((const double2*)p), b = __ldg((const double2*)p + 1);
        return Vec4<R>{a.x, a.y, b.x, b.y};
    }
}

template <typename R>
__device__ __forceinline__ R lerp8(R c000, R c100, R c010, R c110, R c001, R c101, R c011, R c111, const Cell<R>& c)
{
    // src/phase_space_gpu_runner.jl:269-275, the order of sample()
    R c00 = c000 * (R(1) - c.tx) + c100 * c.tx;
    R c10 = c010 * (R(1) - c.tx) + c110 * c.tx;
    R c01 = c001 * (R(1) - c.tx) + c101 * c.tx;
    R c11 = c011 * (R(1) - c.tx) + c111 * c.tx;
    R c0 = c00 * (R(1) - c.ty) + c10 * c.ty;
    R c1 = c01 * (R(1) - c.ty) + c11 * c.ty;
    return c0 * (R(1) - c.tz) + c1 * c.tz;
}

// phase_space_mu() with B read from interleaved node records
template <typename R>
__device__ __forceinline__ R phase_space_mu4(R xx, R yy, R zz, R px, R py, R pz, const Vec4<R>* __restrict__ B4,
                                             const pt_grid& g)
{
    const R xmin = (R)g.xmin, ymin = (R)g.ymin, zmin = (R)g.zmin;
    const R xmax = (R)g.xmax, ymax = (R)g.ymax, zmax = (R)g.zmax;
    const R dx = (R)g.dx, dy = (R)g.dy, dz = (R)g.dz;
    R v = R(NAN);
    if (!(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) && xmin <= xx &&
        xx <= xmax && ymin <= yy && yy <= ymax && zmin <= zz && zz <= zmax) {
        Cell<R> c = locate<R>(xx, yy, zz, xmin, ymin, zmin, dx, dy, dz, g.nx, g.ny, g.nz);
        const int64_t sy = g.nx, sz = g.nx * g.ny;
        const Vec4<R>* b = B4 + c.base;
        const Vec4<R> v000 = load_vec4(b), v100 = load_vec4(b + 1), v010 = load_vec4(b + sy),
                      v110 = load_vec4(b + 1 + sy), v001 = load_vec4(b + sz), v101 = load_vec4(b + 1 + sz),
                      v011 = load_vec4(b + sy + sz), v111 = load_vec4(b + 1 + sy + sz);
        const R b0 = lerp8(v000.x, v100.x, v010.x, v110.x, v001.x, v101.x, v011.x, v111.x, c);
        const R b1 = lerp8(v000.y, v100.y, v010.y, v110.y, v001.y, v101.y, v011.y, v111.y, c);
        const R b2 = lerp8(v000.z, v100.z, v010.z, v110.z, v001.z, v101.z, v011.z, v111.z, c);
        v = pitch_mu<R>(px, py, pz, b0, b1, b2);
    }
    return v;
}

// B of the 8 corners of one cell as one record: corner-major in the order of
// lerp8 (c000, c100, c010, c110, c001, c101, c011, c111), (Bx, By, Bz) within
// a corner.  Indexed by the cell's base node (i0, j0, k0), so a sample reads
// one contiguous 24-value record instead of 8 node records spread over 4 rows
// of the grid.  The values and the arithmetic are those of sample().
template <typename R>
struct alignas(32) CellB {
    R v[24];
};

template <typename R>
__device__ __forceinline__ void load_cell(const CellB<R>* p, R out[24])
{
    if constexpr (sizeof(R) == 4) {
        // three 32-byte read-only loads (the record is 96 bytes, 32-byte aligned)
        const char* b = (const char*)p;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            uint32_t w[8];
            asm volatile("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]),
                           "=r"(w[7])
                         : "l"(b + 32 * q));
#pragma unroll
            for (int k = 0; k < 8; ++k) out[8 * q + k] = __uint_as_float(w[k]);
        }
    } else {
        const double2* b = (const double2*)p;
#pragma unroll
        for (int q = 0; q < 12; ++q) {
            const double2 v = __ldg(b + q);
            out[2 * q] = v.x;
            out[2 * q + 1] = v.y;
        }
    }
}

// phase_space_mu() with B read from cell records
template <typename R>
__device__ __forceinline__ R phase_space_mu_cell(R xx, R yy, R zz, R px, R py, R pz,
                                                 const CellB<R>* __restrict__ cells, const pt_grid& g)
{
    const R xmin = (R)g.xmin, ymin = (R)g.ymin, zmin = (R)g.zmin;
    const R xmax = (R)g.xmax, ymax = (R)g.ymax, zmax = (R)g.zmax;
    const R dx = (R)g.dx, dy = (R)g.dy, dz = (R)g.dz;
    R v = R(NAN);
    if (!(isnan(xx) || isnan(yy) || isnan(zz) || isnan(px) || isnan(py) || isnan(pz)) && xmin <= xx &&
        xx <= xmax && ymin <= yy && yy <= ymax && zmin <= zz && zz <= zmax) {
        Cell<R> c = locate<R>(xx, yy, zz, xmin, ymin, zmin, dx, dy, dz, g.nx, g.ny, g.nz);
        R r[24];
        load_cell(cells + c.base, r);
        const R b0 = lerp8(r[0], r[3], r[6], r[9], r[12], r[15], r[18], r[21], c);
        const R b1 = lerp8(r[1], r[4], r[7], r[10], r[13], r[16], r[19], r[22], c);
        const R b2 = lerp8(r[2], r[5], r[8], r[11], r[14], r[17], r[20], r[23], c);
        v = pitch_mu<R>(px, py, pz, b0, b1, b2);
    }
    return v;
}

}  // namespace exact
}  // namespace pt
