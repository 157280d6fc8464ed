// Particle initialisation on the device: the formulas of init_particles,
// rand_unit_vector and fixed_mu_unit_vector
// (src/phase_space_gpu_runner.jl:51-66, 170-245) over a counter-based
// SplitMix64 stream, one thread per particle.
//
// Compiled with --fmad=false: every product and sum is rounded on its own in
// the order the reference writes it, so a host restatement of the same stream
// gives identical positions and B samples; only cos/sin may differ in the
// last bits.
#include <cmath>

#include "pt_internal.cuh"

namespace pt {
namespace {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;
constexpr double TWO_PI = 6.283185307179586;  // Float64(2 * pi)
constexpr double GEV_TO_J = 1e9 * 1.602176634e-19;

// SplitMix64 finaliser (Steele, Lea, Flood 2014; constants of Vigna's splitmix64.c)
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ inline double draw(uint64_t key, int64_t i, int d)
{
    const uint64_t c = (uint64_t)i * 8u + (uint64_t)d + 1u;
    return (double)(mix64(key + c * GOLDEN) >> 11) * 0x1.0p-53;
}

struct InitArgs {
    int64_t n;
    uint64_t key;
    double lo[3], len[3], fixed[3];
    int random_pos, fixed_mu;
    double mu0, perp, pscale;
    // field for fixed mu
    int storage;
    const double* B[3];   // PT_FIELD_REF_F64
    const void* nodes;    // brick forms
    const uint32_t* offs;
    float boff[3];        // BF16 forms: the mean field the nodes are stored less
    pt_grid g;
    double* out[6];
    int* bad;
};

// component c (0..2) of B at node (i, j, k) as stored by the field
__device__ inline double node_B(const InitArgs& a, int64_t i, int64_t j, int64_t k, int c)
{
    if (a.storage == PT_FIELD_REF_F64) return a.B[c][(k * a.g.ny + j) * a.g.nx + i];
    const uint32_t node = a.offs[i] + a.offs[a.g.nx + j] + a.offs[a.g.nx + a.g.ny + k];
    if (a.storage == PT_FIELD_BRICK_F64) return ((const double*)a.nodes)[4 * (size_t)node + c];  // SI head plane
    if (a.storage == PT_FIELD_BRICK_F32) return (double)((const float*)a.nodes)[8 * (size_t)node + c];
    const size_t words = a.storage == PT_FIELD_BRICK_BF16 ? 4 : 8;  // 16 B records or 32 B x-pair records
    const uint32_t w = ((const uint32_t*)a.nodes)[words * node + (c >> 1)];
    return (double)__uint_as_float((c & 1) ? (w & 0xFFFF0000u) : (w << 16)) + (double)a.boff[c];
}

// trilinear_sample, src/phase_space_gpu_runner.jl:247-276 (x, then y, then z lerps)
__device__ double sample_B(const InitArgs& a, int c, double x, double y, double z)
{
    const pt_grid& g = a.g;
    const double fx = (x - g.xmin) / g.dx + 1.0;
    const double fy = (y - g.ymin) / g.dy + 1.0;
    const double fz = (z - g.zmin) / g.dz + 1.0;
    const double i0 = fmin(fmax(floor(fx), 1.0), (double)(g.nx - 1));
    const double j0 = fmin(fmax(floor(fy), 1.0), (double)(g.ny - 1));
    const double k0 = fmin(fmax(floor(fz), 1.0), (double)(g.nz - 1));
    const double tx = fx - i0, ty = fy - j0, tz = fz - k0;
    const int64_t i = (int64_t)i0 - 1, j = (int64_t)j0 - 1, k = (int64_t)k0 - 1;
    const double c000 = node_B(a, i, j, k, c), c100 = node_B(a, i + 1, j, k, c);
    const double c010 = node_B(a, i, j + 1, k, c), c110 = node_B(a, i + 1, j + 1, k, c);
    const double c001 = node_B(a, i, j, k + 1, c), c101 = node_B(a, i + 1, j, k + 1, c);
    const double c011 = node_B(a, i, j + 1, k + 1, c), c111 = node_B(a, i + 1, j + 1, k + 1, c);
    const double c00 = c000 * (1.0 - tx) + c100 * tx;
    const double c10 = c010 * (1.0 - tx) + c110 * tx;
    const double c01 = c001 * (1.0 - tx) + c101 * tx;
    const double c11 = c011 * (1.0 - tx) + c111 * tx;
    const double c0 = c00 * (1.0 - ty) + c10 * ty;
    const double c1 = c01 * (1.0 - ty) + c11 * ty;
    return c0 * (1.0 - tz) + c1 * tz;
}

__global__ void init_particles_kernel(InitArgs a)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        double x[3];
        for (int d = 0; d < 3; ++d)
            x[d] = a.random_pos ? draw(a.key, i, d) * a.len[d] + a.lo[d] : a.fixed[d];
        double ux, uy, uz;
        if (a.fixed_mu) {
            // fixed_mu_unit_vector, src/phase_space_gpu_runner.jl:170-194
            const double bx = sample_B(a, 0, x[0], x[1], x[2]);
            const double by = sample_B(a, 1, x[0], x[1], x[2]);
            const double bz = sample_B(a, 2, x[0], x[1], x[2]);
            const double bn = sqrt(bx * bx + by * by + bz * bz);
            if (!isfinite(bn) || bn == 0.0) {
                atomicAdd(a.bad, 1);
                ux = uy = uz = nan("");
            } else {
                const double bhx = bx / bn, bhy = by / bn, bhz = bz / bn;
                double e1x, e1y, e1z;
                if (fabs(bhx) < 0.9) {
                    e1x = 0.0; e1y = bhz; e1z = -bhy;
                } else {
                    e1x = -bhz; e1y = 0.0; e1z = bhx;
                }
                const double e1n = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
                e1x = e1x / e1n; e1y = e1y / e1n; e1z = e1z / e1n;
                const double e2x = bhy * e1z - bhz * e1y;
                const double e2y = bhz * e1x - bhx * e1z;
                const double e2z = bhx * e1y - bhy * e1x;
                const double phi = TWO_PI * draw(a.key, i, 3);
                const double cphi = cos(phi), sphi = sin(phi);
                ux = a.mu0 * bhx + a.perp * (cphi * e1x + sphi * e2x);
                uy = a.mu0 * bhy + a.perp * (cphi * e1y + sphi * e2y);
                uz = a.mu0 * bhz + a.perp * (cphi * e1z + sphi * e2z);
            }
        } else {
            // rand_unit_vector, src/phase_space_gpu_runner.jl:61-66
            const double z = 2.0 * draw(a.key, i, 3) - 1.0;
            const double phi = TWO_PI * draw(a.key, i, 4);
            const double r = sqrt(fmax(0.0, 1.0 - z * z));
            ux = r * cos(phi);
            uy = r * sin(phi);
            uz = z;
        }
        a.out[0][i] = x[0];
        a.out[1][i] = x[1];
        a.out[2][i] = x[2];
        a.out[3][i] = a.pscale * ux;
        a.out[4][i] = a.pscale * uy;
        a.out[5][i] = a.pscale * uz;
    }
}

}  // namespace
}  // namespace pt

using namespace pt;

extern "C" int pt_particles_init_device(pt_ctx* ctx, const pt_field* field, const pt_init_params* prm, double* d_x1,
                                        double* d_x2, double* d_x3, double* d_p1, double* d_p2, double* d_p3)
{
    if (!ctx || !field || !prm) return fail(PT_ERR_ARG, "null argument");
    if (prm->n < 0) return fail(PT_ERR_ARG, "n must be >= 0");
    if (prm->injection != PT_INJECT_ISOTROPIC && prm->injection != PT_INJECT_FIXED_MU)
        return fail(PT_ERR_ARG, "injection_mode must be isotropic or fixed-mu");
    if (prm->position_mode != PT_POSITION_RANDOM && prm->position_mode != PT_POSITION_FIXED)
        return fail(PT_ERR_ARG, "injection_position_mode must be random or fixed");
    if (prm->injection == PT_INJECT_FIXED_MU && !(-1.0 <= prm->mu0 && prm->mu0 <= 1.0))
        return fail(PT_ERR_ARG, "injection_mu0 must be in [-1, 1]");
    if (!(std::isfinite(prm->energy_GeV) && prm->energy_GeV > 0.0)) return fail(PT_ERR_ARG, "energy must be > 0");
    if (prm->n == 0) return PT_OK;
    if (!(d_x1 && d_x2 && d_x3 && d_p1 && d_p2 && d_p3)) return fail(PT_ERR_ARG, "null pointer");

    InitArgs a{};
    const pt_grid& g = field->grid;
    a.n = prm->n;
    a.key = mix64(prm->seed);
    const double lo[3] = {g.xmin, g.ymin, g.zmin}, hi[3] = {g.xmax, g.ymax, g.zmax};
    for (int d = 0; d < 3; ++d) {
        a.lo[d] = lo[d];
        a.len[d] = hi[d] - lo[d];
        // fixed_injection_position, box-fraction unit (src/phase_space_gpu_runner.jl:145-167)
        a.fixed[d] = lo[d] + prm->position[d] * (hi[d] - lo[d]);
        if (prm->position_mode == PT_POSITION_FIXED && !(lo[d] <= a.fixed[d] && a.fixed[d] <= hi[d]))
            return fail(PT_ERR_ARG, "fixed injection position is outside the simulation box");
    }
    a.random_pos = prm->position_mode == PT_POSITION_RANDOM;
    a.fixed_mu = prm->injection == PT_INJECT_FIXED_MU;
    a.mu0 = prm->mu0;
    a.perp = std::sqrt(std::max(0.0, 1.0 - prm->mu0 * prm->mu0));
    // energy_to_gamma / energy_to_speed (src/phase_space_gpu_runner.jl:51-59), pscale = gamma0 m v0 (:210)
    const double kinetic = prm->energy_GeV * GEV_TO_J;
    const double gamma0 = kinetic / (M_P * (C_LIGHT * C_LIGHT)) + 1.0;
    const double v0 = C_LIGHT * std::sqrt(1.0 - 1.0 / (gamma0 * gamma0));
    a.pscale = gamma0 * M_P * v0;
    a.storage = field->storage;
    for (int c = 0; c < 3; ++c) a.B[c] = field->comp[c];
    a.nodes = field->nodes;
    a.offs = field->offs;
    for (int c = 0; c < 3; ++c) a.boff[c] = field->boff[c];
    a.g = g;
    double* outs[6] = {d_x1, d_x2, d_x3, d_p1, d_p2, d_p3};
    for (int c = 0; c < 6; ++c) a.out[c] = outs[c];

    PT_DEVICE_SCOPE(ctx->device);
    int* d_bad = nullptr;
    int rc = scratch_get(ctx, 3, sizeof(int), (void**)&d_bad);
    if (rc) return rc;
    a.bad = d_bad;
    cudaStream_t s = ctx->stream;
    PT_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    const int threads = 256;
    const int64_t want = (prm->n + threads - 1) / threads;
    const int blocks = (int)std::min<int64_t>(want, (int64_t)ctx->num_sms * 16);
    init_particles_kernel<<<blocks, threads, 0, s>>>(a);
    PT_CHECK_LAUNCH("init_particles_kernel");
    int bad = 0;
    PT_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    PT_CUDA(cudaStreamSynchronize(s));
    if (bad) return fail(PT_ERR_ARG, "cannot use fixed-mu injection where local B is zero or non-finite");
    return PT_OK;
}
