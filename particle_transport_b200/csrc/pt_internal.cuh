// Internal declarations shared by the libptb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <string>
#include <vector>

#include "../../include/ptb200.h"

namespace pt {

// Physical constants: src/phase_space_gpu_runner.jl:8-12.
constexpr double C_LIGHT = 2.99792458e8;
constexpr double Q_E = 1.602176634e-19;
constexpr double M_P = 1.67262192369e-27;

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define PT_CUDA(call)                                         \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return ::pt::cuda_fail(_e, #call); \
    } while (0)

#define PT_CHECK_LAUNCH(what)                                  \
    do {                                                       \
        cudaError_t _e = cudaGetLastError();                   \
        if (_e != cudaSuccess) return ::pt::cuda_fail(_e, what); \
    } while (0)

// Makes a context's device current for one entry-point call and gives the
// calling thread its own current device back on every return path, so the
// attribute queries, occupancy queries and launches of the call all target
// the device the context's stream and buffers belong to.
class DeviceScope {
public:
    explicit DeviceScope(int device)
    {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
        if (cur == device) return;
        err_ = cudaSetDevice(device);
        if (err_ == cudaSuccess) prev_ = cur;
    }
    ~DeviceScope()
    {
        if (prev_ >= 0) cudaSetDevice(prev_);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    cudaError_t error() const { return err_; }

private:
    int prev_ = -1;
    cudaError_t err_ = cudaSuccess;
};

#define PT_DEVICE_SCOPE(device)                                               \
    ::pt::DeviceScope pt_device_scope_(device);                               \
    if (pt_device_scope_.error() != cudaSuccess)                              \
    return ::pt::cuda_fail(pt_device_scope_.error(), "cudaSetDevice")

// ---------------------------------------------------------------- context
struct ScratchBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace pt

struct pt_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;      // stream used by *_device calls
    cudaStream_t copy_stream = nullptr; // egress copies in pt_push_run
    pt::ScratchBuf scratch[6];          // reusable device scratch, grown on demand
    pt::ScratchBuf pinned;              // pinned host staging of pt_push_run, grown on demand
    pt_fast_state* run_fs = nullptr;    // FP32-push state reused by pt_push_run
};

struct pt_field {
    pt_ctx* ctx = nullptr;
    int storage = PT_FIELD_REF_F64;
    pt_grid grid{};
    double B_ref = 1.0;
    // REF_F64: six column-major arrays
    double* comp[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // brick forms: node array + per-axis node offsets (in nodes)
    void* nodes = nullptr;
    int64_t n_nodes = 0;
    uint32_t* offs = nullptr;  // [nx + ny + nz]: offx, offy, offz
    int64_t bytes = 0;
    cudaTextureObject_t tex = 0;  // brick forms: node records as uint4 texels (0 if over the texture limit)
    // BF16 forms: the mean of B / B_ref per component, subtracted before the
    // rounding to BF16 and added back after the interpolation (0 otherwise)
    float boff[3] = {0.0f, 0.0f, 0.0f};
};

struct pt_fast_state {
    pt_ctx* ctx = nullptr;
    int64_t n = 0;
    double* x = nullptr;    // [3][n] positions in cell units, (x - xmin)/dx
    float* p = nullptr;     // [3][n] momentum / (m c)
    double* p2 = nullptr;   // [n] |p/(m c)|^2 carried in FP64
    int32_t* pid = nullptr; // [n] particle id of each slot
    uint8_t* alive = nullptr;
    // second copy of the state: the brick sort scatters into it and swaps
    double* x_alt = nullptr;
    float* p_alt = nullptr;
    double* p2_alt = nullptr;
    int32_t* pid_alt = nullptr;
    uint8_t* alive_alt = nullptr;
    const pt_field* field = nullptr; // field the state was created against (grid, units)
    int64_t last_sort = INT64_MIN;   // step of the last brick re-sort
    // scratch for the re-sort
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
};

namespace pt {

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Grow-only device scratch owned by the context (slot = independent user).
// Slots: 0 D_mumu, 1 D_pp, 2 pt_push_run state, 3 particle initialisation,
// 4 phase-space D_mumu (interleaved B + mu chunk).
int scratch_get(pt_ctx* ctx, int slot, size_t bytes, void** out);

// ---------------------------------------------------------------- host I/O
// Grow-only pinned host buffer of the context.
int pinned_get(pt_ctx* ctx, size_t bytes, void** out);
struct HostSeg {
    char* host;  // pageable host bytes
    char* dev;   // device bytes
    size_t bytes;
};
// Copy every segment host -> device (or device -> host) on stream s through
// nbuf pinned chunks of `chunk` bytes at `stage`, filled and drained by host
// threads while the copy engine moves the previous chunk.  Both return after
// the last byte has arrived.
int staged_h2d(const std::vector<HostSeg>& segs, char* stage, size_t chunk, int nbuf, cudaStream_t s);
int staged_d2h(const std::vector<HostSeg>& segs, char* stage, size_t chunk, int nbuf, cudaStream_t s);
int64_t count_nonzero(const uint8_t* v, int64_t n);

// ---------------------------------------------------------------- launches
struct PushArgsRef {
    const double* f[6];
    pt_grid g;
    double* x[3];
    double* p[3];
    uint8_t* alive;
    int64_t n;
    double dt;
    int64_t nsteps, stride;
    int periodic, cache_mode, cache_f64;
    int64_t step_begin, step_count;
    void* cache;
    int64_t row_base, rows;
    int64_t* deaths;
};
int launch_push_ref(const PushArgsRef& a, cudaStream_t s);

// The same FP64 push over a BRICK_F64 field: the corner values are read from
// node records in two planes (2 loads per corner) instead of 6 arrays, and the
// state may be in brick-sorted slot order with pid[slot] the particle's cache
// column.  Same arithmetic, so the results are bit-identical.
struct PushArgsExactBrick {
    const void* nodes;     // head plane: (Bx, By, Bz, ux) per node, 32 bytes
    const void* tail;      // tail plane: (uy, uz) per node, 16 bytes
    const uint32_t* offs;  // [nx + ny + nz] per-axis node offsets
    pt_grid g;
    double* x[3];
    double* p[3];
    uint8_t* alive;
    const int32_t* pid;    // cache column of each slot (null: the slot itself)
    int64_t n;
    double dt;
    int64_t nsteps, stride;
    int periodic, cache_mode, cache_f64;
    int64_t step_begin, step_count;
    void* cache;
    int64_t row_base, rows;
    int64_t* deaths;
};
int launch_push_exact_brick(const PushArgsExactBrick& a, cudaStream_t s);
// FP64 SI state in slots: xs = [6][n] (x1, x2, x3, p1, p2, p3), pid[n], alive[n]
// brick re-sort into xd/pidd/ad (hist: n_bricks + 1 buckets; cursor: the
// buckets then sort_scan_tiles() tile offsets)
int launch_exact_sort(const double* xs, const int32_t* pids, const uint8_t* as, int64_t n, const pt_field* f,
                      double* xd, int32_t* pidd, uint8_t* ad, uint32_t* hist, uint32_t* cursor, int num_sms,
                      cudaStream_t s);
// caller arrays -> slots (pid = slot), and slots -> caller arrays by pid
int launch_exact_import(double* const src[6], const uint8_t* alive, int64_t n, double* xs, int32_t* pids,
                        uint8_t* as, int num_sms, cudaStream_t s);
int launch_exact_export(const double* xs, const int32_t* pids, const uint8_t* as, int64_t n, double* const dst[6],
                        uint8_t* alive, int num_sms, cudaStream_t s);

// node record layouts of the brick forms
enum { LAYOUT_BF16 = 0, LAYOUT_F32 = 1, LAYOUT_BF16_XPAIR = 2, LAYOUT_F64 = 3 };
inline int field_layout(int storage)
{
    return storage == PT_FIELD_BRICK_F32         ? LAYOUT_F32
           : storage == PT_FIELD_BRICK_BF16_XPAIR ? LAYOUT_BF16_XPAIR
           : storage == PT_FIELD_BRICK_F64        ? LAYOUT_F64
                                                  : LAYOUT_BF16;
}
inline size_t record_bytes(int storage)
{
    return storage == PT_FIELD_BRICK_BF16 ? 16 : (storage == PT_FIELD_BRICK_F64 ? 48 : 32);
}
// brick forms read by the FP32 push
inline bool fast_storage(int storage)
{
    return storage == PT_FIELD_BRICK_F32 || storage == PT_FIELD_BRICK_BF16 || storage == PT_FIELD_BRICK_BF16_XPAIR;
}

struct FieldArgsBrick {
    const void* nodes;
    const uint32_t* offs;
    int64_t nx, ny, nz;
    int bf16;    // 1 for the BF16 forms
    int layout;  // LAYOUT_*
    cudaTextureObject_t tex;  // the node records as a linear uint4 texture (0: none)
    float boff[3];            // BF16 forms: mean field added back after the interpolation
};
struct PushArgsFast {
    FieldArgsBrick fld;
    double wx, wy, wz;     // periodic widths in cell units ((xmax-xmin)/dx)
    double* x;             // [3][n]
    float* p;              // [3][n]
    double* p2;
    int32_t* pid;
    uint8_t* alive;
    int64_t n;
    float hB;              // q B_ref dt / (2 m)
    float vfac[3];         // c dt / dx, c dt / dy, c dt / dz
    double xmin[3], dxs[3];
    int64_t nsteps, stride;
    int periodic, cache_mode, cache_f64;
    int64_t step_begin, step_count;
    void* cache;
    int64_t row_base, rows;
    int64_t* deaths;
    int variant;           // launch shape, see pt_push_params.kernel_variant
    int ring;              // 1: save row r goes to cache row r % rows
    int64_t n_cache;       // particles per cache row
    float* mom_cache;      // with a mu cache: momenta rows [rows][3][n_mom] of particles pid < n_mom, or null
    int64_t n_mom;
    int64_t pitch;         // mu cache: 0 = rows [r][n_cache]; > 0 = time-fastest, element r of pid at pid * pitch + r
};
int launch_push_fast(const PushArgsFast& a, cudaStream_t s);

// ---------------------------------------------------------------- batches
// A batch is an arena of particle slots shared by many campaigns (each a
// contiguous slot range with its own field, dt, step counter and cache).
// Campaigns sort on their own cadence (every sort_every-th epoch they run),
// so each keeps its slots in its own buffer of the ping-pong pair (par); the
// fields step, epochs and par are owned by the device (advanced by the
// epochs), the others by the host.
struct BatchCampaignDev {
    PushArgsFast a;      // per-campaign constants (state pointers unused)
    int64_t slot0, n;    // slot range in the arena (the same in both buffers)
    int64_t step, K;     // next step; steps per epoch
    int64_t key_base;    // first sort bucket
    int64_t n_bricks;    // bricks of the campaign's field (bucket n_bricks = dead)
    int64_t dense_base;  // sort position of the campaign's first bucket in the current epoch
    int64_t epochs;      // epochs run so far
    int32_t sort_every;  // re-sorted before every sort_every-th epoch it runs (0: never)
    int32_t par;         // buffer (0/1) holding the campaign's slots
    int32_t active;      // holds particles
    int32_t running;     // pushed, sorted and stepped by the epochs (0: paused, slots held as they are)
};
// Whether campaign C is re-sorted before its next epoch.
__host__ __device__ inline bool batch_sort_due(const BatchCampaignDev& C)
{
    return C.active && C.running && C.sort_every > 0 && C.step < C.a.nsteps && C.epochs % C.sort_every == 0;
}
constexpr int kBatchTile = 256;  // particles per tile of a batch (= block size of its kernels)
struct BatchTile {
    int32_t campaign;
    int32_t count;
    int64_t begin;     // first slot of the tile (arena index)
};
struct BatchStateDev {
    double* x;         // [3][cap]
    float* p;          // [3][cap]
    double* p2;
    int32_t* pid;      // campaign-local particle index
    uint8_t* alive;
    int64_t cap;
};
struct BatchLaunch {
    const BatchCampaignDev* camps;
    const BatchTile* tiles;
    const int* n_tiles;
    int* tile_counter;
    BatchStateDev st[2];
    int sorted;        // the epoch re-sorted the due campaigns into their other buffer
    int layout;        // LAYOUT_* shared by the batch's fields
    int smem_words;    // max (nx + ny + nz) over the batch's fields
    int grid;
    int threads;       // threads per block of the push: 64, 128 or kBatchTile (particles per thread = kBatchTile / threads)
};
int launch_push_batch(const BatchLaunch& L, cudaStream_t s);
int launch_batch_apply(BatchCampaignDev* camps, const BatchCampaignDev* staged, int n_camps, int fresh,
                       cudaStream_t s);
int launch_batch_epoch_end(BatchCampaignDev* camps, int n_camps, int* tile_counter, int sorted, cudaStream_t s);
// buckets per tile of the two-level bucket scan of the brick sorts, and the
// number of tile offsets that follow the cursor array of m buckets
constexpr int64_t kSortScanTile = 2048;
inline int64_t sort_scan_tiles(int64_t m) { return (m + kSortScanTile - 1) / kSortScanTile; }
// cursor must hold max_buckets + sort_scan_tiles(max_buckets) entries
int launch_batch_sort(BatchCampaignDev* camps, int n_camps, const BatchTile* tiles, const int* n_tiles, int grid,
                      BatchStateDev st0, BatchStateDev st1, uint32_t* keys, uint32_t* hist, uint32_t* cursor,
                      const int64_t* d_m, int64_t max_buckets, int num_sms, cudaStream_t s);
int launch_batch_import(BatchStateDev st, int64_t slot0, int64_t n, const pt_field* f, const double* x1,
                        const double* x2, const double* x3, const double* p1, const double* p2, const double* p3,
                        const uint8_t* alive, int num_sms, cudaStream_t s);
// reads the campaign's buffer parity from camps[id] on the device
int launch_batch_export(BatchStateDev st0, BatchStateDev st1, const BatchCampaignDev* camps, int id, int64_t slot0,
                        int64_t n, const pt_field* f, double* x1, double* x2, double* x3, double* p1, double* p2,
                        double* p3, uint8_t* alive, int num_sms, cudaStream_t s);
int launch_fast_import(pt_fast_state* st, const pt_field* f, const double* x1, const double* x2, const double* x3,
                       const double* p1, const double* p2, const double* p3, const uint8_t* alive, cudaStream_t s);
int launch_fast_export(const pt_fast_state* st, const pt_field* f, double* x1, double* x2, double* x3, double* p1,
                       double* p2, double* p3, uint8_t* alive, cudaStream_t s);
int fast_sort(pt_ctx* ctx, pt_fast_state* st, const pt_field* f, cudaStream_t s);

int launch_brick_convert(const double* const comps[6], const pt_grid& g, double B_ref, int layout, void* nodes,
                         const uint32_t* offs, int64_t n_nodes, const float boff[3], cudaStream_t s);
// rows [rows][n] of a time-fastest mu cache [n][pitch] (save r of particle p
// at p * pitch + r), for the row-by-row egress of pt_push_run
int launch_tf_to_rows(const float* tf, int64_t n, int pitch, int rows, float* out, cudaStream_t s);
// mean of the finite values of each of the three B components (device
// arrays of nn values; 0 when none is finite), summed in a fixed order (the
// same bits on every call); waits for the stream
int field_means(pt_ctx* ctx, const double* const comps[6], int64_t nn, double mean[3], cudaStream_t s);

struct DmumuArgs {
    const float* mu;
    int64_t n, nsave, sp, ss;
    const int64_t* lags;
    int n_lags;
    const double* edges;
    int n_bins;
    int injection, bin_abs;
    int64_t* counts;
    double* sum_d;
    double* sum_d2;
    int64_t* w_count;
    double* w_mean;
    double* w_m2;
    double* pair_ss;
    int64_t* pair_n;
};
int run_dmumu(pt_ctx* ctx, const DmumuArgs& a, cudaStream_t s);
// D_mumu of a phase-space chunk (a.mu, a.sp, a.ss unused): mu reconstructed
// on the device into a scratch chunk, then binned; component c of save s of
// particle p at pos/mom + s * row + c * comp + p, elements and B in the
// compute precision.
int run_dmumu_phase_space(pt_ctx* ctx, const DmumuArgs& a, const void* pos, const void* mom, int64_t row,
                          int64_t comp, const void* const bfield[3], const pt_grid& g, int f64, cudaStream_t s);

struct DppArgs {
    const float* mom;
    int64_t chunk, nsave;
    const int64_t* lags;
    int n_lags;
    double p0;
    int64_t* counts;
    double *sdp, *sdp2, *sdn, *sdn2;
};
int run_dpp(pt_ctx* ctx, const DppArgs& a, cudaStream_t s);
int launch_energy_snapshots(const float* mom, int64_t chunk, int64_t nsave, const int64_t* snaps, int n_snap,
                            int64_t offset, double* out, cudaStream_t s);
int launch_energy_histogram(const float* mom, int64_t chunk, int64_t nsave, const int64_t* snaps, int n_snap,
                            double e_min, double e_max, int n_hist, int64_t* counts, cudaStream_t s);
int launch_reconstruct_mu(const void* pos, const void* mom, int64_t chunk, int64_t nsave, const void* const b[3],
                          const pt_grid& g, int f64, void* mu_out, cudaStream_t s);

}  // namespace pt
