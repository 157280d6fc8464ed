/*
 * ptb200.h -- C ABI of libptb200.so, the B200 (sm_100a) implementation of the
 * trajectory and transport-statistics hot path of particle_transport.
 *
 * The reference has no FFI layer: its hot path sits behind Julia functions.
 * Each entry point below names the reference function (file:line, paths in
 * the reference project) whose body it replaces; the Julia host keeps the
 * function's signature, its HDF5 I/O and its config handling and calls the
 * library through ccall (see INTEGRATION.md for the bindings).
 *
 * Conventions
 *  - Every function returns PT_OK (0) or a negative PT_ERR_* code; the
 *    message of the last failure on the calling thread is pt_last_error().
 *  - Host arrays are owned by the caller and use the reference's Julia
 *    (column-major) layouts, spelled out per argument below.  The library
 *    never frees caller memory.  Device memory lives behind opaque handles.
 *  - Statistics accumulators are add-into, like the reference's `+=` across
 *    particle chunks; per-lag Welford triples are merged with the reference's
 *    combine_welford_stats! formula (Chan et al.).
 *  - NaN marks dead or invalid samples, exactly as in the reference.
 *  - A pt_ctx is not re-entrant: use one per host thread / Julia task.
 *    Calls are synchronous unless their name ends in _device (those enqueue
 *    on the context stream and take device pointers).
 */
#ifndef PTB200_H
#define PTB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTB200_VERSION 1

enum {
    PT_OK = 0,
    PT_ERR_ARG = -1,      /* invalid argument (null, size, range)                 */
    PT_ERR_CUDA = -2,     /* CUDA runtime failure                                 */
    PT_ERR_OOM = -3,      /* device allocation failed / over the device budget    */
    PT_ERR_TIMEOUT = -4,  /* a bounded device-side wait gave up                    */
    PT_ERR_CALLBACK = -5, /* the caller's save callback returned non-zero          */
    PT_ERR_STATE = -6     /* object used in the wrong state                        */
};

/* field storage on the device */
enum {
    PT_FIELD_REF_F64 = 0, /* six column-major Float64 arrays, SI units (parity form)        */
    PT_FIELD_BRICK_F32 = 1, /* Morton 8^3 bricks, 6 comps interleaved per node, Float32      */
    PT_FIELD_BRICK_BF16 = 2, /* Morton 8^3 bricks, 6 comps interleaved per node, bfloat16;
                                B is stored less its grid mean per component (computed at
                                upload), which the push adds back after the interpolation */
    PT_FIELD_BRICK_BF16_XPAIR = 3, /* as BF16, each 32-byte record holds a node and its +x neighbour:
                                      the 8 corners of a cell are 4 x 32-byte loads          */
    PT_FIELD_BRICK_F64 = 4 /* Morton 8^3 bricks of Float64 SI values in two planes: (Bx, By, Bz, ux)
                              32 bytes and (uy, uz) 16 bytes per node.  The FP64 push reads the
                              same values as from REF_F64 (bit-identical results), 2 loads per
                              corner                                                       */
};

/* cache written at every save step (pre-push state) */
enum { PT_CACHE_NONE = 0, PT_CACHE_MU = 1, PT_CACHE_PHASE_SPACE = 2 };

/* push arithmetic */
enum { PT_PUSH_F64 = 0, PT_PUSH_F32 = 1 };

/* D_mumu estimator (dmumu_start_mode) */
enum { PT_START_SLIDING = 0, PT_START_INJECTION = 1 };

typedef struct pt_ctx pt_ctx;
typedef struct pt_field pt_field;

/* Node grid: nodes at xmin + i*dx, i = 0..nx-1 (reference build_uniform_coords,
 * src/phase_space_gpu_runner.jl:125-130: xmin = x[1], xmax = x[end],
 * dx = x[2] - x[1]). */
typedef struct {
    int64_t nx, ny, nz;
    double xmin, ymin, zmin;
    double xmax, ymax, zmax;
    double dx, dy, dz;
} pt_grid;

typedef struct {
    double dt;                /* integration step [s] (trajectory_time.dt_s)            */
    int64_t nsteps;           /* integration samples; nsteps-1 pushes                   */
    int64_t stride;           /* save stride; saves at steps 0, stride, ... (0-based)   */
    int32_t periodic;         /* 1: wrap positions, 0: open boundary (kill on exit)     */
    int32_t cache_mode;       /* PT_CACHE_*                                             */
    int32_t cache_f64;        /* 0: Float32 cache (reference default), 1: Float64       */
    int32_t precision;        /* PT_PUSH_F64 (REF_F64 field) or PT_PUSH_F32 (bricks)    */
    int32_t steps_per_launch; /* steps kept in registers per launch; 0 = auto           */
    int32_t sort_every;       /* F32 form: re-sort particles by brick every N steps; 0 off */
    int32_t kernel_variant;   /* F32 form: launch shape, threads per block x resident
                                 blocks per SM: 0 = auto (= 1), 1 = 256 x occupancy,
                                 2 = 256 x 4, 3 = 128 x 8, 4 = 512 x 2, 5 = 256 x 1,
                                 6 = 512 x 1, 7 = 128 x 3, 8 = 128 x 2; BRICK_BF16
                                 fields: 9 = as 1 with half of the corners fetched
                                 through the texture path, 10 = as 1 with all of
                                 them, 11 = as 6 with half (same results)       */
    int32_t cache_pitch;      /* mu caches of the F32 form (pt_push_advance_fast): 0 = rows,
                                 save row r of particle p at (r - cache_row_base) * n + p (the
                                 reference's on-disk layout); > 0 = time-fastest, at
                                 p * cache_pitch + (r - cache_row_base) (the Julia mu_chunk
                                 layout, sp = cache_pitch, ss = 1 for pt_dmumu_accumulate*),
                                 cache_pitch >= cache_rows.  The saves of a particle then sit side
                                 by side and are written by one thread within microseconds, so L2
                                 merges them into whole 32-byte DRAM sectors, where rows (the
                                 particles in brick order) cost a sector per 4-byte save.  Must
                                 be 0 elsewhere.                                                */
} pt_push_params;

/* Save sink for pt_push_run: called on the calling thread once per save row,
 * in save order.  data holds the row in the cache layout of the reference
 * writers: mu: n values (src/multimode_multienergy_cache_pipeline.jl:1318-1321);
 * phase space: positions[3][n] then momenta[3][n]
 * (src/phase_space_gpu_runner.jl:413-421).  Return non-zero to abort. */
typedef int (*pt_save_fn)(void* user, int64_t save_index, const void* data, int64_t nbytes);

const char* pt_last_error(void);
int pt_version(void);

int pt_ctx_create(int device, pt_ctx** out);
int pt_ctx_destroy(pt_ctx* ctx);
/* Use the given cudaStream_t for all *_device entry points: NULL selects the
 * library's own (non-blocking) stream; pass cudaStreamLegacy ((void*)0x1)
 * for the legacy default stream. */
int pt_ctx_set_stream(pt_ctx* ctx, void* cuda_stream);
int pt_ctx_synchronize(pt_ctx* ctx);
/* Free the buffers a context keeps between calls: device scratch, the pinned
 * host staging and the particle state of pt_push_run (all grow-only, reused
 * by the next call of the same size).  pt_ctx_destroy frees them too.  No
 * reference counterpart (the reference allocates per run). */
int pt_ctx_trim(pt_ctx* ctx);

/* Upload a static field library (load_static_fields output,
 * src/phase_space_gpu_runner.jl:95-123; SI units: B in T, u in m/s).
 * comps = {Bx, By, Bz, ux, uy, uz}, each nx*ny*nz doubles, x fastest.
 * storage = PT_FIELD_*; B_ref_T scales the nondimensional brick forms
 * (B stored as B/B_ref_T, u as u/c); it is ignored for REF_F64. */
int pt_field_upload(pt_ctx* ctx, const double* const comps[6], const pt_grid* grid, int storage,
                    double B_ref_T, pt_field** out);
/* Same, from device pointers (e.g. fields generated on the GPU). */
int pt_field_upload_device(pt_ctx* ctx, const double* const d_comps[6], const pt_grid* grid, int storage,
                           double B_ref_T, pt_field** out);
int pt_field_destroy(pt_field* field);
int64_t pt_field_device_bytes(const pt_field* field);

/*
 * Whole-ensemble push with host state: replaces the body of
 *   run_gpu_ensemble       src/phase_space_gpu_runner.jl:476 (lines 506-592)
 *   run_mu_cache_ensemble  src/multimode_multienergy_cache_pipeline.jl:1380 (lines 1410-1500)
 * x1..p3: n doubles each (SI), updated in place to the final state; alive: n
 * bytes (1 live), updated in place.  Each save row is handed to `save` on the
 * calling thread while the next steps run on the GPU.  alive_count[nsteps]
 * receives sum(dalive) after each step (src/phase_space_gpu_runner.jl:576).
 * The state crosses the link through the context's pinned staging chunks
 * (host threads copy while the DMA engine moves the previous chunk); the
 * device state, staging and the FP32-push state stay in the context for the
 * next call (pt_ctx_trim releases them).  The FP32 push with a Float32 mu
 * cache writes each 64-step chunk's saves time-fastest on the device and
 * transposes them to rows before the egress (two slots of up to 8 rows of
 * n floats, device and pinned, plus the [n][8] buffer).
 */
int pt_push_run(pt_ctx* ctx, const pt_field* field, double* x1, double* x2, double* x3, double* p1, double* p2,
                double* p3, uint8_t* alive, int64_t n, const pt_push_params* params, pt_save_fn save, void* user,
                int64_t* alive_count);

/*
 * Device-resident push of steps [step_begin, step_begin + step_count) on the
 * context stream (advance_particles_kernel!, src/phase_space_gpu_runner.jl:330-391,
 * fused with reconstruct_mu_step_kernel!, pipeline:1349-1374).
 * PT_PUSH_F64: d_x1..d_p3 are the SI Float64 state (n each).
 * PT_PUSH_F32: the state is a pt_fast_state created by pt_fast_state_create
 *   and d_x1..d_p3 must be NULL (pass the state via pt_push_advance_fast).
 * Save rows r in [cache_row_base, cache_row_base + cache_rows) are written to
 * d_cache + (r - cache_row_base) * row_elems (mu: n elements; phase space:
 * 6n, positions then momenta).  d_deaths[nsteps] (int64, may be NULL)
 * counts particles killed at each step (open boundary).
 */
int pt_push_advance_device(pt_ctx* ctx, const pt_field* field, double* d_x1, double* d_x2, double* d_x3,
                           double* d_p1, double* d_p2, double* d_p3, uint8_t* d_alive, int64_t n,
                           const pt_push_params* params, int64_t step_begin, int64_t step_count, void* d_cache,
                           int64_t cache_row_base, int64_t cache_rows, int64_t* d_deaths);

/* Mixed-precision state (FP32 momentum, FP64 positions in cell units, FP64
 * |p|^2 per particle, particle ids and optional brick sort).  Converts from /
 * to the SI Float64 state. */
typedef struct pt_fast_state pt_fast_state;
int pt_fast_state_create(pt_ctx* ctx, const pt_field* field, const double* d_x1, const double* d_x2,
                         const double* d_x3, const double* d_p1, const double* d_p2, const double* d_p3,
                         const uint8_t* d_alive, int64_t n, pt_fast_state** out);
int pt_fast_state_export(pt_ctx* ctx, const pt_fast_state* st, double* d_x1, double* d_x2, double* d_x3,
                         double* d_p1, double* d_p2, double* d_p3, uint8_t* d_alive);
int pt_fast_state_destroy(pt_fast_state* st);
/* Re-sort the particle slots by the brick holding their cell (one-digit
 * radix / counting sort); results do not depend on the slot order.  Runs on
 * the context stream.  No reference counterpart (the reference keeps the
 * particles in index order). */
int pt_fast_state_sort(pt_ctx* ctx, pt_fast_state* st);
int pt_push_advance_fast(pt_ctx* ctx, const pt_field* field, pt_fast_state* st, const pt_push_params* params,
                         int64_t step_begin, int64_t step_count, void* d_cache, int64_t cache_row_base,
                         int64_t cache_rows, int64_t* d_deaths);

/*
 * Batched campaigns.  A batch is an arena of particle slots on one device
 * holding many campaigns (mode x energy, or jobs of a server), each with its
 * own field, dt, step count, save stride and mu cache.  One persistent
 * kernel advances every campaign by steps_per_epoch steps per epoch
 * (finished campaigns idle); with sort = 1 each campaign's slots are
 * re-sorted by brick before every sort_every-th epoch it runs.  Epochs run as CUDA graphs (one
 * per sort buffer parity) when use_graph = 1.  Campaigns can be added and
 * removed between epochs.  A particle's trajectory and cache rows are
 * bit-identical to a single-campaign pt_push_advance_fast run.
 * No reference counterpart: the reference runs campaigns one after another
 * (run_mode_campaigns, src/multimode_multienergy_cache_pipeline.jl:2924).
 */
typedef struct pt_batch pt_batch;

typedef struct {
    const pt_field* field;     /* brick field (all campaigns of a batch share its storage type) */
    double dt;                 /* integration step of this campaign [s]                      */
    int64_t nsteps;            /* samples; nsteps - 1 pushes                                  */
    int64_t stride;            /* save stride                                                */
    int32_t periodic;
    int32_t cache_f64;         /* 0: Float32 mu cache                                        */
    int64_t n;                 /* particles                                                  */
    const double* d_x1;        /* initial SI state on the device (n each)                    */
    const double* d_x2;
    const double* d_x3;
    const double* d_p1;
    const double* d_p2;
    const double* d_p3;
    const uint8_t* d_alive;
    void* d_cache;             /* mu cache of cache_rows saves (NULL: no cache), laid out as
                                  cache_pitch says                                          */
    int64_t cache_rows;
    int32_t cache_ring;        /* 1: save row r goes to row r % cache_rows                   */
    int32_t sort_every;        /* re-sort this campaign's slots by brick before every sort_every-th
                                  epoch it runs (0 or 1: every epoch); batches made with sort = 0
                                  never sort.  Fast particles lose their brick order within a few
                                  steps and gain from frequent sorts, slow ones do not.          */
    int64_t* d_deaths;         /* [nsteps] particles killed per step (open boundary), or NULL */
    float* d_mom_cache;        /* with d_cache: momenta rows [cache_rows][3][n_mom] (Float32, SI, the
                                  phase-space writer's momenta, src/phase_space_gpu_runner.jl:413-421)
                                  of particles 0 .. n_mom-1 -- the D_pp subset -- or NULL */
    int64_t n_mom;
    int64_t cache_pitch;       /* 0: mu rows [cache_rows][n]; > 0: time-fastest, save row r of
                                  particle p at p * cache_pitch + r (ring: r % cache_rows),
                                  cache_pitch >= cache_rows (see pt_push_params.cache_pitch) */
} pt_campaign_desc;

/* capacity: particle slots; blocks_per_sm: resident blocks of the persistent
 * kernel per SM (0 = 2). */
int pt_batch_create(pt_ctx* ctx, int64_t capacity, int max_campaigns, int storage, int steps_per_epoch, int sort,
                    int blocks_per_sm, pt_batch** out);
int pt_batch_add(pt_ctx* ctx, pt_batch* batch, const pt_campaign_desc* campaign, int* id);
int pt_batch_remove(pt_ctx* ctx, pt_batch* batch, int id);
/* Run `epochs` epochs on the context stream (asynchronous). */
int pt_batch_run(pt_ctx* ctx, pt_batch* batch, int64_t epochs, int use_graph);
/* Choose which campaigns the following epochs advance: exactly ids[0 .. n_ids)
 * (n_ids = -1: every campaign).  A paused campaign keeps its slots, step
 * counter and caches as they are; the sort leaves its slots alone, and it
 * continues from the same step when it runs again, so its trajectory is the
 * one it would have had running throughout.  New campaigns (pt_batch_add)
 * run.  The campaign server uses this to give its epochs to the jobs with
 * the least work left.  No reference counterpart (the reference has no
 * serving mode). */
int pt_batch_set_running(pt_ctx* ctx, pt_batch* batch, const int* ids, int n_ids);
/* Launch shape of the batch's persistent push kernel: threads_per_block
 * (64, 128 or 256) and resident blocks per SM (1..16).  A tile holds 256
 * particles; each thread advances 256 / threads_per_block of them, one after
 * another.  Results do not depend on the shape.  The tuner of the Python
 * host (batch.tune_batch) picks it with the steps per epoch and the sort
 * cadences.  No reference counterpart. */
int pt_batch_set_launch(pt_ctx* ctx, pt_batch* batch, int threads_per_block, int blocks_per_sm);
/* Next step of campaign `id` (synchronises the context stream). */
int pt_batch_step(pt_ctx* ctx, pt_batch* batch, int id, int64_t* step);
/* Copy campaign `id`'s state back to SI device arrays (n each). */
int pt_batch_export(pt_ctx* ctx, pt_batch* batch, int id, double* d_x1, double* d_x2, double* d_x3, double* d_p1,
                    double* d_p2, double* d_p3, uint8_t* d_alive);
int pt_batch_destroy(pt_batch* batch);

/*
 * D_mumu / <dmu^2> lag-pair accumulation: replaces process_mu_chunk_dmumu_cpu!
 *   src/compute_delta_mu2_dmumu_full.jl:656 (sliding :457-560, injection :562-654),
 * called from pipeline:1718 and dmumu:1150.
 * mu: Float32, element (particle p, save s) at mu[p*sp + s*ss]; the Julia
 *   mu_chunk (nsave, chunk) is sp = nsave, ss = 1; the device mu cache
 *   [nsave][n] is sp = 1, ss = n.
 * lag_steps[n_lags]: save offsets (same in 0- and 1-based indexing).
 * mu_edges[n_bins+1]: the Float64 edges of build_mu_edges_full (dmumu:289-302).
 * counts/sum_d/sum_d2: Julia (n_bins, n_lags) = [lag][bin], add-into.
 * w_count/w_mean/w_m2/pair_ss/pair_n: [n_lags], merged / added into.
 * Host pointers (synchronous).
 */
int pt_dmumu_accumulate(pt_ctx* ctx, const float* mu, int64_t n, int64_t nsave, int64_t sp, int64_t ss,
                        const int64_t* lag_steps, int n_lags, const double* mu_edges, int n_bins, int start_mode,
                        int bin_abs, int64_t* counts, double* sum_d, double* sum_d2, int64_t* w_count,
                        double* w_mean, double* w_m2, double* pair_ss, int64_t* pair_n);
/* Same with device pointers for mu, lag_steps, mu_edges and all accumulators
 * (enqueued on the context stream). */
int pt_dmumu_accumulate_device(pt_ctx* ctx, const float* d_mu, int64_t n, int64_t nsave, int64_t sp, int64_t ss,
                               const int64_t* d_lag_steps, int n_lags, const double* d_mu_edges, int n_bins,
                               int start_mode, int bin_abs, int64_t* d_counts, double* d_sum_d, double* d_sum_d2,
                               int64_t* d_w_count, double* d_w_mean, double* d_w_m2, double* d_pair_ss,
                               int64_t* d_pair_n);

/*
 * Fused phase-space D_mumu: the body of the phase-space branch of the D_mumu
 * driver (src/compute_delta_mu2_dmumu_full.jl:1137-1164) on the device --
 * reconstruct_mu_chunk_gpu (src/compute_delta_mu2_curve.jl:186-225) feeding
 * process_mu_chunk_dmumu_cpu! -- without the mu chunk leaving the device: mu
 * is reconstructed into a device scratch chunk (at most 1 GiB of particles,
 * with B read as interleaved node records) and binned there.
 * d_pos / d_mom: positions (m) and momenta (kg m/s), component c of save s of
 * particle p at base + s*row_stride + c*comp_stride + p (the Julia
 * (chunk, 3, nsave) datasets: row_stride = 3*chunk, comp_stride = chunk; the
 * device phase-space cache [nsave][6][n]: d_mom = d_pos + 3n, row_stride = 6n,
 * comp_stride = n).  f64 selects the compute precision T of the reference
 * (0: Float32, the default; 1: Float64); positions, momenta and d_bfield
 * ({Bx, By, Bz} column-major, nx*ny*nz each) are in T.  mu is bit-identical
 * to pt_reconstruct_mu at the same precision; the accumulators are those of
 * pt_dmumu_accumulate_device (device pointers, add-into).  No reference
 * counterpart as a single function.
 */
int pt_dmumu_accumulate_phase_space_device(pt_ctx* ctx, const void* d_pos, const void* d_mom, int64_t n,
                                           int64_t nsave, int64_t row_stride, int64_t comp_stride,
                                           const void* const d_bfield[3], const pt_grid* grid, int f64,
                                           const int64_t* d_lag_steps, int n_lags, const double* d_mu_edges,
                                           int n_bins, int start_mode, int bin_abs, int64_t* d_counts,
                                           double* d_sum_d, double* d_sum_d2, int64_t* d_w_count, double* d_w_mean,
                                           double* d_w_m2, double* d_pair_ss, int64_t* d_pair_n);

/*
 * Same as pt_dmumu_accumulate_device, but allocates no device memory: no
 * cudaMalloc / cudaFree and no allocating library call.  It has no
 * counterpart in the reference.  It is for callers that cannot let a
 * library allocate: a host that owns every device byte through its own pool
 * (the Julia host's CUDA.jl pool, a server admitting jobs by HBM budget)
 * cannot account for an allocation made behind its back, and cudaFree
 * synchronises the whole device, stalling other streams.
 * The per-CTA partials live in one fixed 16 MiB device array that every GPU
 * loading the library keeps until the process exits.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress); make
 * the first call on each device before any stream capture.  All calls share
 * the array and fully overwrite the part they use, so nothing carries over
 * between calls, but calls that overlap on the GPU (two streams, two host
 * threads) race on it: serialise them.  Limits: the (lag batch x bin)
 * partials must fit in the 16 MiB array, and each particle's mu series must
 * fit on chip (about 20,000 saves at 50 bins and 64 lags); larger requests fail with
 * PT_ERR_ARG and a message naming the limit.
 */
int pt_dmumu_accumulate_device_noalloc(pt_ctx* ctx, const float* d_mu, int64_t n, int64_t nsave, int64_t sp,
                                       int64_t ss, const int64_t* d_lag_steps, int n_lags, const double* d_mu_edges,
                                       int n_bins, int start_mode, int bin_abs, int64_t* d_counts, double* d_sum_d,
                                       double* d_sum_d2, int64_t* d_w_count, double* d_w_mean, double* d_w_m2,
                                       double* d_pair_ss, int64_t* d_pair_n);

/*
 * D_pp lag statistics: replaces process_momenta_chunk_dpp_cpu!
 *   src/compute_dpp_full.jl:247-288.
 * mom: Float32 phase-space momenta, Julia (chunk, 3, nsave): element
 *   (p, c, s) at mom[(s*3 + c)*chunk + p].
 * counts/sdp/sdp2/sdn/sdn2: [n_lags], add-into.
 */
int pt_dpp_accumulate(pt_ctx* ctx, const float* mom, int64_t chunk, int64_t nsave, const int64_t* lag_steps,
                      int n_lags, double p0, int64_t* counts, double* sdp, double* sdp2, double* sdn, double* sdn2);
int pt_dpp_accumulate_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave,
                             const int64_t* d_lag_steps, int n_lags, double p0, int64_t* d_counts, double* d_sdp,
                             double* d_sdp2, double* d_sdn, double* d_sdn2);

/*
 * Kinetic-energy snapshots: replaces fill_energy_snapshots!
 *   src/compute_dpp_full.jl:290-299 (kinetic_energy_gev_from_pmag :236-240).
 * snap_steps[n_snap]: 0-based save indices.  out: Julia (n_snap, n_total)
 * Float64, written for columns particle_offset .. particle_offset+chunk-1.
 */
int pt_energy_snapshots(pt_ctx* ctx, const float* mom, int64_t chunk, int64_t nsave, const int64_t* snap_steps,
                        int n_snap, int64_t particle_offset, double* out);
/* Same on the device: d_mom and d_snap_steps are device arrays, d_out the
 * device (n_snap, n_total) array; enqueued on the context stream.  A snapshot
 * index outside [0, nsave) gives NaN (the device indices are not checked on
 * the host). */
int pt_energy_snapshots_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave,
                               const int64_t* d_snap_steps, int n_snap, int64_t particle_offset, double* d_out);
/* On-device histogram of the snapshot energies into n_hist log-spaced bins on
 * [e_min, e_max] GeV (counts[n_snap][n_hist], add-into; out-of-range and NaN
 * energies, and snapshot indices outside [0, nsave), are not counted).  No reference counterpart: the reference stores
 * the raw energies and bins them in Python (scripts/plot_energy_distribution.py:167-174). */
int pt_energy_histogram_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave,
                               const int64_t* d_snap_steps, int n_snap, double e_min, double e_max, int n_hist,
                               int64_t* d_counts);

/*
 * Phase-space mu reconstruction: replaces reconstruct_mu_chunk_gpu
 *   src/compute_delta_mu2_curve.jl:186-225 (kernel :151-184).
 * pos/mom: Julia (chunk, 3, nsave) in the compute precision (f32: float,
 * f64: double); bfield = {Bx, By, Bz} host column-major in the compute
 * precision; grid scalars already in that precision.
 * mu_out: Julia (nsave, chunk) = [p][s] (time fastest).
 */
int pt_reconstruct_mu(pt_ctx* ctx, const void* pos, const void* mom, int64_t chunk, int64_t nsave,
                      const void* const bfield[3], const pt_grid* grid, int f64, void* mu_out);

/*
 * Initial particle state written on the device: the formulas of
 * init_particles, rand_unit_vector and fixed_mu_unit_vector
 * (src/phase_space_gpu_runner.jl:61-66, 170-245) -- uniform positions
 * u (xmax - xmin) + xmin, isotropic directions (z = 2u - 1, phi = 2 pi u) or
 * pitch cosine mu0 about the local B with a random gyrophase, |p| = gamma0 m v0
 * (gamma0, v0 from the kinetic energy, src/phase_space_gpu_runner.jl:51-59).
 * The reference draws from a Julia MersenneTwister, which is not restated:
 * draw d of particle i here is the SplitMix64 output of counter 8 i + d + 1
 * under the key mix64(seed), as a double (h >> 11) 2^-53.  Draws 0-2: the
 * position (random mode); draw 3: z (isotropic) or phi (fixed mu); draw 4:
 * phi (isotropic).  For fixed mu, B at the position is the trilinear sample
 * of the field's own values (FP64 for PT_FIELD_REF_F64; the stored FP32/BF16
 * values for bricks, with the BF16 forms' mean field added back).  Positions are exact; momenta agree with a host
 * restatement to the last bits of cos/sin.  Synchronous: returns PT_ERR_ARG
 * ("cannot use fixed-mu injection where local B is zero or non-finite", as
 * the reference) after the kernel if any particle met such a field.
 * No reference counterpart as a C entry (the reference initialises on the
 * host); it lets a serving loop admit jobs without host work.
 */
enum { PT_INJECT_ISOTROPIC = 0, PT_INJECT_FIXED_MU = 1 };
enum { PT_POSITION_RANDOM = 0, PT_POSITION_FIXED = 1 };
typedef struct pt_init_params {
    int64_t n;
    uint64_t seed;
    double energy_GeV;   /* kinetic energy of every particle */
    int32_t injection;   /* PT_INJECT_* */
    int32_t position_mode; /* PT_POSITION_* */
    double mu0;          /* fixed mu, in [-1, 1] */
    double position[3];  /* PT_POSITION_FIXED: box fractions, in [0, 1] */
} pt_init_params;
int pt_particles_init_device(pt_ctx* ctx, const pt_field* field, const pt_init_params* params, double* d_x1,
                             double* d_x2, double* d_x3, double* d_p1, double* d_p2, double* d_p3);

#ifdef __cplusplus
}
#endif

#endif /* PTB200_H */
