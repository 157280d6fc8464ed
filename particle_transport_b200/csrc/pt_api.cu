// C ABI of libptb200: contexts, field libraries, push runners and the
// statistics entry points.  See include/ptb200.h for the contract of each
// function and the reference function it replaces.
#include "pt_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace pt {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    set_error(m);
    return (e == cudaErrorMemoryAllocation) ? PT_ERR_OOM : PT_ERR_CUDA;
}

int scratch_get(pt_ctx* ctx, int slot, size_t bytes, void** out)
{
    ScratchBuf& b = ctx->scratch[slot];
    if (b.bytes < bytes) {
        if (b.ptr) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(b.ptr);
        }
        b.ptr = nullptr;
        b.bytes = 0;
        // generous first size and 1.5x growth (at most 256 MiB of slack): a
        // regrowth frees the old buffer, and cudaFree waits for every stream
        // of the device
        size_t want = std::max(bytes + std::min(bytes / 2, (size_t)256 << 20), (size_t)16 << 20);
        cudaError_t e = cudaMalloc(&b.ptr, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PT_ERR_OOM, "scratch allocation of " + std::to_string(want) + " bytes failed");
        }
        b.bytes = want;
    }
    *out = b.ptr;
    return PT_OK;
}

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t bytes)
    {
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(PT_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
        return PT_OK;
    }
    template <typename T> T* as() const { return (T*)p; }
};

int check_grid(const pt_grid* g)
{
    if (!g) return fail(PT_ERR_ARG, "grid is null");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return fail(PT_ERR_ARG, "grid needs at least 2 nodes per axis");
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0)) return fail(PT_ERR_ARG, "grid spacing must be positive");
    if (!(g->xmax > g->xmin && g->ymax > g->ymin && g->zmax > g->zmin))
        return fail(PT_ERR_ARG, "grid extent must be positive");
    return PT_OK;
}

uint32_t spread3(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 10; ++b) r |= ((v >> b) & 1u) << (3 * b);
    return r;
}

// Node offsets of the Morton-bricked layout: node(i, j, k) = offx[i] + offy[j] + offz[k].
// Inside an 8^3 brick nodes are in Morton order (a 2x2x2 cell corner set is
// 8 consecutive nodes when the cell is even-aligned); bricks are in Morton
// order when the brick grid is a power-of-two cube, else x-fastest.
void brick_offsets(const pt_grid& g, std::vector<uint32_t>& offs, int64_t& n_nodes)
{
    const int64_t nbx = (g.nx + 7) / 8, nby = (g.ny + 7) / 8, nbz = (g.nz + 7) / 8;
    const bool cube_pow2 = nbx == nby && nby == nbz && (nbx & (nbx - 1)) == 0 && nbx <= 128;
    offs.resize(g.nx + g.ny + g.nz);
    for (int64_t i = 0; i < g.nx; ++i)
        offs[i] = cube_pow2 ? spread3((uint32_t)i) : (uint32_t)((i >> 3) * 512 + spread3((uint32_t)(i & 7)));
    for (int64_t j = 0; j < g.ny; ++j)
        offs[g.nx + j] = cube_pow2 ? (spread3((uint32_t)j) << 1)
                                   : (uint32_t)((j >> 3) * 512 * nbx + (spread3((uint32_t)(j & 7)) << 1));
    for (int64_t k = 0; k < g.nz; ++k)
        offs[g.nx + g.ny + k] = cube_pow2 ? (spread3((uint32_t)k) << 2)
                                          : (uint32_t)((k >> 3) * 512 * nbx * nby + (spread3((uint32_t)(k & 7)) << 2));
    n_nodes = cube_pow2 ? (8 * nbx) * (8 * nbx) * (8 * nbx) : 512 * nbx * nby * nbz;
}

int field_create(pt_ctx* ctx, const double* const comps[6], bool on_device, const pt_grid* grid, int storage,
                 double B_ref, pt_field** out)
{
    if (!ctx || !out || !comps) return fail(PT_ERR_ARG, "null argument");
    int rc = check_grid(grid);
    if (rc) return rc;
    for (int c = 0; c < 6; ++c)
        if (!comps[c]) return fail(PT_ERR_ARG, "field component is null");
    if (storage < PT_FIELD_REF_F64 || storage > PT_FIELD_BRICK_F64) return fail(PT_ERR_ARG, "unknown field storage");
    if (fast_storage(storage) && !(B_ref > 0 && std::isfinite(B_ref)))
        return fail(PT_ERR_ARG, "B_ref_T must be finite and positive for the FP32-push brick storages");
    if (grid->nx > 4096 || grid->ny > 4096 || grid->nz > 4096) return fail(PT_ERR_ARG, "grid axis above 4096 nodes");
    PT_DEVICE_SCOPE(ctx->device);
    pt_field* f = new (std::nothrow) pt_field();
    if (!f) return fail(PT_ERR_OOM, "host allocation failed");
    f->ctx = ctx;
    f->storage = storage;
    f->grid = *grid;
    f->B_ref = B_ref;
    const int64_t nn = grid->nx * grid->ny * grid->nz;
    const size_t cb = sizeof(double) * (size_t)nn;
    cudaStream_t s = ctx->stream;
    auto cleanup = [&](int code) {
        pt_field_destroy(f);
        return code;
    };
    // FP64 copies (kept for REF_F64, temporary for bricks when uploading from host)
    double* tmp[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const bool keep64 = storage == PT_FIELD_REF_F64;
    if (keep64 || !on_device) {
        for (int c = 0; c < 6; ++c) {
            cudaError_t e = cudaMalloc(&tmp[c], cb);
            if (e != cudaSuccess) {
                cudaGetLastError();
                for (int q = 0; q < c; ++q) cudaFree(tmp[q]);
                return cleanup(fail(PT_ERR_OOM, "field allocation failed"));
            }
            e = cudaMemcpyAsync(tmp[c], comps[c], cb, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) {
                for (int q = 0; q <= c; ++q) cudaFree(tmp[q]);
                return cleanup(cuda_fail(e, "field upload"));
            }
        }
    }
    if (keep64) {
        for (int c = 0; c < 6; ++c) f->comp[c] = tmp[c];
        f->bytes = 6 * (int64_t)cb;
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "field upload"));
        *out = f;
        return PT_OK;
    }
    std::vector<uint32_t> offs;
    brick_offsets(*grid, offs, f->n_nodes);
    const size_t node_bytes = record_bytes(storage);
    cudaError_t e = cudaMalloc(&f->nodes, node_bytes * (size_t)f->n_nodes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&f->offs, sizeof(uint32_t) * offs.size());
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (int c = 0; c < 6; ++c) if (tmp[c]) cudaFree(tmp[c]);
        return cleanup(fail(PT_ERR_OOM, "brick field allocation failed"));
    }
    f->bytes = (int64_t)(node_bytes * f->n_nodes + sizeof(uint32_t) * offs.size());
    e = cudaMemcpyAsync(f->offs, offs.data(), sizeof(uint32_t) * offs.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(f->nodes, 0, node_bytes * (size_t)f->n_nodes, s);
    if (e != cudaSuccess) {
        for (int c = 0; c < 6; ++c) if (tmp[c]) cudaFree(tmp[c]);
        return cleanup(cuda_fail(e, "brick field init"));
    }
    const double* src[6];
    for (int c = 0; c < 6; ++c) src[c] = on_device ? comps[c] : tmp[c];
    if (field_layout(storage) == LAYOUT_BF16 || field_layout(storage) == LAYOUT_BF16_XPAIR) {
        // BF16 keeps 8 significant bits: B stored as B - <B> (|B - <B>| ~ dB
        // instead of ~ B0) rounds with the spacing of the fluctuation, which
        // for a mean field above the fluctuation is several times finer
        double mean[3];
        rc = field_means(ctx, src, nn, mean, s);
        if (rc) {
            for (int c = 0; c < 6; ++c) if (tmp[c]) cudaFree(tmp[c]);
            return cleanup(rc);
        }
        for (int c = 0; c < 3; ++c) f->boff[c] = (float)(mean[c] / B_ref);
    }
    rc = launch_brick_convert(src, *grid, B_ref, field_layout(storage), f->nodes, f->offs, f->n_nodes, f->boff, s);
    e = cudaStreamSynchronize(s);
    for (int c = 0; c < 6; ++c) if (tmp[c]) cudaFree(tmp[c]);
    if (rc) return cleanup(rc);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "brick conversion"));
    // the node records as a linear texture of 16-byte texels, so that a push
    // can fetch part of its corners through the texture path; a field larger
    // than the device's linear-texture limit simply has none
    const size_t texels = node_bytes * (size_t)f->n_nodes / 16;
    int max_texels = 0;
    cudaDeviceGetAttribute(&max_texels, cudaDevAttrMaxTexture1DLinearWidth, ctx->device);
    if (texels <= (size_t)max_texels && texels <= (size_t)INT32_MAX) {
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeLinear;
        rd.res.linear.devPtr = f->nodes;
        rd.res.linear.desc = cudaCreateChannelDesc<uint4>();
        rd.res.linear.sizeInBytes = texels * 16;
        cudaTextureDesc td{};
        td.readMode = cudaReadModeElementType;
        if (cudaCreateTextureObject(&f->tex, &rd, &td, nullptr) != cudaSuccess) {
            cudaGetLastError();
            f->tex = 0;
        }
    }
    *out = f;
    return PT_OK;
}

int check_params(const pt_push_params* p, const pt_field* f)
{
    if (!p) return fail(PT_ERR_ARG, "params is null");
    if (!(p->dt > 0 && std::isfinite(p->dt))) return fail(PT_ERR_ARG, "dt must be finite and positive");
    if (p->nsteps < 1) return fail(PT_ERR_ARG, "nsteps must be >= 1");
    if (p->stride < 1) return fail(PT_ERR_ARG, "stride must be >= 1");
    if (p->cache_mode < PT_CACHE_NONE || p->cache_mode > PT_CACHE_PHASE_SPACE) return fail(PT_ERR_ARG, "cache_mode");
    if (p->precision == PT_PUSH_F64 && f->storage != PT_FIELD_REF_F64 && f->storage != PT_FIELD_BRICK_F64)
        return fail(PT_ERR_ARG, "the FP64 push needs a REF_F64 or BRICK_F64 field");
    if (p->precision == PT_PUSH_F32 && !fast_storage(f->storage))
        return fail(PT_ERR_ARG, "the FP32 push needs a brick field (BRICK_F32 or BRICK_BF16)");
    if (p->precision != PT_PUSH_F64 && p->precision != PT_PUSH_F32) return fail(PT_ERR_ARG, "precision");
    if (p->cache_pitch < 0) return fail(PT_ERR_ARG, "cache_pitch must be >= 0");
    if (p->cache_pitch > 0 && (p->precision != PT_PUSH_F32 || p->cache_mode != PT_CACHE_MU))
        return fail(PT_ERR_ARG, "cache_pitch (time-fastest layout) applies to the mu cache of the FP32 push only");
    return PT_OK;
}

PushArgsFast fast_args(const pt_field* f, pt_fast_state* st, const pt_push_params* p)
{
    const pt_grid& g = f->grid;
    PushArgsFast a{};
    a.fld.nodes = f->nodes;
    a.fld.offs = f->offs;
    a.fld.nx = g.nx; a.fld.ny = g.ny; a.fld.nz = g.nz;
    a.fld.bf16 = f->storage != PT_FIELD_BRICK_F32;
    a.fld.layout = field_layout(f->storage);
    a.fld.tex = f->tex;
    for (int c = 0; c < 3; ++c) a.fld.boff[c] = f->boff[c];
    a.wx = (g.xmax - g.xmin) / g.dx;
    a.wy = (g.ymax - g.ymin) / g.dy;
    a.wz = (g.zmax - g.zmin) / g.dz;
    a.x = st->x; a.p = st->p; a.p2 = st->p2; a.pid = st->pid; a.alive = st->alive; a.n = st->n;
    a.hB = (float)(Q_E * f->B_ref * p->dt / (2.0 * M_P));
    a.vfac[0] = (float)(C_LIGHT * p->dt / g.dx);
    a.vfac[1] = (float)(C_LIGHT * p->dt / g.dy);
    a.vfac[2] = (float)(C_LIGHT * p->dt / g.dz);
    a.xmin[0] = g.xmin; a.xmin[1] = g.ymin; a.xmin[2] = g.zmin;
    a.dxs[0] = g.dx; a.dxs[1] = g.dy; a.dxs[2] = g.dz;
    a.nsteps = p->nsteps; a.stride = p->stride;
    a.periodic = p->periodic; a.cache_mode = p->cache_mode; a.cache_f64 = p->cache_f64;
    a.variant = p->kernel_variant;
    a.ring = 0;
    a.n_cache = st->n;
    a.pitch = p->cache_pitch;
    return a;
}

}  // namespace

// The FP64 push over a BRICK_F64 field.  Without a sort cadence it runs on
// the caller's arrays (slot = particle).  With one (sort_every > 0) the state
// is copied into slots of a context-owned buffer pair, re-sorted by brick at
// the start and every sort_every steps, pushed there (cache columns by
// particle id), and scattered back to the caller's order at the end.
static int advance_exact_brick(pt_ctx* ctx, const pt_field* f, double* d_x1, double* d_x2, double* d_x3, double* d_p1,
                               double* d_p2, double* d_p3, uint8_t* d_alive, int64_t n, const pt_push_params* p,
                               int64_t step_begin, int64_t step_count, void* d_cache, int64_t row_base, int64_t rows,
                               int64_t* d_deaths)
{
    if (n <= 0 || step_count <= 0) return PT_OK;
    PushArgsExactBrick a{};
    a.nodes = f->nodes;
    a.tail = (const char*)f->nodes + 32 * (size_t)f->n_nodes;
    a.offs = f->offs;
    a.g = f->grid;
    a.n = n; a.dt = p->dt; a.nsteps = p->nsteps; a.stride = p->stride;
    a.periodic = p->periodic; a.cache_mode = p->cache_mode; a.cache_f64 = p->cache_f64;
    a.cache = d_cache; a.row_base = row_base; a.rows = rows; a.deaths = d_deaths;
    const int64_t K = p->steps_per_launch > 0 ? p->steps_per_launch : 64;
    const int64_t end = step_begin + step_count;
    cudaStream_t s = ctx->stream;
    double* user[6] = {d_x1, d_x2, d_x3, d_p1, d_p2, d_p3};
    if (p->sort_every <= 0) {
        for (int k = 0; k < 3; ++k) {
            a.x[k] = user[k];
            a.p[k] = user[3 + k];
        }
        a.alive = d_alive;
        a.pid = nullptr;
        for (int64_t s0 = step_begin; s0 < end; s0 += K) {
            a.step_begin = s0;
            a.step_count = std::min(K, end - s0);
            int rc = launch_push_exact_brick(a, s);
            if (rc) return rc;
        }
        return PT_OK;
    }
    if (n > INT32_MAX) return fail(PT_ERR_ARG, "particle count above 2^31 for the sorted FP64 push");
    // slot buffers: 2 x ([6][n] doubles, pid[n], alive[n]), then the sort's buckets
    const int64_t m = (f->n_nodes + 511) / 512 + 1;
    auto a256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t xs_b = a256(sizeof(double) * 6 * (size_t)n), pid_b = a256(sizeof(int32_t) * (size_t)n),
                 al_b = a256((size_t)n), set_b = xs_b + pid_b + al_b;
    const size_t hist_b = a256(sizeof(uint32_t) * (size_t)m),
                 cur_b = a256(sizeof(uint32_t) * (size_t)(m + sort_scan_tiles(m)));
    void* base = nullptr;
    int rc = scratch_get(ctx, 5, 2 * set_b + hist_b + cur_b, &base);
    if (rc) return rc;
    char* b0 = (char*)base;
    double* xs[2] = {(double*)b0, (double*)(b0 + set_b)};
    int32_t* pid[2] = {(int32_t*)(b0 + xs_b), (int32_t*)(b0 + set_b + xs_b)};
    uint8_t* al[2] = {(uint8_t*)(b0 + xs_b + pid_b), (uint8_t*)(b0 + set_b + xs_b + pid_b)};
    uint32_t* hist = (uint32_t*)(b0 + 2 * set_b);
    uint32_t* cursor = (uint32_t*)(b0 + 2 * set_b + hist_b);
    if ((rc = launch_exact_import(user, d_alive, n, xs[0], pid[0], al[0], ctx->num_sms, s))) return rc;
    int cur = 0;
    int64_t last_sort = INT64_MIN;
    for (int64_t s0 = step_begin; s0 < end;) {
        if (last_sort == INT64_MIN || s0 - last_sort >= p->sort_every) {
            rc = launch_exact_sort(xs[cur], pid[cur], al[cur], n, f, xs[1 - cur], pid[1 - cur], al[1 - cur], hist,
                                   cursor, ctx->num_sms, s);
            if (rc) return rc;
            cur = 1 - cur;
            last_sort = s0;
        }
        const int64_t c = std::min(std::min(K, end - s0), last_sort + p->sort_every - s0);
        for (int k = 0; k < 3; ++k) {
            a.x[k] = xs[cur] + (size_t)k * n;
            a.p[k] = xs[cur] + (size_t)(3 + k) * n;
        }
        a.alive = al[cur];
        a.pid = pid[cur];
        a.step_begin = s0;
        a.step_count = c;
        if ((rc = launch_push_exact_brick(a, s))) return rc;
        s0 += c;
    }
    return launch_exact_export(xs[cur], pid[cur], al[cur], n, user, d_alive, ctx->num_sms, s);
}

// Advance the fast state over [s0, s0 + count), splitting launches at the
// re-sort cadence (sort_every steps) and at steps_per_launch.
static int advance_fast(pt_ctx* ctx, const pt_field* f, pt_fast_state* st, const pt_push_params* p, int64_t s0,
                        int64_t count, void* cache, int64_t row_base, int64_t rows, int64_t* deaths)
{
    PushArgsFast a = fast_args(f, st, p);
    a.cache = cache; a.row_base = row_base; a.rows = rows; a.deaths = deaths;
    const int64_t K = p->steps_per_launch > 0 ? p->steps_per_launch : count;
    int64_t s = s0;
    const int64_t end = s0 + count;
    while (s < end) {
        if (p->sort_every > 0 && (st->last_sort == INT64_MIN || s - st->last_sort >= p->sort_every)) {
            int rc = fast_sort(ctx, st, f, ctx->stream);
            if (rc) return rc;
            st->last_sort = s;
        }
        int64_t c = std::min(K, end - s);
        if (p->sort_every > 0) c = std::min(c, st->last_sort + p->sort_every - s);
        // the sort swaps the state buffers: take the current ones
        a.x = st->x; a.p = st->p; a.p2 = st->p2; a.pid = st->pid; a.alive = st->alive;
        a.step_begin = s;
        a.step_count = c;
        int rc = launch_push_fast(a, ctx->stream);
        if (rc) return rc;
        s += c;
    }
    return PT_OK;
}

}  // namespace pt

using namespace pt;

extern "C" {

const char* pt_last_error(void) { return g_last_error.c_str(); }

int pt_version(void) { return PTB200_VERSION; }

int pt_ctx_create(int device, pt_ctx** out)
{
    if (!out) return fail(PT_ERR_ARG, "out is null");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) return fail(PT_ERR_ARG, "device index out of range");
    PT_DEVICE_SCOPE(device);
    cudaDeviceProp prop;
    PT_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(PT_ERR_ARG, "libptb200 is built for sm_100a (B200); device is sm_" +
                                                     std::to_string(prop.major) + std::to_string(prop.minor));
    pt_ctx* c = new (std::nothrow) pt_ctx();
    if (!c) return fail(PT_ERR_OOM, "host allocation failed");
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate");
    }
    c->stream = c->own_stream;
    *out = c;
    return PT_OK;
}

int pt_ctx_destroy(pt_ctx* ctx)
{
    if (!ctx) return PT_OK;
    ::pt::DeviceScope device_scope(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    pt_ctx_trim(ctx);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return PT_OK;
}

int pt_ctx_trim(pt_ctx* ctx)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    PT_DEVICE_SCOPE(ctx->device);
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->copy_stream) PT_CUDA(cudaStreamSynchronize(ctx->copy_stream));
    for (auto& b : ctx->scratch) {
        if (b.ptr) cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    if (ctx->pinned.ptr) cudaFreeHost(ctx->pinned.ptr);
    ctx->pinned.ptr = nullptr;
    ctx->pinned.bytes = 0;
    if (ctx->run_fs) pt_fast_state_destroy(ctx->run_fs);
    ctx->run_fs = nullptr;
    return PT_OK;
}

int pt_ctx_set_stream(pt_ctx* ctx, void* stream)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return PT_OK;
}

int pt_ctx_synchronize(pt_ctx* ctx)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    return PT_OK;
}

int pt_field_upload(pt_ctx* ctx, const double* const comps[6], const pt_grid* grid, int storage, double B_ref_T,
                    pt_field** out)
{
    return field_create(ctx, comps, false, grid, storage, B_ref_T, out);
}

int pt_field_upload_device(pt_ctx* ctx, const double* const d_comps[6], const pt_grid* grid, int storage,
                           double B_ref_T, pt_field** out)
{
    return field_create(ctx, d_comps, true, grid, storage, B_ref_T, out);
}

int pt_field_destroy(pt_field* f)
{
    if (!f) return PT_OK;
    for (int c = 0; c < 6; ++c)
        if (f->comp[c]) cudaFree(f->comp[c]);
    if (f->tex) cudaDestroyTextureObject(f->tex);
    if (f->nodes) cudaFree(f->nodes);
    if (f->offs) cudaFree(f->offs);
    delete f;
    return PT_OK;
}

int64_t pt_field_device_bytes(const pt_field* f) { return f ? f->bytes : 0; }

int pt_push_advance_device(pt_ctx* ctx, const pt_field* f, double* d_x1, double* d_x2, double* d_x3, double* d_p1,
                           double* d_p2, double* d_p3, uint8_t* d_alive, int64_t n, const pt_push_params* p,
                           int64_t step_begin, int64_t step_count, void* d_cache, int64_t row_base, int64_t rows,
                           int64_t* d_deaths)
{
    if (!ctx || !f) return fail(PT_ERR_ARG, "null context or field");
    PT_DEVICE_SCOPE(ctx->device);
    int rc = check_params(p, f);
    if (rc) return rc;
    if (p->precision != PT_PUSH_F64) return fail(PT_ERR_ARG, "use pt_push_advance_fast for the FP32 push");
    if (n < 0 || step_begin < 0 || step_count < 0 || step_begin + step_count > p->nsteps)
        return fail(PT_ERR_ARG, "step range outside [0, nsteps)");
    if (n > 0 && !(d_x1 && d_x2 && d_x3 && d_p1 && d_p2 && d_p3 && d_alive)) return fail(PT_ERR_ARG, "null state");
    if (p->cache_mode != PT_CACHE_NONE && rows > 0 && !d_cache) return fail(PT_ERR_ARG, "null cache");
    if (f->storage == PT_FIELD_BRICK_F64)
        return advance_exact_brick(ctx, f, d_x1, d_x2, d_x3, d_p1, d_p2, d_p3, d_alive, n, p, step_begin, step_count,
                                   d_cache, row_base, rows, d_deaths);
    PushArgsRef a{};
    for (int c = 0; c < 6; ++c) a.f[c] = f->comp[c];
    a.g = f->grid;
    a.x[0] = d_x1; a.x[1] = d_x2; a.x[2] = d_x3;
    a.p[0] = d_p1; a.p[1] = d_p2; a.p[2] = d_p3;
    a.alive = d_alive; a.n = n; a.dt = p->dt; a.nsteps = p->nsteps; a.stride = p->stride;
    a.periodic = p->periodic; a.cache_mode = p->cache_mode; a.cache_f64 = p->cache_f64;
    a.cache = d_cache; a.row_base = row_base; a.rows = rows; a.deaths = d_deaths;
    const int64_t K = p->steps_per_launch > 0 ? p->steps_per_launch : 64;
    for (int64_t s = step_begin; s < step_begin + step_count; s += K) {
        a.step_begin = s;
        a.step_count = std::min(K, step_begin + step_count - s);
        rc = launch_push_ref(a, ctx->stream);
        if (rc) return rc;
    }
    return PT_OK;
}

int pt_fast_state_create(pt_ctx* ctx, const pt_field* f, const double* d_x1, const double* d_x2, const double* d_x3,
                         const double* d_p1, const double* d_p2, const double* d_p3, const uint8_t* d_alive,
                         int64_t n, pt_fast_state** out)
{
    if (!ctx || !f || !out) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (!fast_storage(f->storage)) return fail(PT_ERR_ARG, "fast state needs an FP32-push brick field");
    if (n < 0 || n > INT32_MAX) return fail(PT_ERR_ARG, "particle count out of range");
    pt_fast_state* st = new (std::nothrow) pt_fast_state();
    if (!st) return fail(PT_ERR_OOM, "host allocation failed");
    st->ctx = ctx;
    st->n = n;
    size_t m = (size_t)std::max<int64_t>(n, 1);
    cudaError_t e = cudaMalloc((void**)&st->x, sizeof(double) * 3 * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->p, sizeof(float) * 3 * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->p2, sizeof(double) * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->pid, sizeof(int32_t) * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->alive, m);
    if (e != cudaSuccess) {
        cudaGetLastError();
        pt_fast_state_destroy(st);
        return fail(PT_ERR_OOM, "fast state allocation failed");
    }
    if (n > 0) {
        int rc = launch_fast_import(st, f, d_x1, d_x2, d_x3, d_p1, d_p2, d_p3, d_alive, ctx->stream);
        if (rc) {
            pt_fast_state_destroy(st);
            return rc;
        }
    }
    st->field = f;
    st->last_sort = INT64_MIN;
    *out = st;
    return PT_OK;
}

int pt_fast_state_export(pt_ctx* ctx, const pt_fast_state* st, double* d_x1, double* d_x2, double* d_x3,
                         double* d_p1, double* d_p2, double* d_p3, uint8_t* d_alive)
{
    if (!ctx || !st) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (st->n == 0) return PT_OK;
    if (!(d_x1 && d_x2 && d_x3 && d_p1 && d_p2 && d_p3 && d_alive)) return fail(PT_ERR_ARG, "null state");
    return launch_fast_export(st, st->field, d_x1, d_x2, d_x3, d_p1, d_p2, d_p3, d_alive, ctx->stream);
}

int pt_fast_state_destroy(pt_fast_state* st)
{
    if (!st) return PT_OK;
    if (st->x) cudaFree(st->x);
    if (st->p) cudaFree(st->p);
    if (st->p2) cudaFree(st->p2);
    if (st->pid) cudaFree(st->pid);
    if (st->alive) cudaFree(st->alive);
    if (st->x_alt) cudaFree(st->x_alt);
    if (st->p_alt) cudaFree(st->p_alt);
    if (st->p2_alt) cudaFree(st->p2_alt);
    if (st->pid_alt) cudaFree(st->pid_alt);
    if (st->alive_alt) cudaFree(st->alive_alt);
    if (st->sort_tmp) cudaFree(st->sort_tmp);
    delete st;
    return PT_OK;
}

int pt_fast_state_sort(pt_ctx* ctx, pt_fast_state* st)
{
    if (!ctx || !st) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    return fast_sort(ctx, st, st->field, ctx->stream);
}

int pt_push_advance_fast(pt_ctx* ctx, const pt_field* f, pt_fast_state* st, const pt_push_params* p,
                         int64_t step_begin, int64_t step_count, void* d_cache, int64_t row_base, int64_t rows,
                         int64_t* d_deaths)
{
    if (!ctx || !f || !st) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    int rc = check_params(p, f);
    if (rc) return rc;
    if (p->precision != PT_PUSH_F32) return fail(PT_ERR_ARG, "pt_push_advance_fast runs the FP32 push");
    if (step_begin < 0 || step_count < 0 || step_begin + step_count > p->nsteps)
        return fail(PT_ERR_ARG, "step range outside [0, nsteps)");
    if (p->cache_mode != PT_CACHE_NONE && rows > 0 && !d_cache) return fail(PT_ERR_ARG, "null cache");
    if (p->cache_pitch > 0 && p->cache_pitch < rows)
        return fail(PT_ERR_ARG, "cache_pitch must be at least cache_rows (the saves of one particle)");
    if (f != st->field) return fail(PT_ERR_ARG, "fast state was created against a different field");
    return advance_fast(ctx, f, st, p, step_begin, step_count, d_cache, row_base, rows, d_deaths);
}

int pt_push_run(pt_ctx* ctx, const pt_field* f, double* x1, double* x2, double* x3, double* p1, double* p2,
                double* p3, uint8_t* alive, int64_t n, const pt_push_params* p, pt_save_fn save, void* user,
                int64_t* alive_count)
{
    if (!ctx || !f) return fail(PT_ERR_ARG, "null context or field");
    int rc = check_params(p, f);
    if (rc) return rc;
    if (n < 0) return fail(PT_ERR_ARG, "n must be >= 0");
    if (n > 0 && !(x1 && x2 && x3 && p1 && p2 && p3 && alive)) return fail(PT_ERR_ARG, "null state");
    if (p->cache_mode != PT_CACHE_NONE && !save) return fail(PT_ERR_ARG, "a cache mode needs a save callback");
    if (p->cache_pitch != 0) return fail(PT_ERR_ARG, "pt_push_run hands the save callback rows: cache_pitch must be 0");
    PT_DEVICE_SCOPE(ctx->device);
    cudaStream_t st = ctx->stream;
    const int64_t nsteps = p->nsteps, stride = p->stride;
    const size_t elem = p->cache_f64 ? 8 : 4;
    const int64_t row_elems = p->cache_mode == PT_CACHE_MU ? n : 6 * n;
    const size_t row_bytes = p->cache_mode == PT_CACHE_NONE ? 0 : elem * (size_t)row_elems;
    // The FP32 push writes its mu saves time-fastest, [n][8] (a particle's
    // saves of a chunk side by side, merged by L2 into whole sectors), and a
    // transpose turns each chunk into the rows the callback receives.
    const bool tf = p->precision == PT_PUSH_F32 && p->cache_mode == PT_CACHE_MU && !p->cache_f64 && n > 0;
    const int tf_pitch = 8;
    // rows per egress chunk: enough steps per launch, bounded staging memory
    int64_t R = tf ? tf_pitch : std::max<int64_t>(1, (256 + stride - 1) / stride);
    const size_t slot_cap = tf ? (512u << 20) : (256u << 20);
    if (row_bytes > 0) R = std::max<int64_t>(1, std::min<int64_t>(R, (int64_t)(slot_cap / row_bytes)));
    const int64_t chunk_steps = R * stride;

    // device: state [6][m] doubles + alive [m] + deaths [nsteps] + two egress slots
    // host: two pinned egress slots + the staging chunks of the state copies
    // (both grow-only in the context, kept between calls)
    const size_t m = (size_t)std::max<int64_t>(n, 1);
    const size_t state_bytes = align_up(sizeof(double) * 6 * m + m, 256);
    const size_t deaths_bytes = align_up(sizeof(int64_t) * (size_t)nsteps, 256);
    const size_t slots_bytes = row_bytes ? 2 * (size_t)R * row_bytes : 0;
    const size_t tf_bytes = tf ? align_up(sizeof(float) * tf_pitch * m, 256) + 256 : 0;
    const size_t stage_chunk = 32u << 20;
    const int stage_nbuf = 3;
    void* dbase = nullptr;
    void* hbase = nullptr;
    if ((rc = scratch_get(ctx, 2, state_bytes + deaths_bytes + slots_bytes + tf_bytes, &dbase))) return rc;
    if ((rc = pinned_get(ctx, slots_bytes + stage_chunk * stage_nbuf, &hbase))) return rc;
    char* stage = (char*)hbase + slots_bytes;
    char* dslot_base = (char*)dbase + state_bytes + deaths_bytes;  // [2][R] device egress rows
    // [n][8] time-fastest saves of a chunk, 32-byte records on 256-byte-aligned storage
    float* dtf = tf ? (float*)(dslot_base + align_up(slots_bytes, 256)) : nullptr;
    char* hslot_base = (char*)hbase;                                // [2][R] pinned egress rows
    int64_t* d_deaths = (int64_t*)((char*)dbase + state_bytes);
    double* d[6];
    for (int k = 0; k < 6; ++k) d[k] = (double*)dbase + (size_t)k * m;
    uint8_t* dal = (uint8_t*)((double*)dbase + 6 * m);
    double* hs[6] = {x1, x2, x3, p1, p2, p3};
    std::vector<HostSeg> segs;
    if (n > 0) {
        for (int k = 0; k < 6; ++k) segs.push_back(HostSeg{(char*)hs[k], (char*)d[k], sizeof(double) * (size_t)n});
        segs.push_back(HostSeg{(char*)alive, (char*)dal, (size_t)n});
    }
    const int64_t alive0 = count_nonzero(alive, n);
    if ((rc = staged_h2d(segs, stage, stage_chunk, stage_nbuf, st))) return rc;
    PT_CUDA(cudaMemsetAsync(d_deaths, 0, sizeof(int64_t) * (size_t)nsteps, st));
    pt_fast_state* fs = nullptr;
    if (p->precision == PT_PUSH_F32) {
        fs = ctx->run_fs;
        if (fs && fs->n == n) {
            // reuse the context's state buffers: import this call's particles
            if (n > 0 && (rc = launch_fast_import(fs, f, d[0], d[1], d[2], d[3], d[4], d[5], dal, st))) return rc;
            fs->field = f;
            fs->last_sort = INT64_MIN;
        } else {
            if (fs) {
                cudaStreamSynchronize(st);
                pt_fast_state_destroy(fs);
                ctx->run_fs = nullptr;
            }
            rc = pt_fast_state_create(ctx, f, d[0], d[1], d[2], d[3], d[4], d[5], dal, n, &fs);
            if (rc) return rc;
            ctx->run_fs = fs;
        }
    }
    cudaEvent_t ev_done[2] = {nullptr, nullptr}, ev_copy[2] = {nullptr, nullptr};
    for (int k = 0; k < 2; ++k) {
        cudaEventCreateWithFlags(&ev_done[k], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev_copy[k], cudaEventDisableTiming);
    }
    auto finish = [&](int code) {
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(ctx->copy_stream);
        for (int k = 0; k < 2; ++k) {
            cudaEventDestroy(ev_done[k]);
            cudaEventDestroy(ev_copy[k]);
        }
        return code;
    };
    struct Pending {
        int64_t row_base = 0, rows = 0;
        int slot = 0;
        bool valid = false;
    } pend;
    auto deliver = [&](const Pending& q) -> int {
        if (!q.valid || q.rows == 0) return PT_OK;
        cudaError_t e = cudaEventSynchronize(ev_copy[q.slot]);
        if (e != cudaSuccess) return cuda_fail(e, "cache egress copy");
        const char* base = hslot_base + (size_t)q.slot * R * row_bytes;
        for (int64_t r = 0; r < q.rows; ++r)
            if (save(user, q.row_base + r, base + (size_t)r * row_bytes, (int64_t)row_bytes) != 0)
                return fail(PT_ERR_CALLBACK, "save callback returned non-zero at save " + std::to_string(q.row_base + r));
        return PT_OK;
    };
    int64_t chunk = 0;
    for (int64_t s0 = 0; s0 < nsteps; s0 += chunk_steps, ++chunk) {
        const int64_t steps = std::min(chunk_steps, nsteps - s0);
        const int slot = (int)(chunk & 1);
        const int64_t row_base = s0 / stride;
        const int64_t rows = row_bytes ? ((s0 + steps - 1) / stride - row_base + 1) : 0;
        void* dslot = row_bytes ? dslot_base + (size_t)slot * R * row_bytes : nullptr;
        if (chunk >= 2 && row_bytes) PT_CUDA(cudaStreamWaitEvent(st, ev_copy[slot], 0));
        if (p->precision == PT_PUSH_F64) {
            pt_push_params q = *p;
            rc = pt_push_advance_device(ctx, f, d[0], d[1], d[2], d[3], d[4], d[5], dal, n, &q, s0, steps, dslot,
                                        row_base, rows, d_deaths);
        } else if (tf) {
            pt_push_params q = *p;
            q.cache_pitch = tf_pitch;
            rc = advance_fast(ctx, f, fs, &q, s0, steps, dtf, row_base, rows, d_deaths);
            if (!rc) rc = launch_tf_to_rows(dtf, n, tf_pitch, (int)rows, (float*)dslot, st);
        } else {
            rc = advance_fast(ctx, f, fs, p, s0, steps, dslot, row_base, rows, d_deaths);
        }
        if (rc) return finish(rc);
        if (row_bytes) {
            PT_CUDA(cudaEventRecord(ev_done[slot], st));
            PT_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ev_done[slot], 0));
            PT_CUDA(cudaMemcpyAsync(hslot_base + (size_t)slot * R * row_bytes, dslot, (size_t)rows * row_bytes,
                                    cudaMemcpyDeviceToHost, ctx->copy_stream));
            PT_CUDA(cudaEventRecord(ev_copy[slot], ctx->copy_stream));
        }
        rc = deliver(pend);
        if (rc) return finish(rc);
        pend = Pending{row_base, rows, slot, row_bytes > 0};
    }
    rc = deliver(pend);
    if (rc) return finish(rc);
    if (fs) {
        rc = launch_fast_export(fs, f, d[0], d[1], d[2], d[3], d[4], d[5], dal, st);
        if (rc) return finish(rc);
    }
    rc = staged_d2h(segs, stage, stage_chunk, stage_nbuf, st);
    if (rc) return finish(rc);
    std::vector<int64_t> deaths((size_t)nsteps);
    PT_CUDA(cudaMemcpyAsync(deaths.data(), d_deaths, sizeof(int64_t) * (size_t)nsteps, cudaMemcpyDeviceToHost, st));
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return finish(cuda_fail(e, "pt_push_run"));
    if (alive_count) {
        int64_t run = alive0;
        for (int64_t s = 0; s < nsteps; ++s) {
            run -= deaths[(size_t)s];
            alive_count[s] = run;
        }
    }
    return finish(PT_OK);
}

static int check_lags_host(const int64_t* lags, int n_lags)
{
    for (int i = 0; i < n_lags; ++i)
        if (lags[i] < 1) return fail(PT_ERR_ARG, "lag steps must be >= 1");
    return PT_OK;
}

int pt_dmumu_accumulate_device(pt_ctx* ctx, const float* d_mu, int64_t n, int64_t nsave, int64_t sp, int64_t ss,
                               const int64_t* d_lags, int n_lags, const double* d_edges, int n_bins, int start_mode,
                               int bin_abs, int64_t* d_counts, double* d_sum_d, double* d_sum_d2, int64_t* d_w_count,
                               double* d_w_mean, double* d_w_m2, double* d_pair_ss, int64_t* d_pair_n)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (n < 0 || nsave < 1 || n_lags < 0 || n_bins < 1) return fail(PT_ERR_ARG, "bad sizes");
    if (start_mode != PT_START_SLIDING && start_mode != PT_START_INJECTION) return fail(PT_ERR_ARG, "start_mode");
    if (n == 0 || n_lags == 0) return PT_OK;
    if (!(d_mu && d_lags && d_edges && d_counts && d_sum_d && d_sum_d2 && d_w_count && d_w_mean && d_w_m2 &&
          d_pair_ss && d_pair_n))
        return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    DmumuArgs a{d_mu, n, nsave, sp, ss, d_lags, n_lags, d_edges, n_bins, start_mode == PT_START_INJECTION, bin_abs != 0,
                d_counts, d_sum_d, d_sum_d2, d_w_count, d_w_mean, d_w_m2, d_pair_ss, d_pair_n};
    return run_dmumu(ctx, a, ctx->stream);
}

int pt_dmumu_accumulate_phase_space_device(pt_ctx* ctx, const void* d_pos, const void* d_mom, int64_t n,
                                           int64_t nsave, int64_t row_stride, int64_t comp_stride,
                                           const void* const d_bfield[3], const pt_grid* grid, int f64,
                                           const int64_t* d_lags, int n_lags, const double* d_edges, int n_bins,
                                           int start_mode, int bin_abs, int64_t* d_counts, double* d_sum_d,
                                           double* d_sum_d2, int64_t* d_w_count, double* d_w_mean, double* d_w_m2,
                                           double* d_pair_ss, int64_t* d_pair_n)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    int rc = check_grid(grid);
    if (rc) return rc;
    if (n < 0 || nsave < 1 || n_lags < 0 || n_bins < 1 || row_stride < 0 || comp_stride < 0)
        return fail(PT_ERR_ARG, "bad sizes");
    if (start_mode != PT_START_SLIDING && start_mode != PT_START_INJECTION) return fail(PT_ERR_ARG, "start_mode");
    if (n == 0 || n_lags == 0) return PT_OK;
    if (!(d_pos && d_mom && d_bfield && d_bfield[0] && d_bfield[1] && d_bfield[2] && d_lags && d_edges &&
          d_counts && d_sum_d && d_sum_d2 && d_w_count && d_w_mean && d_w_m2 && d_pair_ss && d_pair_n))
        return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    DmumuArgs a{nullptr, n, nsave, 0, 0, d_lags, n_lags, d_edges, n_bins, start_mode == PT_START_INJECTION,
                bin_abs != 0, d_counts, d_sum_d, d_sum_d2, d_w_count, d_w_mean, d_w_m2, d_pair_ss, d_pair_n};
    return run_dmumu_phase_space(ctx, a, d_pos, d_mom, row_stride, comp_stride, d_bfield, *grid, f64 != 0,
                                 ctx->stream);
}

int pt_dmumu_accumulate(pt_ctx* ctx, const float* mu, int64_t n, int64_t nsave, int64_t sp, int64_t ss,
                        const int64_t* lags, int n_lags, const double* edges, int n_bins, int start_mode, int bin_abs,
                        int64_t* counts, double* sum_d, double* sum_d2, int64_t* w_count, double* w_mean,
                        double* w_m2, double* pair_ss, int64_t* pair_n)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (n < 0 || nsave < 1 || n_lags < 0 || n_bins < 1 || sp < 0 || ss < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (n == 0 || n_lags == 0) return PT_OK;
    if (!(mu && lags && edges && counts && sum_d && sum_d2 && w_count && w_mean && w_m2 && pair_ss && pair_n))
        return fail(PT_ERR_ARG, "null pointer");
    int rc = check_lags_host(lags, n_lags);
    if (rc) return rc;
    PT_DEVICE_SCOPE(ctx->device);
    const size_t extent = (size_t)((n - 1) * sp + (nsave - 1) * ss + 1);
    const size_t nlb = (size_t)n_lags * n_bins;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_mu = take(4 * extent), o_l = take(8 * (size_t)n_lags), o_e = take(8 * (size_t)(n_bins + 1)),
                 o_c = take(8 * nlb), o_sd = take(8 * nlb), o_sd2 = take(8 * nlb), o_wc = take(8 * (size_t)n_lags),
                 o_wm = take(8 * (size_t)n_lags), o_wm2 = take(8 * (size_t)n_lags), o_ss = take(8 * (size_t)n_lags),
                 o_pn = take(8 * (size_t)n_lags);
    DevBuf buf;
    if ((rc = buf.alloc(off))) return rc;
    char* b = (char*)buf.p;
    cudaStream_t s = ctx->stream;
    struct { size_t o; const void* h; size_t bytes; } up[] = {
        {o_mu, mu, 4 * extent}, {o_l, lags, 8 * (size_t)n_lags}, {o_e, edges, 8 * (size_t)(n_bins + 1)},
        {o_c, counts, 8 * nlb}, {o_sd, sum_d, 8 * nlb}, {o_sd2, sum_d2, 8 * nlb}, {o_wc, w_count, 8 * (size_t)n_lags},
        {o_wm, w_mean, 8 * (size_t)n_lags}, {o_wm2, w_m2, 8 * (size_t)n_lags}, {o_ss, pair_ss, 8 * (size_t)n_lags},
        {o_pn, pair_n, 8 * (size_t)n_lags}};
    for (auto& u : up) PT_CUDA(cudaMemcpyAsync(b + u.o, u.h, u.bytes, cudaMemcpyHostToDevice, s));
    rc = pt_dmumu_accumulate_device(ctx, (const float*)(b + o_mu), n, nsave, sp, ss, (const int64_t*)(b + o_l), n_lags,
                                    (const double*)(b + o_e), n_bins, start_mode, bin_abs, (int64_t*)(b + o_c),
                                    (double*)(b + o_sd), (double*)(b + o_sd2), (int64_t*)(b + o_wc),
                                    (double*)(b + o_wm), (double*)(b + o_wm2), (double*)(b + o_ss),
                                    (int64_t*)(b + o_pn));
    if (rc) {
        cudaStreamSynchronize(s);
        return rc;
    }
    void* outs[] = {counts, sum_d, sum_d2, w_count, w_mean, w_m2, pair_ss, pair_n};
    for (int k = 0; k < 8; ++k) {
        const auto& u = up[3 + k];
        PT_CUDA(cudaMemcpyAsync(outs[k], b + u.o, u.bytes, cudaMemcpyDeviceToHost, s));
    }
    PT_CUDA(cudaStreamSynchronize(s));
    return PT_OK;
}

int pt_dpp_accumulate_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave, const int64_t* d_lags,
                             int n_lags, double p0, int64_t* d_counts, double* d_sdp, double* d_sdp2, double* d_sdn,
                             double* d_sdn2)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (chunk < 0 || nsave < 1 || n_lags < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (!(std::isfinite(p0) && p0 > 0.0)) return fail(PT_ERR_ARG, "p0 must be finite and positive");
    if (chunk == 0 || n_lags == 0) return PT_OK;
    if (!(d_mom && d_lags && d_counts && d_sdp && d_sdp2 && d_sdn && d_sdn2)) return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    DppArgs a{d_mom, chunk, nsave, d_lags, n_lags, p0, d_counts, d_sdp, d_sdp2, d_sdn, d_sdn2};
    return run_dpp(ctx, a, ctx->stream);
}

int pt_dpp_accumulate(pt_ctx* ctx, const float* mom, int64_t chunk, int64_t nsave, const int64_t* lags, int n_lags,
                      double p0, int64_t* counts, double* sdp, double* sdp2, double* sdn, double* sdn2)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (chunk < 0 || nsave < 1 || n_lags < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (!(std::isfinite(p0) && p0 > 0.0)) return fail(PT_ERR_ARG, "p0 must be finite and positive");
    if (chunk == 0 || n_lags == 0) return PT_OK;
    if (!(mom && lags && counts && sdp && sdp2 && sdn && sdn2)) return fail(PT_ERR_ARG, "null pointer");
    int rc = check_lags_host(lags, n_lags);
    if (rc) return rc;
    PT_DEVICE_SCOPE(ctx->device);
    const size_t nm = (size_t)chunk * 3 * nsave, L = (size_t)n_lags;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_m = take(4 * nm), o_l = take(8 * L), o_a[5] = {take(8 * L), take(8 * L), take(8 * L), take(8 * L),
                                                                  take(8 * L)};
    DevBuf buf;
    if ((rc = buf.alloc(off))) return rc;
    char* b = (char*)buf.p;
    cudaStream_t s = ctx->stream;
    void* acc[5] = {counts, sdp, sdp2, sdn, sdn2};
    PT_CUDA(cudaMemcpyAsync(b + o_m, mom, 4 * nm, cudaMemcpyHostToDevice, s));
    PT_CUDA(cudaMemcpyAsync(b + o_l, lags, 8 * L, cudaMemcpyHostToDevice, s));
    for (int k = 0; k < 5; ++k) PT_CUDA(cudaMemcpyAsync(b + o_a[k], acc[k], 8 * L, cudaMemcpyHostToDevice, s));
    rc = pt_dpp_accumulate_device(ctx, (const float*)(b + o_m), chunk, nsave, (const int64_t*)(b + o_l), n_lags, p0,
                                  (int64_t*)(b + o_a[0]), (double*)(b + o_a[1]), (double*)(b + o_a[2]),
                                  (double*)(b + o_a[3]), (double*)(b + o_a[4]));
    if (rc) {
        cudaStreamSynchronize(s);
        return rc;
    }
    for (int k = 0; k < 5; ++k) PT_CUDA(cudaMemcpyAsync(acc[k], b + o_a[k], 8 * L, cudaMemcpyDeviceToHost, s));
    PT_CUDA(cudaStreamSynchronize(s));
    return PT_OK;
}

int pt_energy_snapshots(pt_ctx* ctx, const float* mom, int64_t chunk, int64_t nsave, const int64_t* snaps, int n_snap,
                        int64_t particle_offset, double* out)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (chunk < 0 || nsave < 1 || n_snap < 0 || particle_offset < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (chunk == 0 || n_snap == 0) return PT_OK;
    if (!(mom && snaps && out)) return fail(PT_ERR_ARG, "null pointer");
    for (int j = 0; j < n_snap; ++j)
        if (snaps[j] < 0 || snaps[j] >= nsave) return fail(PT_ERR_ARG, "snapshot index outside [0, nsave)");
    PT_DEVICE_SCOPE(ctx->device);
    const size_t nm = (size_t)chunk * 3 * nsave;
    DevBuf dm, ds, dout;
    int rc;
    if ((rc = dm.alloc(4 * nm)) || (rc = ds.alloc(8 * (size_t)n_snap)) || (rc = dout.alloc(8 * (size_t)chunk * n_snap)))
        return rc;
    cudaStream_t s = ctx->stream;
    PT_CUDA(cudaMemcpyAsync(dm.p, mom, 4 * nm, cudaMemcpyHostToDevice, s));
    PT_CUDA(cudaMemcpyAsync(ds.p, snaps, 8 * (size_t)n_snap, cudaMemcpyHostToDevice, s));
    rc = launch_energy_snapshots(dm.as<float>(), chunk, nsave, ds.as<int64_t>(), n_snap, 0, dout.as<double>(), s);
    if (rc) return rc;
    PT_CUDA(cudaMemcpyAsync(out + particle_offset * n_snap, dout.p, 8 * (size_t)chunk * n_snap, cudaMemcpyDeviceToHost,
                            s));
    PT_CUDA(cudaStreamSynchronize(s));
    return PT_OK;
}

int pt_energy_snapshots_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave,
                               const int64_t* d_snap_steps, int n_snap, int64_t particle_offset, double* d_out)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (chunk < 0 || nsave < 1 || n_snap < 0 || particle_offset < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (chunk == 0 || n_snap == 0) return PT_OK;
    if (!(d_mom && d_snap_steps && d_out)) return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    return launch_energy_snapshots(d_mom, chunk, nsave, d_snap_steps, n_snap, particle_offset, d_out, ctx->stream);
}

int pt_energy_histogram_device(pt_ctx* ctx, const float* d_mom, int64_t chunk, int64_t nsave,
                               const int64_t* d_snaps, int n_snap, double e_min, double e_max, int n_hist,
                               int64_t* d_counts)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (chunk < 0 || nsave < 1 || n_snap < 0 || n_hist < 1) return fail(PT_ERR_ARG, "bad sizes");
    if (!(e_min > 0.0 && e_max > e_min && std::isfinite(e_max))) return fail(PT_ERR_ARG, "need 0 < e_min < e_max");
    if (chunk == 0 || n_snap == 0) return PT_OK;
    if (!(d_mom && d_snaps && d_counts)) return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    return launch_energy_histogram(d_mom, chunk, nsave, d_snaps, n_snap, e_min, e_max, n_hist, d_counts, ctx->stream);
}

int pt_reconstruct_mu(pt_ctx* ctx, const void* pos, const void* mom, int64_t chunk, int64_t nsave,
                      const void* const bfield[3], const pt_grid* grid, int f64, void* mu_out)
{
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    int rc = check_grid(grid);
    if (rc) return rc;
    if (chunk < 0 || nsave < 0) return fail(PT_ERR_ARG, "bad sizes");
    if (chunk == 0 || nsave == 0) return PT_OK;
    if (!(pos && mom && mu_out && bfield && bfield[0] && bfield[1] && bfield[2])) return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    const size_t el = f64 ? 8 : 4;
    const size_t nps = (size_t)chunk * 3 * nsave, nf = (size_t)(grid->nx * grid->ny * grid->nz);
    DevBuf dp, dm, db, dout;
    if ((rc = dp.alloc(el * nps)) || (rc = dm.alloc(el * nps)) || (rc = db.alloc(3 * el * nf)) ||
        (rc = dout.alloc(el * (size_t)chunk * nsave)))
        return rc;
    cudaStream_t s = ctx->stream;
    PT_CUDA(cudaMemcpyAsync(dp.p, pos, el * nps, cudaMemcpyHostToDevice, s));
    PT_CUDA(cudaMemcpyAsync(dm.p, mom, el * nps, cudaMemcpyHostToDevice, s));
    const void* bd[3];
    for (int c = 0; c < 3; ++c) {
        bd[c] = (char*)db.p + c * el * nf;
        PT_CUDA(cudaMemcpyAsync((void*)bd[c], bfield[c], el * nf, cudaMemcpyHostToDevice, s));
    }
    rc = launch_reconstruct_mu(dp.p, dm.p, chunk, nsave, bd, *grid, f64, dout.p, s);
    if (rc) return rc;
    PT_CUDA(cudaMemcpyAsync(mu_out, dout.p, el * (size_t)chunk * nsave, cudaMemcpyDeviceToHost, s));
    PT_CUDA(cudaStreamSynchronize(s));
    return PT_OK;
}

}  // extern "C"
