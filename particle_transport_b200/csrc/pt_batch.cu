// Batched campaigns (pt_batch_*): an arena of particle slots shared by many
// campaigns, advanced together by push_batch_kernel.  See include/ptb200.h.
#include "pt_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace pt;

struct pt_batch {
    pt_ctx* ctx = nullptr;
    int64_t cap = 0;
    int max_camps = 0;
    int storage = PT_FIELD_BRICK_BF16;
    int K = 64;
    int sort = 1;
    int grid = 148;
    int threads = kBatchTile; // threads per block of the persistent push
    BatchStateDev buf[2]{};   // ping-pong state (each campaign's current buffer is its device-side par)
    int sort_grid = 1;        // blocks of the sort's tile kernels (a power of two >= the tiles, with slack)
    BatchCampaignDev* d_camps = nullptr;
    std::vector<BatchCampaignDev> h_camps;
    std::vector<const pt_field*> fields;
    BatchTile* d_tiles = nullptr;
    int* d_ntiles = nullptr;
    int* d_counter = nullptr;
    uint32_t* keys = nullptr;
    uint32_t* hist = nullptr;
    uint32_t* cursor = nullptr;
    int64_t hist_cap = 0;
    int64_t* d_m = nullptr;
    int smem_words = 1;
    std::vector<std::pair<int64_t, int64_t>> free_ranges;  // (start, length), sorted
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_dirty = true;
    // pinned staging of the campaign and tile tables (rebuild_tables)
    static constexpr int kStages = 4;
    struct Stage {
        void* host = nullptr;
        size_t bytes = 0;
        cudaEvent_t ev = nullptr;
        bool pending = false;  // an upload from it is enqueued
    } stage[kStages];
    int stage_next = 0;
    BatchCampaignDev* d_stage = nullptr;
    std::vector<BatchTile> tile_scratch;
};

namespace {

void free_state(BatchStateDev& s)
{
    if (s.x) cudaFree(s.x);
    if (s.p) cudaFree(s.p);
    if (s.p2) cudaFree(s.p2);
    if (s.pid) cudaFree(s.pid);
    if (s.alive) cudaFree(s.alive);
    s = BatchStateDev{};
}

int alloc_state(BatchStateDev& s, int64_t cap)
{
    s.cap = cap;
    const size_t m = (size_t)std::max<int64_t>(cap, 1);
    cudaError_t e = cudaMalloc((void**)&s.x, sizeof(double) * 3 * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s.p, sizeof(float) * 3 * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s.p2, sizeof(double) * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s.pid, sizeof(int32_t) * m);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s.alive, m);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PT_ERR_OOM, "batch state allocation failed");
    }
    return PT_OK;
}

void drop_graphs(pt_batch* b)
{
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->graph_dirty = true;
}

// Recompute sort buckets and tile table after the campaign set changed and
// upload them behind the epochs already enqueued, without waiting for them.
// The step counters are advanced on the device by every epoch, so the host
// table's steps are stale: batch_apply_kernel installs the new table but
// keeps each running campaign's device step (`fresh`, a campaign just added,
// takes its step 0 from the table).  The table goes through a ring of pinned
// staging buffers; one is written again only after its upload has run.
int rebuild_tables(pt_batch* b, int fresh)
{
    int64_t key = 0;
    std::vector<BatchTile>& tiles = b->tile_scratch;
    tiles.clear();
    for (int c = 0; c < b->max_camps; ++c) {
        BatchCampaignDev& C = b->h_camps[c];
        if (!C.active || !C.running) continue;
        C.key_base = key;
        key += C.n_bricks + 1;
        for (int64_t s = 0; s < C.n; s += kBatchTile)
            tiles.push_back(BatchTile{c, (int32_t)std::min<int64_t>(kBatchTile, C.n - s), C.slot0 + s});
    }
    if (key > UINT32_MAX) return fail(PT_ERR_ARG, "too many sort buckets in the batch");
    if (key > b->hist_cap) {
        const int64_t want = std::max<int64_t>(key, 2 * b->hist_cap);
        if (b->hist) cudaFree(b->hist);
        if (b->cursor) cudaFree(b->cursor);
        b->hist = b->cursor = nullptr;
        b->hist_cap = 0;
        cudaError_t e = cudaMalloc((void**)&b->hist, sizeof(uint32_t) * want);
        // cursor[want] followed by the scan's per-tile offsets
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->cursor, sizeof(uint32_t) * (want + sort_scan_tiles(want)));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PT_ERR_OOM, "batch sort buckets allocation failed");
        }
        b->hist_cap = want;
        drop_graphs(b);
    }
    const int nt = (int)tiles.size();
    const int64_t max_tiles = b->cap / kBatchTile + b->max_camps + 1;
    if (nt > max_tiles) return fail(PT_ERR_ARG, "internal: tile table overflow");
    {
        // the sort kernels run one block per tile; their grid is part of the
        // captured graphs, so it changes (and the graphs are captured again)
        // only when the tiles outgrow it or fall below a quarter of it
        int want = 1;
        while (want < nt && want < (1 << 30)) want <<= 1;
        if (want > b->sort_grid || 4 * want < b->sort_grid) {
            b->sort_grid = want;
            drop_graphs(b);
        }
    }
    // staging layout: campaigns | n_tiles (int) | buckets (int64) | tiles
    const size_t camps_bytes = sizeof(BatchCampaignDev) * (size_t)b->max_camps;
    const size_t o_nt = (camps_bytes + 15) & ~(size_t)15, o_m = o_nt + 16, o_tiles = o_m + 16;
    const size_t need = o_tiles + sizeof(BatchTile) * (size_t)nt;
    pt_batch::Stage& S = b->stage[b->stage_next];
    b->stage_next = (b->stage_next + 1) % pt_batch::kStages;
    if (S.pending) {
        PT_CUDA(cudaEventSynchronize(S.ev));
        S.pending = false;
    }
    if (S.bytes < need) {
        if (S.host) cudaFreeHost(S.host);
        S.host = nullptr;
        S.bytes = 0;
        const size_t want = std::max(need + need / 2, (size_t)1 << 16);
        cudaError_t e = cudaMallocHost(&S.host, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            S.host = nullptr;
            return fail(PT_ERR_OOM, "pinned staging allocation of the batch tables failed");
        }
        S.bytes = want;
    }
    char* h = (char*)S.host;
    std::memcpy(h, b->h_camps.data(), camps_bytes);
    std::memcpy(h + o_nt, &nt, sizeof(int));
    std::memcpy(h + o_m, &key, sizeof(int64_t));
    if (nt) std::memcpy(h + o_tiles, tiles.data(), sizeof(BatchTile) * (size_t)nt);
    cudaStream_t s = b->ctx->stream;
    PT_CUDA(cudaMemcpyAsync(b->d_stage, h, camps_bytes, cudaMemcpyHostToDevice, s));
    if (nt) PT_CUDA(cudaMemcpyAsync(b->d_tiles, h + o_tiles, sizeof(BatchTile) * nt, cudaMemcpyHostToDevice, s));
    PT_CUDA(cudaMemcpyAsync(b->d_ntiles, h + o_nt, sizeof(int), cudaMemcpyHostToDevice, s));
    PT_CUDA(cudaMemcpyAsync(b->d_m, h + o_m, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    int rc = launch_batch_apply(b->d_camps, b->d_stage, b->max_camps, fresh, s);
    if (rc) return rc;
    PT_CUDA(cudaEventRecord(S.ev, s));
    S.pending = true;
    return PT_OK;
}

// One epoch: re-sort the campaigns due for it (each into its other buffer),
// push every running campaign K steps from its own buffer, advance the
// device-side counters.  Every decision is made on the device from the
// campaign table, so one captured graph replays every epoch.
int enqueue_epoch(pt_batch* b, cudaStream_t s)
{
    if (b->sort) {
        int rc = launch_batch_sort(b->d_camps, b->max_camps, b->d_tiles, b->d_ntiles, b->sort_grid, b->buf[0],
                                   b->buf[1], b->keys, b->hist, b->cursor, b->d_m, b->hist_cap, b->ctx->num_sms, s);
        if (rc) return rc;
    }
    BatchLaunch L{b->d_camps, b->d_tiles, b->d_ntiles, b->d_counter, {b->buf[0], b->buf[1]}, b->sort,
                  field_layout(b->storage), b->smem_words, b->grid, b->threads};
    int rc = launch_push_batch(L, s);
    if (rc) return rc;
    return launch_batch_epoch_end(b->d_camps, b->max_camps, b->d_counter, b->sort, s);
}

int capture(pt_batch* b)
{
    cudaGraph_t g = nullptr;
    PT_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_epoch(b, b->cap_stream);
    cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return PT_OK;
}

}  // namespace

extern "C" {

int pt_batch_create(pt_ctx* ctx, int64_t capacity, int max_campaigns, int storage, int steps_per_epoch, int sort,
                    int blocks_per_sm, pt_batch** out)
{
    if (!ctx || !out) return fail(PT_ERR_ARG, "null argument");
    if (capacity < 1 || capacity > INT32_MAX) return fail(PT_ERR_ARG, "capacity must be in [1, 2^31)");
    if (max_campaigns < 1 || max_campaigns > 4096) return fail(PT_ERR_ARG, "max_campaigns must be in [1, 4096]");
    if (storage != PT_FIELD_BRICK_BF16 && storage != PT_FIELD_BRICK_F32 && storage != PT_FIELD_BRICK_BF16_XPAIR)
        return fail(PT_ERR_ARG, "batches run the FP32 push: storage must be a brick form");
    if (steps_per_epoch < 1) return fail(PT_ERR_ARG, "steps_per_epoch must be >= 1");
    PT_DEVICE_SCOPE(ctx->device);
    pt_batch* b = new (std::nothrow) pt_batch();
    if (!b) return fail(PT_ERR_OOM, "host allocation failed");
    b->ctx = ctx;
    b->cap = capacity;
    b->max_camps = max_campaigns;
    b->storage = storage;
    b->K = steps_per_epoch;
    b->sort = sort ? 1 : 0;
    b->h_camps.assign(max_campaigns, BatchCampaignDev{});
    b->fields.assign(max_campaigns, nullptr);
    b->free_ranges.push_back({0, capacity});
    int rc = alloc_state(b->buf[0], capacity);
    if (!rc && b->sort) rc = alloc_state(b->buf[1], capacity);
    const int64_t max_tiles = capacity / kBatchTile + max_campaigns + 1;
    cudaError_t e = cudaSuccess;
    if (!rc) {
        e = cudaMalloc((void**)&b->d_camps, sizeof(BatchCampaignDev) * max_campaigns);
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_stage, sizeof(BatchCampaignDev) * max_campaigns);
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_tiles, sizeof(BatchTile) * max_tiles);
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_ntiles, sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_counter, sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_m, sizeof(int64_t));
        if (e == cudaSuccess && b->sort) e = cudaMalloc((void**)&b->keys, sizeof(uint32_t) * capacity);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
        for (auto& st : b->stage)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cudaGetLastError();
            rc = fail(PT_ERR_OOM, "batch allocation failed");
        }
    }
    if (!rc) {
        cudaStream_t s = ctx->stream;
        const int zero = 0;
        const int64_t zero64 = 0;
        e = cudaMemsetAsync(b->d_camps, 0, sizeof(BatchCampaignDev) * max_campaigns, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_ntiles, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_counter, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_m, &zero64, sizeof(int64_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "batch init");
    }
    if (rc) {
        pt_batch_destroy(b);
        return rc;
    }
    // persistent grid: resident blocks of push_batch_kernel per SM
    const int per_sm = blocks_per_sm > 0 ? std::min(blocks_per_sm, 8) : 2;
    b->grid = ctx->num_sms * per_sm;
    *out = b;
    return PT_OK;
}

int pt_batch_add(pt_ctx* ctx, pt_batch* b, const pt_campaign_desc* d, int* id)
{
    if (!ctx || !b || !d || !id) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    const pt_field* f = d->field;
    if (!f || f->storage != b->storage) return fail(PT_ERR_ARG, "campaign field must use the batch's brick storage");
    if (!(d->dt > 0 && std::isfinite(d->dt))) return fail(PT_ERR_ARG, "dt must be finite and positive");
    if (d->nsteps < 1 || d->stride < 1) return fail(PT_ERR_ARG, "nsteps and stride must be >= 1");
    if (d->n < 1) return fail(PT_ERR_ARG, "a campaign needs at least one particle");
    if (!(d->d_x1 && d->d_x2 && d->d_x3 && d->d_p1 && d->d_p2 && d->d_p3 && d->d_alive))
        return fail(PT_ERR_ARG, "null state");
    if (d->d_cache && d->cache_rows < 1) return fail(PT_ERR_ARG, "cache_rows must be >= 1");
    if (d->d_cache && !d->cache_ring && d->cache_rows < (d->nsteps - 1) / d->stride + 1)
        return fail(PT_ERR_ARG, "a non-ring cache needs one row per save");
    if (d->d_mom_cache && (!d->d_cache || d->n_mom < 1 || d->n_mom > d->n))
        return fail(PT_ERR_ARG, "a momenta cache needs the mu cache and 1 <= n_mom <= n");
    if (d->sort_every < 0) return fail(PT_ERR_ARG, "sort_every must be >= 0");
    if (d->cache_pitch < 0 || (d->d_cache && d->cache_pitch > 0 && d->cache_pitch < d->cache_rows))
        return fail(PT_ERR_ARG, "cache_pitch must be 0 (rows) or at least cache_rows (time-fastest)");
    int c = -1;
    for (int i = 0; i < b->max_camps; ++i)
        if (!b->h_camps[i].active) {
            c = i;
            break;
        }
    if (c < 0) return fail(PT_ERR_STATE, "batch is full (max_campaigns)");
    int64_t slot0 = -1;
    for (auto& r : b->free_ranges)
        if (r.second >= d->n) {
            slot0 = r.first;
            r.first += d->n;
            r.second -= d->n;
            break;
        }
    if (slot0 < 0) return fail(PT_ERR_OOM, "no free slot range of " + std::to_string(d->n) + " particles in the batch");
    b->free_ranges.erase(std::remove_if(b->free_ranges.begin(), b->free_ranges.end(),
                                        [](const std::pair<int64_t, int64_t>& r) { return r.second == 0; }),
                         b->free_ranges.end());
    cudaStream_t s = ctx->stream;
    // a new campaign starts in buffer 0
    int rc = launch_batch_import(b->buf[0], slot0, d->n, f, d->d_x1, d->d_x2, d->d_x3, d->d_p1, d->d_p2,
                                 d->d_p3, d->d_alive, ctx->num_sms, s);
    if (rc) return rc;
    BatchCampaignDev C{};
    const pt_grid& g = f->grid;
    PushArgsFast& a = C.a;
    a.fld.nodes = f->nodes;
    a.fld.offs = f->offs;
    a.fld.nx = g.nx; a.fld.ny = g.ny; a.fld.nz = g.nz;
    a.fld.bf16 = f->storage != PT_FIELD_BRICK_F32;
    a.fld.layout = field_layout(f->storage);
    a.fld.tex = f->tex;
    for (int k = 0; k < 3; ++k) a.fld.boff[k] = f->boff[k];
    a.wx = (g.xmax - g.xmin) / g.dx;
    a.wy = (g.ymax - g.ymin) / g.dy;
    a.wz = (g.zmax - g.zmin) / g.dz;
    a.n = d->n;
    a.hB = (float)(Q_E * f->B_ref * d->dt / (2.0 * M_P));
    a.vfac[0] = (float)(C_LIGHT * d->dt / g.dx);
    a.vfac[1] = (float)(C_LIGHT * d->dt / g.dy);
    a.vfac[2] = (float)(C_LIGHT * d->dt / g.dz);
    a.xmin[0] = g.xmin; a.xmin[1] = g.ymin; a.xmin[2] = g.zmin;
    a.dxs[0] = g.dx; a.dxs[1] = g.dy; a.dxs[2] = g.dz;
    a.nsteps = d->nsteps;
    a.stride = d->stride;
    a.periodic = d->periodic;
    a.cache_mode = d->d_cache ? PT_CACHE_MU : PT_CACHE_NONE;
    a.cache_f64 = d->cache_f64;
    a.cache = d->d_cache;
    a.row_base = 0;
    a.rows = d->cache_rows;
    a.ring = d->cache_ring;
    a.n_cache = d->n;
    a.deaths = d->d_deaths;
    a.mom_cache = d->d_mom_cache;
    a.n_mom = d->d_mom_cache ? d->n_mom : 0;
    a.pitch = d->d_cache ? d->cache_pitch : 0;
    C.slot0 = slot0;
    C.n = d->n;
    C.step = 0;
    C.K = b->K;
    C.n_bricks = (f->n_nodes + 511) / 512;
    C.epochs = 0;
    C.sort_every = b->sort ? std::max(d->sort_every, 1) : 0;
    C.par = 0;
    C.active = 1;
    C.running = 1;
    b->h_camps[c] = C;
    b->fields[c] = f;
    const int words = (int)(g.nx + g.ny + g.nz);
    if (words > b->smem_words) {
        b->smem_words = words;
        drop_graphs(b);
    }
    rc = rebuild_tables(b, c);
    if (rc) return rc;
    *id = c;
    return PT_OK;
}

int pt_batch_remove(pt_ctx* ctx, pt_batch* b, int id)
{
    if (!ctx || !b) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (id < 0 || id >= b->max_camps || !b->h_camps[id].active) return fail(PT_ERR_ARG, "no such campaign");
    BatchCampaignDev& C = b->h_camps[id];
    b->free_ranges.push_back({C.slot0, C.n});
    std::sort(b->free_ranges.begin(), b->free_ranges.end());
    std::vector<std::pair<int64_t, int64_t>> merged;
    for (auto& r : b->free_ranges) {
        if (!merged.empty() && merged.back().first + merged.back().second == r.first) merged.back().second += r.second;
        else merged.push_back(r);
    }
    b->free_ranges.swap(merged);
    C = BatchCampaignDev{};
    b->fields[id] = nullptr;
    return rebuild_tables(b, -1);
}

int pt_batch_run(pt_ctx* ctx, pt_batch* b, int64_t epochs, int use_graph)
{
    if (!ctx || !b) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (epochs < 0) return fail(PT_ERR_ARG, "epochs must be >= 0");
    cudaStream_t s = ctx->stream;
    if (use_graph) {
        if (b->graph_dirty) {
            drop_graphs(b);
            int rc = capture(b);
            if (rc) return rc;
            b->graph_dirty = false;
        }
        for (int64_t e = 0; e < epochs; ++e) PT_CUDA(cudaGraphLaunch(b->graph, s));
        return PT_OK;
    }
    for (int64_t e = 0; e < epochs; ++e) {
        int rc = enqueue_epoch(b, s);
        if (rc) return rc;
    }
    return PT_OK;
}

int pt_batch_set_running(pt_ctx* ctx, pt_batch* b, const int* ids, int n_ids)
{
    if (!ctx || !b) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (n_ids > 0 && !ids) return fail(PT_ERR_ARG, "null ids");
    std::vector<char> want((size_t)b->max_camps, n_ids < 0 ? 1 : 0);
    for (int k = 0; k < n_ids; ++k) {
        const int id = ids[k];
        if (id < 0 || id >= b->max_camps || !b->h_camps[id].active) return fail(PT_ERR_ARG, "no such campaign");
        want[id] = 1;
    }
    bool changed = false;
    for (int c = 0; c < b->max_camps; ++c) {
        BatchCampaignDev& C = b->h_camps[c];
        if (!C.active || (int)want[c] == C.running) continue;
        // a paused campaign's slots stay in the buffer they are in (its
        // device-side par); neither the sort nor the push touches them
        C.running = want[c];
        changed = true;
    }
    return changed ? rebuild_tables(b, -1) : PT_OK;
}

int pt_batch_set_launch(pt_ctx* ctx, pt_batch* b, int threads_per_block, int blocks_per_sm)
{
    if (!ctx || !b) return fail(PT_ERR_ARG, "null argument");
    if (threads_per_block != 64 && threads_per_block != 128 && threads_per_block != kBatchTile)
        return fail(PT_ERR_ARG, "threads_per_block must be 64, 128 or 256");
    if (blocks_per_sm < 1 || blocks_per_sm > 16) return fail(PT_ERR_ARG, "blocks_per_sm must be in [1, 16]");
    PT_DEVICE_SCOPE(ctx->device);
    b->threads = threads_per_block;
    b->grid = ctx->num_sms * blocks_per_sm;
    drop_graphs(b);  // the next epoch captures the new shape
    return PT_OK;
}

int pt_batch_step(pt_ctx* ctx, pt_batch* b, int id, int64_t* step)
{
    if (!ctx || !b || !step) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (id < 0 || id >= b->max_camps || !b->h_camps[id].active) return fail(PT_ERR_ARG, "no such campaign");
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    PT_CUDA(cudaMemcpy(step, &b->d_camps[id].step, sizeof(int64_t), cudaMemcpyDeviceToHost));
    return PT_OK;
}

int pt_batch_export(pt_ctx* ctx, pt_batch* b, int id, double* x1, double* x2, double* x3, double* p1, double* p2,
                    double* p3, uint8_t* alive)
{
    if (!ctx || !b) return fail(PT_ERR_ARG, "null argument");
    PT_DEVICE_SCOPE(ctx->device);
    if (id < 0 || id >= b->max_camps || !b->h_camps[id].active) return fail(PT_ERR_ARG, "no such campaign");
    if (!(x1 && x2 && x3 && p1 && p2 && p3 && alive)) return fail(PT_ERR_ARG, "null state");
    const BatchCampaignDev& C = b->h_camps[id];
    return launch_batch_export(b->buf[0], b->buf[1], b->d_camps, id, C.slot0, C.n, b->fields[id], x1, x2, x3, p1, p2,
                               p3, alive, ctx->num_sms, ctx->stream);
}

int pt_batch_destroy(pt_batch* b)
{
    if (!b) return PT_OK;
    if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
    drop_graphs(b);
    free_state(b->buf[0]);
    free_state(b->buf[1]);
    for (auto& st : b->stage) {
        if (st.host) cudaFreeHost(st.host);
        if (st.ev) cudaEventDestroy(st.ev);
    }
    for (void* p : {(void*)b->d_stage, (void*)b->d_camps, (void*)b->d_tiles, (void*)b->d_ntiles, (void*)b->d_counter,
                    (void*)b->keys, (void*)b->hist, (void*)b->cursor, (void*)b->d_m})
        if (p) cudaFree(p);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    delete b;
    return PT_OK;
}

}  // extern "C"
