// Host side of pt_push_run: moving the caller's pageable state arrays to and
// from the device.
//
// A pageable cudaMemcpy goes through the driver's own small staging buffers
// at roughly a fifth of the DMA rate.  Here the bytes go through pinned
// chunks owned by the context instead: host threads fill chunk j (or drain
// it) while the copy engine moves chunk j - 1, so the link runs near its
// pinned rate.  The pinned buffer is grow-only and lives until
// pt_ctx_trim / pt_ctx_destroy, so repeated calls do not pin memory again.
#include "pt_internal.cuh"

#include <atomic>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>

namespace pt {
namespace {

// A fixed set of host threads that run fn(0..n-1) with the caller.
class HostPool {
  public:
    static HostPool& get()
    {
        static HostPool pool;
        return pool;
    }
    void run(int n, const std::function<void(int)>& fn)
    {
        std::lock_guard<std::mutex> serial(run_m_);  // callers on several host threads take turns
        if (workers_.empty() || n <= 1) {
            for (int i = 0; i < n; ++i) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &fn;
            n_ = n;
            next_.store(0);
            pending_ = (int)workers_.size();
            ++gen_;
        }
        cv_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
        fn_ = nullptr;
    }

  private:
    HostPool()
    {
        // workers besides the calling thread: 7 (at most hardware threads - 1),
        // or PTB200_HOST_THREADS - 1
        const unsigned hw = std::thread::hardware_concurrency();
        int k = (int)std::min<unsigned>(7u, hw > 1 ? hw - 1 : 0u);
        if (const char* e = std::getenv("PTB200_HOST_THREADS")) {
            const int t = std::atoi(e);
            if (t >= 1) k = std::min(t - 1, 63);
        }
        for (int i = 0; i < k; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    void drain()
    {
        for (int i; (i = next_.fetch_add(1)) < n_;) (*fn_)(i);
    }
    void loop()
    {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            drain();
            std::lock_guard<std::mutex> lk(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex run_m_, m_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* fn_ = nullptr;
    int n_ = 0, pending_ = 0;
    std::atomic<int> next_{0};
    uint64_t gen_ = 0;
    bool stop_ = false;
};

constexpr size_t kPiece = 4u << 20;  // bytes per host thread task

void parallel_copy(char* dst, const char* src, size_t bytes)
{
    const int parts = (int)((bytes + kPiece - 1) / kPiece);
    HostPool::get().run(parts, [&](int i) {
        const size_t off = (size_t)i * kPiece;
        std::memcpy(dst + off, src + off, std::min(kPiece, bytes - off));
    });
}

struct Events {
    std::vector<cudaEvent_t> ev;
    explicit Events(int n) : ev((size_t)n, nullptr)
    {
        for (auto& e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    ~Events()
    {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    bool ok() const
    {
        for (auto e : ev)
            if (!e) return false;
        return true;
    }
};

}  // namespace

int pinned_get(pt_ctx* ctx, size_t bytes, void** out)
{
    ScratchBuf& b = ctx->pinned;
    if (b.bytes < bytes) {
        if (b.ptr) {
            cudaStreamSynchronize(ctx->stream);
            cudaStreamSynchronize(ctx->copy_stream);
            cudaFreeHost(b.ptr);
        }
        b.ptr = nullptr;
        b.bytes = 0;
        cudaError_t e = cudaMallocHost(&b.ptr, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PT_ERR_OOM, "pinned host allocation of " + std::to_string(bytes) + " bytes failed");
        }
        b.bytes = bytes;
    }
    *out = b.ptr;
    return PT_OK;
}

int staged_h2d(const std::vector<HostSeg>& segs, char* stage, size_t chunk, int nbuf, cudaStream_t s)
{
    Events E(nbuf);
    if (!E.ok()) return fail(PT_ERR_CUDA, "event creation failed");
    int64_t j = 0;
    for (const HostSeg& g : segs) {
        for (size_t off = 0; off < g.bytes; off += chunk, ++j) {
            const size_t len = std::min(chunk, g.bytes - off);
            const int b = (int)(j % nbuf);
            char* buf = stage + (size_t)b * chunk;
            if (j >= nbuf) PT_CUDA(cudaEventSynchronize(E.ev[b]));  // the DMA out of this buffer is done
            parallel_copy(buf, g.host + off, len);
            PT_CUDA(cudaMemcpyAsync(g.dev + off, buf, len, cudaMemcpyHostToDevice, s));
            PT_CUDA(cudaEventRecord(E.ev[b], s));
        }
    }
    // the staging buffer may be rewritten as soon as this returns
    for (auto e : E.ev) PT_CUDA(cudaEventSynchronize(e));
    return PT_OK;
}

int staged_d2h(const std::vector<HostSeg>& segs, char* stage, size_t chunk, int nbuf, cudaStream_t s)
{
    Events E(nbuf);
    if (!E.ok()) return fail(PT_ERR_CUDA, "event creation failed");
    struct Pending {
        char* host;
        const char* buf;
        size_t len;
        int b;
    };
    std::deque<Pending> q;
    auto drain_one = [&]() -> int {
        const Pending p = q.front();
        q.pop_front();
        PT_CUDA(cudaEventSynchronize(E.ev[p.b]));
        parallel_copy(p.host, p.buf, p.len);
        return PT_OK;
    };
    int64_t j = 0;
    for (const HostSeg& g : segs) {
        for (size_t off = 0; off < g.bytes; off += chunk, ++j) {
            const size_t len = std::min(chunk, g.bytes - off);
            const int b = (int)(j % nbuf);
            if ((int)q.size() == nbuf) {  // the oldest pending copy holds buffer b
                int rc = drain_one();
                if (rc) return rc;
            }
            char* buf = stage + (size_t)b * chunk;
            PT_CUDA(cudaMemcpyAsync(buf, g.dev + off, len, cudaMemcpyDeviceToHost, s));
            PT_CUDA(cudaEventRecord(E.ev[b], s));
            q.push_back(Pending{g.host + off, buf, len, b});
        }
    }
    while (!q.empty()) {
        int rc = drain_one();
        if (rc) return rc;
    }
    return PT_OK;
}

int64_t count_nonzero(const uint8_t* v, int64_t n)
{
    const int64_t piece = 1 << 22;
    const int parts = (int)((n + piece - 1) / piece);
    std::vector<int64_t> part((size_t)std::max(parts, 1), 0);
    HostPool::get().run(parts, [&](int i) {
        const int64_t a = (int64_t)i * piece, b = std::min(n, a + piece);
        int64_t c = 0;
        for (int64_t k = a; k < b; ++k) c += v[k] != 0;
        part[(size_t)i] = c;
    });
    int64_t t = 0;
    for (int64_t c : part) t += c;
    return t;
}

}  // namespace pt
