// Continuous-batching request loop for permanents of mixed size and type.
//
//   submit ─► admission: the request's matrix needs room in the device pool
//      (cfg.admit_bytes of device memory, first fit in 256-byte units); the
//      matrix is copied into the pool's page-locked host mirror at the same
//      offset, and stays reserved until the request completes.
//      A real matrix with zeros is first pruned and decomposed on the host
//      (spb_plan_pieces: perfect-matching pruning, connected components,
//      DecomposePerman); its pieces are admitted as independent child
//      requests, and the parent completes with the product over components
//      of the sum of their pieces' permanents.
//   ─► per-(n, real/complex) queues:
//      small (n <= kSmallN): the batch worker packs up to max_batch requests
//        of one shape into a free slot: H2D copy of the slot's offset table,
//        then batch_walk, whose warps each copy their matrix from the pinned
//        mirror into its reserved device location and compute its permanent
//        there, then D2H of the results, all on the small stream;
//        replayed from one CUDA graph per (shape, padded count, slot) once
//        that key has been used kGraphAfterUses times.  Completion is
//        detected with an event per slot, so up to `slots` batches are in
//        flight while new requests keep arriving.
//      mid (kSmallN < n <= batch_max_n): batched like the small ones when
//        their queue holds enough requests to beat single calls
//        (mid_batch_min), else handed to the large queue.
//      large: `large_workers` threads each run the whole-GPU walk through
//        their own device context (stream, events, arenas), so the host work
//        and short kernels of one call overlap the walk of another; matrices
//        are copied from the mirror into the pool on that context's stream
//        (real matrices with zeros go through the host entry, whose planner
//        may pick the row-compacted walk).
//   poll / wait ─► result with admission and completion timestamps.
//
// A request's result depends only on its own matrix: the batch kernel gives
// each matrix its own warp, tables and reduction (padding entries read a
// zero matrix and are discarded), and the whole-GPU walk's result does not
// depend on what else runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "context.h"
#include "dense_host.h"
#include "spb_common.cuh"

namespace spb {
namespace serve {

constexpr int kSmallN = 20;                   // always batched up to here
constexpr int kMaxN = batch::kMaxN;           // batch kernel limit (24)
constexpr size_t kUnit = batch::kOffsetUnit * sizeof(double);  // pool granule, 256 B
constexpr int kGraphAfterUses = 3;            // uses of a key before its graph is captured

// Mid-size shapes are batched when at least this many requests of the shape
// are queued: one warp per matrix takes about 2^(n-21) * 1.5 ms at n > 20,
// a whole-GPU call about 0.1 ms, so batching pays from ~16 * 2^(n-21)
// requests on.
inline size_t mid_batch_min(int n) { return (size_t)16 << (n > 21 ? n - 21 : 0); }

// Host-side double-double product (Dekker with exact FMA).
inline dd dd_mul_host(dd a, dd b)
{
    const double p = mul_rn(a.hi, b.hi);
    double e = std::fma(a.hi, b.hi, -p);
    e = std::fma(a.hi, b.lo, e);
    e = std::fma(a.lo, b.hi, e);
    return fast_two_sum(p, e);
}

// Pool allocator over [0, size) in kUnit granules: a free list per block
// size (requests recur in a few sizes), a bump pointer for new blocks, and,
// when both fail, the smallest larger free block split in two.  When the
// pool empties it is reset, which undoes any fragmentation.
class PoolMap {
public:
    void reset(size_t units)
    {
        size_ = units;
        top_ = 0;
        used_ = 0;
        for (auto& l : by_size_) l.clear();
    }
    bool take(size_t units, size_t* off)
    {
        if (units == 0 || units >= kClasses) return bump(units, off);
        auto& l = by_size_[units];
        if (!l.empty()) {
            *off = l.back();
            l.pop_back();
            used_ += units;
            return true;
        }
        if (bump(units, off)) return true;
        for (size_t u = units + 1; u < kClasses; ++u)
            if (!by_size_[u].empty()) {
                *off = by_size_[u].back();
                by_size_[u].pop_back();
                by_size_[u - units].push_back(*off + units);
                used_ += units;
                return true;
            }
        return false;
    }
    void give(size_t off, size_t units)
    {
        used_ -= units;
        if (units < kClasses) by_size_[units].push_back(off);
        if (used_ == 0) reset(size_);
    }
    size_t used() const { return used_; }

private:
    bool bump(size_t units, size_t* off)
    {
        if (top_ + units > size_) return false;
        *off = top_;
        top_ += units;
        used_ += units;
        return true;
    }
    // blocks up to 63 x 63 complex (249 granules) have their own lists
    static constexpr size_t kClasses = 256;
    std::vector<size_t> by_size_[kClasses];
    size_t size_ = 0, top_ = 0, used_ = 0;
};

struct Request {
    int n = 0, comps = 1;
    size_t off = 0, units = 0;  // device pool reservation (kUnit granules)
    bool zeros = false;         // real matrix with a zero entry
    double t_submit = 0, t_done = 0;
    double res[4] = {0, 0, 0, 0};
    int status = SPB_ERR_BUSY;  // SPB_ERR_BUSY while pending
    bool done = false, cancelled = false, in_flight = false;
    // decomposed requests: the parent holds per-component sums of its pieces
    uint64_t parent = 0;        // nonzero for a piece
    int component = 0;
    int pending = 0;            // parent: pieces not yet complete
    int child_status = SPB_OK;  // parent: first failure among its pieces
    std::vector<dd> comp_sum;   // parent: per component
    std::vector<uint64_t> children;
};

struct Slot {
    unsigned* d_offs = nullptr;
    unsigned* h_offs = nullptr;
    double* d_out = nullptr;
    double* h_out = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    int n = 0, comps = 1, count = 0;
    std::vector<uint64_t> ids;
};

struct GraphKey {
    int n, comps, bucket, slot;
    bool operator<(const GraphKey& o) const
    {
        return std::tie(n, comps, bucket, slot) < std::tie(o.n, o.comps, o.bucket, o.slot);
    }
};

class Server {
public:
    explicit Server(const spb_server_config& c) : cfg(c) {}
    ~Server();
    int start();
    int submit(const double* a, int n, int comps, uint64_t* ticket);
    int poll(uint64_t id, spb_request_result* out, bool erase);
    int wait(uint64_t id, double timeout_s, spb_request_result* out);
    int cancel(uint64_t id);
    void stats(spb_server_stats* out);

private:
    void batch_loop();
    void large_loop(DeviceContext* ctx);
    bool harvest();                 // completes finished slots; true if any
    bool launch_ready(bool force);  // starts a batch if a slot and a shape are ready
    int launch_slot(int si, int n, int comps, std::vector<uint64_t>& ids);
    void finish(uint64_t id, Request& r, int status);  // with mu held
    void enqueue(uint64_t id, const Request& r);       // with mu held
    int admit(const double* a, int n, int comps, uint64_t parent, int component, uint64_t* id);
    int submit_split(const double* a, int n, uint64_t* ticket);

    spb_server_config cfg;
    int device = 0;
    cudaStream_t small_stream = nullptr;
    std::vector<Slot> slots;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    std::map<GraphKey, int> key_uses;

    // device pool and its mapped host mirror (same offsets)
    double* d_pool = nullptr;
    double* h_pool = nullptr;
    double* h_pool_dev = nullptr;  // the mirror as seen from the device
    size_t pool_units = 0;
    size_t zero_off = 0;           // a zero matrix of the largest batched shape (padding)
    size_t zero_units = 0;
    PoolMap pool;

    std::mutex mu;
    std::condition_variable cv_work, cv_large, cv_done;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> small_q[2][kMaxN + 1];
    std::deque<uint64_t> large_q;
    uint64_t next_id = 1;
    bool stopping = false;
    std::thread t_batch;
    std::vector<std::thread> t_large;
    std::vector<DeviceContext*> large_ctx;
    spb_server_stats st{};
};

}  // namespace serve
}  // namespace spb

extern "C" int spb_plan_pieces(const double* a, int n, int* components, int* count, int* sizes,
                               int* piece_component, double* data, int max_pieces, size_t max_doubles);

namespace spb {
namespace serve {

int Server::start()
{
    if (cfg.batch_max_n <= 0) cfg.batch_max_n = kMaxN;
    if (cfg.batch_max_n > kMaxN) cfg.batch_max_n = kMaxN;
    if (cfg.max_batch <= 0) cfg.max_batch = 2048;
    if (cfg.slots <= 0) cfg.slots = 4;
    if (cfg.max_wait_s <= 0) cfg.max_wait_s = 200e-6;
    if (cfg.admit_bytes == 0) cfg.admit_bytes = (size_t)256 << 20;
    if (cfg.large_workers <= 0) cfg.large_workers = 2;
    device = cfg.device;
    int st0 = SPB_OK;
    if (!get_context(device, &st0)) return st0;  // device checks, kernel set-up of the shared context
    SPB_CUDA_TRY(cudaSetDevice(device));
    // Batches go on the highest-priority stream: when SMs free up between
    // whole-GPU walks, a waiting batch is scheduled before the next walk.
    int prio_lo = 0, prio_hi = 0;
    SPB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    SPB_CUDA_TRY(cudaStreamCreateWithPriority(&small_stream, cudaStreamNonBlocking, prio_hi));
    // device pool: admitted matrices, plus one zero matrix for padding
    // the zero block sits after the requests' part, outside the allocator
    zero_units = (sizeof(double) * kMaxN * kMaxN * 2 + kUnit - 1) / kUnit;
    pool_units = cfg.admit_bytes / kUnit + zero_units;
    if (injected_failure("serving pool") || cudaMalloc(&d_pool, pool_units * kUnit) != cudaSuccess ||
        cudaHostAlloc(&h_pool, pool_units * kUnit, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
        cudaHostGetDevicePointer(&h_pool_dev, h_pool, 0) != cudaSuccess) {
        cudaGetLastError();
        spb_set_error("spb_server_create: could not allocate the %zu-byte request pool", pool_units * kUnit);
        return SPB_ERR_OOM;
    }
    pool.reset(pool_units - zero_units);
    zero_off = pool_units - zero_units;
    std::memset(h_pool + zero_off * batch::kOffsetUnit, 0, zero_units * kUnit);
    SPB_CUDA_TRY(cudaMemset(d_pool + zero_off * batch::kOffsetUnit, 0, zero_units * kUnit));
    slots.resize(cfg.slots);
    for (auto& s : slots) {
        if (injected_failure("serving slot") ||
            cudaMalloc(&s.d_offs, sizeof(unsigned) * cfg.max_batch) != cudaSuccess ||
            cudaMalloc(&s.d_out, sizeof(double) * 4 * cfg.max_batch) != cudaSuccess ||
            cudaMallocHost(&s.h_offs, sizeof(unsigned) * cfg.max_batch) != cudaSuccess ||
            cudaMallocHost(&s.h_out, sizeof(double) * 4 * cfg.max_batch) != cudaSuccess) {
            cudaGetLastError();
            spb_set_error("spb_server_create: could not allocate %d batch slots", cfg.slots);
            return SPB_ERR_OOM;
        }
        SPB_CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
    }
    for (int k = 0; k < cfg.large_workers; ++k) {
        DeviceContext* ctx = create_context(device, &st0);
        if (!ctx) return st0;
        large_ctx.push_back(ctx);
    }
    t_batch = std::thread(&Server::batch_loop, this);
    for (DeviceContext* ctx : large_ctx) t_large.emplace_back(&Server::large_loop, this, ctx);
    return SPB_OK;
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lk(mu);
        stopping = true;
    }
    cv_work.notify_all();
    cv_large.notify_all();
    if (t_batch.joinable()) t_batch.join();
    for (auto& t : t_large)
        if (t.joinable()) t.join();
    for (DeviceContext* ctx : large_ctx) destroy_context(ctx);
    cudaSetDevice(device);
    if (small_stream) cudaStreamSynchronize(small_stream);
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto& s : slots) {
        if (s.ev) cudaEventDestroy(s.ev);
        if (s.d_offs) cudaFree(s.d_offs);
        if (s.d_out) cudaFree(s.d_out);
        if (s.h_offs) cudaFreeHost(s.h_offs);
        if (s.h_out) cudaFreeHost(s.h_out);
    }
    if (d_pool) cudaFree(d_pool);
    if (h_pool) cudaFreeHost(h_pool);
    if (small_stream) cudaStreamDestroy(small_stream);
}

void Server::enqueue(uint64_t id, const Request& r)
{
    if (r.n <= cfg.batch_max_n) {
        small_q[r.comps - 1][r.n].push_back(id);
        cv_work.notify_one();
    } else {
        large_q.push_back(id);
        cv_large.notify_one();
    }
}

// Reserves pool room for one matrix and copies it into the mirror (mu held).
int Server::admit(const double* a, int n, int comps, uint64_t parent, int component, uint64_t* id)
{
    const size_t doubles = (size_t)n * n * comps;
    const size_t units = (doubles * sizeof(double) + kUnit - 1) / kUnit;
    size_t off = 0;
    if (!pool.take(units, &off)) return SPB_ERR_BUSY;
    const uint64_t k = next_id++;
    Request& r = reqs[k];
    r.n = n;
    r.comps = comps;
    r.off = off;
    r.units = units;
    r.parent = parent;
    r.component = component;
    r.t_submit = wall_seconds();
    double* dst = h_pool + off * batch::kOffsetUnit;
    std::memcpy(dst, a, doubles * sizeof(double));
    if (comps == 1)
        for (size_t i = 0; i < doubles && !r.zeros; ++i) r.zeros = dst[i] == 0.0;
    *id = k;
    return SPB_OK;
}

int Server::submit(const double* a, int n, int comps, uint64_t* ticket)
{
    if (!a || !ticket || n < 1 || n > 63) {
        spb_set_error("spb_server_submit: null pointer or n=%d outside 1..63", n);
        return SPB_ERR_INVALID;
    }
    if (comps == 1 && cfg.split >= 0) {
        bool zeros = false;
        for (size_t i = 0; i < (size_t)n * n && !zeros; ++i) zeros = a[i] == 0.0;
        if (zeros) return submit_split(a, n, ticket);
    }
    std::unique_lock<std::mutex> lk(mu);
    uint64_t id = 0;
    if (admit(a, n, comps, 0, 0, &id) != SPB_OK) {
        ++st.rejected;
        spb_set_error("spb_server_submit: admission refused (%zu of %zu pool bytes in use)",
                      pool.used() * kUnit, (pool_units - zero_units) * kUnit);
        return SPB_ERR_BUSY;
    }
    ++st.submitted;
    enqueue(id, reqs[id]);
    *ticket = id;
    return SPB_OK;
}

// A real matrix with zeros: pruned and decomposed on the host, its pieces
// admitted as children of one parent request (all or none).
int Server::submit_split(const double* a, int n, uint64_t* ticket)
{
    int comps = 0, count = 0;
    int st0 = spb_plan_pieces(a, n, &comps, &count, nullptr, nullptr, nullptr, 0, 0);
    if (st0 != SPB_OK) return st0;
    std::vector<int> sizes(count > 0 ? count : 1), owner(count > 0 ? count : 1);
    const size_t total = (size_t)(count > 0 ? count : 1) * n * n;  // pieces are at most n x n
    std::vector<double> data(total);
    if (count > 0 &&
        (st0 = spb_plan_pieces(a, n, &comps, &count, sizes.data(), owner.data(), data.data(), count, total)) != SPB_OK)
        return st0;
    for (int k = 0; k < count; ++k)
        if (sizes[k] > 63) {
            spb_set_error("spb_server_submit: a decomposed piece has n=%d > 63", sizes[k]);
            return SPB_ERR_INVALID;
        }
    std::unique_lock<std::mutex> lk(mu);
    const uint64_t pid = next_id++;
    Request& p = reqs[pid];
    p.n = n;
    p.comps = 1;
    p.t_submit = wall_seconds();
    p.comp_sum.assign(comps, dd{0.0, 0.0});
    size_t off = 0;
    for (int k = 0; k < count; ++k) {
        uint64_t cid = 0;
        if (admit(data.data() + off, sizes[k], 1, pid, owner[k], &cid) != SPB_OK) {
            for (uint64_t c : reqs[pid].children) {
                Request& cr = reqs[c];
                pool.give(cr.off, cr.units);
                reqs.erase(c);
            }
            reqs.erase(pid);
            ++st.rejected;
            spb_set_error("spb_server_submit: admission refused for a decomposed matrix (%zu of %zu pool bytes "
                          "in use)", pool.used() * kUnit, (pool_units - zero_units) * kUnit);
            return SPB_ERR_BUSY;
        }
        reqs[pid].children.push_back(cid);
        off += (size_t)sizes[k] * sizes[k];
    }
    Request& parent = reqs[pid];
    parent.pending = count;
    ++st.submitted;
    ++st.split_requests;
    st.pieces += count;
    if (count == 0) {
        finish(pid, parent, SPB_OK);  // structurally zero: product of an empty sum
        cv_done.notify_all();
    } else {
        for (uint64_t c : parent.children) enqueue(c, reqs[c]);
    }
    *ticket = pid;
    return SPB_OK;
}

void Server::finish(uint64_t id, Request& r, int status)
{
    r.done = true;
    r.in_flight = false;
    r.status = r.cancelled ? SPB_ERR_CANCELLED : status;
    r.t_done = wall_seconds();
    if (r.units) pool.give(r.off, r.units);
    r.units = 0;
    if (r.parent) {
        // a piece: fold its result into its parent, complete the parent with the last one
        const uint64_t pid = r.parent;
        const int comp = r.component;
        const dd v = {r.res[0], r.res[1]};
        const int rs = r.status;
        reqs.erase(id);
        auto it = reqs.find(pid);
        if (it == reqs.end()) return;
        Request& p = it->second;
        if (rs != SPB_OK && p.child_status == SPB_OK) p.child_status = rs;
        p.comp_sum[comp] = dd_add(p.comp_sum[comp], v);
        if (--p.pending == 0) {
            dd prod = {1.0, 0.0};
            for (const dd& s : p.comp_sum) prod = dd_mul_host(prod, s);
            const double hi = add_rn(prod.hi, prod.lo);
            p.res[0] = hi;
            p.res[1] = sub_rn(prod.lo, sub_rn(hi, prod.hi));
            finish(pid, p, p.child_status);
        }
        return;
    }
    if (r.status == SPB_ERR_CANCELLED) ++st.cancelled;
    else ++st.completed;
}

int Server::poll(uint64_t id, spb_request_result* out, bool erase)
{
    std::lock_guard<std::mutex> lk(mu);
    auto it = reqs.find(id);
    if (it == reqs.end() || it->second.parent) {
        spb_set_error("spb_server_poll: unknown ticket %llu", (unsigned long long)id);
        return SPB_ERR_INVALID;
    }
    Request& r = it->second;
    if (!r.done) return SPB_ERR_BUSY;
    if (out) {
        out->re = r.res[0];
        out->re_lo = r.res[1];
        out->im = r.res[2];
        out->im_lo = r.res[3];
        out->submit_s = r.t_submit;
        out->done_s = r.t_done;
        out->n = r.n;
        out->is_complex = r.comps == 2;
        out->status = r.status;
    }
    if (erase) reqs.erase(it);
    return SPB_OK;
}

int Server::wait(uint64_t id, double timeout_s, spb_request_result* out)
{
    {
        std::unique_lock<std::mutex> lk(mu);
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
        const bool ok = cv_done.wait_until(lk, deadline, [&] {
            auto it = reqs.find(id);
            return it == reqs.end() || it->second.done;
        });
        if (!ok) return SPB_ERR_TIMEOUT;
    }
    return poll(id, out, true);
}

int Server::cancel(uint64_t id)
{
    std::lock_guard<std::mutex> lk(mu);
    auto it = reqs.find(id);
    if (it == reqs.end() || it->second.parent) return SPB_ERR_INVALID;
    std::vector<uint64_t> ids = it->second.children;
    if (ids.empty()) ids.push_back(id);
    if (!it->second.children.empty()) it->second.cancelled = !it->second.done;
    for (uint64_t k : ids) {
        auto jt = reqs.find(k);
        if (jt == reqs.end()) continue;
        Request& r = jt->second;
        if (r.done) continue;
        r.cancelled = true;
        if (!r.in_flight) {
            // queued: in its shape queue, or in the large queue (large, or a
            // mid-size request handed over)
            if (r.n <= cfg.batch_max_n) {
                auto& q = small_q[r.comps - 1][r.n];
                q.erase(std::remove(q.begin(), q.end(), k), q.end());
            }
            large_q.erase(std::remove(large_q.begin(), large_q.end(), k), large_q.end());
            finish(k, r, SPB_ERR_CANCELLED);
        }
    }
    cv_done.notify_all();
    return SPB_OK;
}

void Server::stats(spb_server_stats* out)
{
    std::lock_guard<std::mutex> lk(mu);
    *out = st;
    out->queued_bytes = pool.used() * kUnit;
    out->pool_bytes = (pool_units - zero_units) * kUnit;
}

}  // namespace serve
}  // namespace spb

namespace spb {
namespace serve {

bool Server::harvest()
{
    bool any = false;
    for (auto& s : slots) {
        if (!s.busy) continue;
        const cudaError_t q = cudaEventQuery(s.ev);
        if (q == cudaErrorNotReady) continue;
        const int status = q == cudaSuccess ? SPB_OK : SPB_ERR_CUDA;
        if (q != cudaSuccess) spb_set_error("batched launch failed: %s", cudaGetErrorString(q));
        const int C = s.comps;
        std::lock_guard<std::mutex> lk(mu);
        for (int k = 0; k < s.count; ++k) {
            auto it = reqs.find(s.ids[k]);
            if (it == reqs.end()) continue;
            Request& r = it->second;
            for (int c = 0; c < C; ++c) {
                r.res[2 * c] = s.h_out[(size_t)k * 2 * C + 2 * c];
                r.res[2 * c + 1] = s.h_out[(size_t)k * 2 * C + 2 * c + 1];
            }
            finish(s.ids[k], r, status);
        }
        s.busy = false;
        s.ids.clear();
        any = true;
        cv_done.notify_all();
    }
    return any;
}

int Server::launch_slot(int si, int n, int comps, std::vector<uint64_t>& ids)
{
    Slot& s = slots[si];
    const int count = (int)ids.size();
    int bucket = 1;
    while (bucket < count) bucket <<= 1;
    if (bucket > cfg.max_batch) bucket = cfg.max_batch;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (int k = 0; k < count; ++k) s.h_offs[k] = (unsigned)reqs.at(ids[k]).off;
    }
    for (int k = count; k < bucket; ++k) s.h_offs[k] = (unsigned)zero_off;
    SPB_CUDA_TRY(cudaSetDevice(device));
    const bool graphs_on = cfg.use_graphs >= 0;
    auto enqueue_chain = [&]() -> int {
        SPB_CUDA_TRY(cudaMemcpyAsync(s.d_offs, s.h_offs, sizeof(unsigned) * bucket, cudaMemcpyHostToDevice,
                                     small_stream));
        const int r = batch::launch_gathered(h_pool_dev, d_pool, s.d_offs, n, comps == 2, bucket, s.d_out,
                                             small_stream);
        if (r != SPB_OK) return r;
        SPB_CUDA_TRY(cudaMemcpyAsync(s.h_out, s.d_out, (size_t)bucket * 2 * comps * sizeof(double),
                                     cudaMemcpyDeviceToHost, small_stream));
        return SPB_OK;
    };
    const GraphKey key{n, comps, bucket, si};
    auto it = graphs_on ? graphs.find(key) : graphs.end();
    const bool replay = graphs_on && (it != graphs.end() || ++key_uses[key] >= kGraphAfterUses);
    if (replay) {
        if (it == graphs.end()) {
            // The key's earlier plain launches set the kernel's attributes
            // outside any capture; capture the copy-walk-copy chain.
            cudaGraph_t g = nullptr;
            SPB_CUDA_TRY(cudaStreamBeginCapture(small_stream, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_chain();
            cudaError_t ce = cudaStreamEndCapture(small_stream, &g);
            if (rc != SPB_OK) return rc;
            SPB_CUDA_TRY(ce);
            cudaGraphExec_t ge = nullptr;
            ce = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            SPB_CUDA_TRY(ce);
            it = graphs.emplace(key, ge).first;
            std::lock_guard<std::mutex> lk(mu);
            ++st.graphs_captured;
        }
        SPB_CUDA_TRY(cudaGraphLaunch(it->second, small_stream));
        std::lock_guard<std::mutex> lk(mu);
        ++st.graph_launches;
    } else {
        const int rc = enqueue_chain();
        if (rc != SPB_OK) return rc;
    }
    SPB_CUDA_TRY(cudaEventRecord(s.ev, small_stream));
    s.busy = true;
    s.n = n;
    s.comps = comps;
    s.count = count;
    s.ids.swap(ids);
    return SPB_OK;
}

// Starts one batch if a slot is free and a shape is due: its queue holds a
// full batch, its oldest request waited max_wait_s, or (force) the batch side
// of the GPU is idle, in which case waiting would only add latency.  A
// mid-size shape with fewer than mid_batch_min(n) queued requests goes to the
// whole-GPU workers once its oldest request has waited max_wait_s.
bool Server::launch_ready(bool force)
{
    int si = -1;
    for (int i = 0; i < (int)slots.size(); ++i)
        if (!slots[i].busy) { si = i; break; }
    std::vector<uint64_t> ids;
    int n = 0, comps = 1;
    {
        std::lock_guard<std::mutex> lk(mu);
        const double now = wall_seconds();
        bool moved = false;
        for (int c = 0; c < 2; ++c)
            for (int k = kSmallN + 1; k <= cfg.batch_max_n; ++k) {
                auto& q = small_q[c][k];
                if (q.empty() || q.size() >= mid_batch_min(k)) continue;
                if (now - reqs.at(q.front()).t_submit < cfg.max_wait_s) continue;
                st.mid_to_large += q.size();
                for (uint64_t id : q) large_q.push_back(id);
                q.clear();
                moved = true;
            }
        if (moved) cv_large.notify_all();
        if (si < 0) return moved;
        double oldest = 1e300;
        int bc = -1, bn = -1;
        for (int c = 0; c < 2; ++c)
            for (int k = 1; k <= cfg.batch_max_n; ++k) {
                auto& q = small_q[c][k];
                if (q.empty()) continue;
                if (k > kSmallN && q.size() < mid_batch_min(k)) continue;
                const double t = reqs.at(q.front()).t_submit;
                if ((int)q.size() >= cfg.max_batch) { oldest = -1; bc = c; bn = k; }
                else if (t < oldest) { oldest = t; bc = c; bn = k; }
            }
        if (bc < 0) return moved;
        auto& q = small_q[bc][bn];
        const bool due = force || (int)q.size() >= cfg.max_batch || now - oldest >= cfg.max_wait_s;
        if (!due) return moved;
        while (!q.empty() && (int)ids.size() < cfg.max_batch) {
            const uint64_t id = q.front();
            q.pop_front();
            reqs.at(id).in_flight = true;
            ids.push_back(id);
        }
        n = bn;
        comps = bc + 1;
        ++st.batches;
        st.batched_requests += ids.size();
    }
    std::vector<uint64_t> keep = ids;
    const int status = launch_slot(si, n, comps, ids);
    if (status != SPB_OK) {
        std::lock_guard<std::mutex> lk(mu);
        for (uint64_t id : keep) {
            auto it = reqs.find(id);
            if (it != reqs.end()) finish(id, it->second, status);
        }
        cv_done.notify_all();
    }
    return true;
}

void Server::batch_loop()
{
    cudaSetDevice(device);
    for (;;) {
        bool progressed = harvest();
        bool busy = false;
        for (auto& s : slots) busy |= s.busy;
        bool stop;
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = stopping;
        }
        if (stop) {
            if (busy) {
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                continue;
            }
            // cancel what never started
            std::lock_guard<std::mutex> lk(mu);
            for (auto& byn : small_q)
                for (auto& q : byn) {
                    for (uint64_t id : q) {
                        auto it = reqs.find(id);
                        if (it == reqs.end()) continue;
                        it->second.cancelled = true;
                        finish(id, it->second, SPB_ERR_CANCELLED);
                    }
                    q.clear();
                }
            cv_done.notify_all();
            return;
        }
        progressed |= launch_ready(!busy);
        if (progressed) continue;
        if (busy) {
            std::this_thread::sleep_for(std::chrono::microseconds(10));
        } else {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait_for(lk, std::chrono::duration<double>(cfg.max_wait_s));
        }
    }
}

void Server::large_loop(DeviceContext* ctx)
{
    cudaSetDevice(device);
    for (;;) {
        uint64_t id;
        const double* h_a;
        double* d_a;
        int n, comps;
        bool zeros;
        size_t bytes;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_large.wait(lk, [&] { return stopping || !large_q.empty(); });
            if (stopping) {
                for (uint64_t q : large_q) {
                    auto it = reqs.find(q);
                    if (it == reqs.end()) continue;
                    it->second.cancelled = true;
                    finish(q, it->second, SPB_ERR_CANCELLED);
                }
                large_q.clear();
                cv_done.notify_all();
                return;
            }
            id = large_q.front();
            large_q.pop_front();
            auto it = reqs.find(id);
            if (it == reqs.end() || it->second.done) continue;
            Request& r = it->second;
            r.in_flight = true;
            h_a = h_pool + r.off * batch::kOffsetUnit;
            d_a = d_pool + r.off * batch::kOffsetUnit;
            n = r.n;
            comps = r.comps;
            zeros = r.zeros;
            bytes = sizeof(double) * (size_t)n * n * comps;
        }
        spb_options o;
        spb_default_options(&o);
        o.device = device;
        o.precision = cfg.precision;
        spb_result res;
        std::memset(&res, 0, sizeof(res));
        int status;
        if (comps == 1 && zeros) {
            // the host entry's planner may pick the row-compacted walk
            status = dense::run_real_host(h_a, n, &o, &res, ctx);
        } else {
            status = SPB_OK;
            if (cudaMemcpyAsync(d_a, h_a, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
                spb_set_error("serving: copy of a request into the device pool failed");
                status = SPB_ERR_CUDA;
            }
            if (status == SPB_OK) status = dense::run(d_a, true, n, comps, &o, &res, nullptr, ctx);
        }
        std::lock_guard<std::mutex> lk(mu);
        auto it = reqs.find(id);
        if (it != reqs.end()) {
            Request& r = it->second;
            r.res[0] = res.value;
            r.res[1] = res.value_lo;
            r.res[2] = res.imag;
            r.res[3] = res.imag_lo;
            finish(id, r, status);
        }
        ++st.large_launches;
        cv_done.notify_all();
    }
}

}  // namespace serve
}  // namespace spb

using spb::serve::Server;

extern "C" void spb_server_default_config(spb_server_config* cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->batch_max_n = spb::serve::kMaxN;
    cfg->max_batch = 2048;
    cfg->slots = 4;
    cfg->max_wait_s = 200e-6;
    cfg->admit_bytes = (size_t)256 << 20;
    cfg->precision = SPB_PREC_DD;
    cfg->large_workers = 2;
}

extern "C" int spb_server_create(const spb_server_config* cfg, void** server)
{
    if (!server) return SPB_ERR_INVALID;
    *server = nullptr;
    spb_server_config c;
    spb_server_default_config(&c);
    if (cfg) c = *cfg;
    auto* s = new Server(c);
    const int st = s->start();
    if (st != SPB_OK) {
        delete s;
        return st;
    }
    *server = s;
    return SPB_OK;
}

extern "C" int spb_server_submit(void* server, const double* a, int n, int is_complex, uint64_t* ticket)
{
    if (!server) return SPB_ERR_INVALID;
    return static_cast<Server*>(server)->submit(a, n, is_complex ? 2 : 1, ticket);
}

extern "C" int spb_server_submit_many(void* server, const double* mats, const int* ns, const int* is_complex,
                                      int count, uint64_t* tickets, int* admitted)
{
    if (!server || !mats || !ns || !tickets || count < 0) return SPB_ERR_INVALID;
    auto* s = static_cast<Server*>(server);
    size_t off = 0;
    int ok = 0;
    for (int k = 0; k < count; ++k) {
        const int c = (is_complex && is_complex[k]) ? 2 : 1;
        tickets[k] = 0;
        const int st = s->submit(mats + off, ns[k], c, &tickets[k]);
        if (st == SPB_OK) ++ok;
        else if (st != SPB_ERR_BUSY) {
            if (admitted) *admitted = ok;
            return st;
        }
        off += (size_t)ns[k] * ns[k] * c;
    }
    if (admitted) *admitted = ok;
    return SPB_OK;
}

extern "C" int spb_server_poll(void* server, uint64_t ticket, spb_request_result* out)
{
    if (!server) return SPB_ERR_INVALID;
    return static_cast<Server*>(server)->poll(ticket, out, true);
}

extern "C" int spb_server_wait(void* server, uint64_t ticket, double timeout_s, spb_request_result* out)
{
    if (!server) return SPB_ERR_INVALID;
    return static_cast<Server*>(server)->wait(ticket, timeout_s, out);
}

extern "C" int spb_server_cancel(void* server, uint64_t ticket)
{
    if (!server) return SPB_ERR_INVALID;
    return static_cast<Server*>(server)->cancel(ticket);
}

extern "C" int spb_server_get_stats(void* server, spb_server_stats* out)
{
    if (!server || !out) return SPB_ERR_INVALID;
    static_cast<Server*>(server)->stats(out);
    return SPB_OK;
}

extern "C" int spb_server_destroy(void* server)
{
    if (!server) return SPB_ERR_INVALID;
    delete static_cast<Server*>(server);
    return SPB_OK;
}

extern "C" double spb_now(void) { return spb::wall_seconds(); }
