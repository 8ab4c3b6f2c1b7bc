// Continuous-batching request loop for permanents of mixed size and type.
//
//   submit ─► admission (queued bytes <= budget) ─► per-(n, real/complex) queue
//      small (n <= batch_max_n):  batch worker packs up to max_batch requests of
//        one shape into a free slot: host copy into the slot's pinned buffer,
//        then H2D copy -> batch_walk (one warp per matrix) -> D2H copy on the
//        small stream, replayed from one CUDA graph per (shape, padded count,
//        slot) once that key has been used kGraphAfterUses times (a capture
//        costs far more than the plain launches of a rarely used key);
//        completion is detected with an event per slot, so up to
//        `slots` batches are in flight while new requests keep arriving.
//      large: the large worker runs the whole-GPU walk on the library stream,
//        concurrently with the batches.
//   poll / wait ─► result with admission and completion timestamps.
//
// A request's result depends only on its own matrix: the batch kernel gives
// each matrix its own warp, tables and reduction, and padding entries are
// zero matrices whose results are discarded.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "context.h"
#include "spb_common.cuh"

namespace spb {
namespace serve {

constexpr int kBatchMaxN = 24;

struct Request {
    int n = 0, comps = 1;
    std::vector<double> a;
    double t_submit = 0, t_done = 0;
    double res[4] = {0, 0, 0, 0};
    int status = SPB_ERR_BUSY;  // SPB_ERR_BUSY while pending
    bool done = false, cancelled = false, in_flight = false;
    size_t bytes = 0;
};

struct Slot {
    double* d_in = nullptr;
    double* d_out = nullptr;
    double* h_in = nullptr;
    double* h_out = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    int n = 0, comps = 1, count = 0;
    std::vector<uint64_t> ids;
};

// Uses of a (shape, padded count, slot) key before its graph is captured.
constexpr int kGraphAfterUses = 3;

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
    void large_loop();
    bool harvest();                 // completes finished slots; true if any
    bool launch_ready(bool force);  // starts a batch if a slot and a shape are ready
    int launch_slot(int si, int n, int comps, std::vector<uint64_t>& ids);
    void finish(uint64_t id, Request& r, int status);

    spb_server_config cfg;
    int device = 0;
    cudaStream_t small_stream = nullptr;
    std::vector<Slot> slots;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    std::map<GraphKey, int> key_uses;  // plain launches per key not yet captured

    std::mutex mu;
    std::condition_variable cv_work, cv_large, cv_done;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> small_q[2][kBatchMaxN + 1];
    std::deque<uint64_t> large_q;
    uint64_t next_id = 1;
    size_t queued_bytes = 0;
    bool stopping = false;
    std::thread t_batch, t_large;
    spb_server_stats st{};
};

}  // namespace serve
}  // namespace spb

namespace spb {
namespace serve {

int Server::start()
{
    if (cfg.batch_max_n <= 0) cfg.batch_max_n = 20;
    if (cfg.batch_max_n > kBatchMaxN) cfg.batch_max_n = kBatchMaxN;
    if (cfg.max_batch <= 0) cfg.max_batch = 2048;
    if (cfg.slots <= 0) cfg.slots = 4;
    if (cfg.max_wait_s <= 0) cfg.max_wait_s = 200e-6;
    if (cfg.admit_bytes == 0) cfg.admit_bytes = (size_t)256 << 20;
    device = cfg.device;
    int st0 = SPB_OK;
    if (!get_context(device, &st0)) return st0;  // stream, events, arena for large requests
    SPB_CUDA_TRY(cudaSetDevice(device));
    SPB_CUDA_TRY(cudaStreamCreateWithFlags(&small_stream, cudaStreamNonBlocking));
    const int bm = cfg.batch_max_n;
    const size_t in_doubles = (size_t)cfg.max_batch * bm * bm * 2;
    const size_t out_doubles = (size_t)cfg.max_batch * 4;
    slots.resize(cfg.slots);
    for (auto& s : slots) {
        if (injected_failure("serving slot") ||
            cudaMalloc(&s.d_in, in_doubles * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&s.d_out, out_doubles * sizeof(double)) != cudaSuccess ||
            cudaMallocHost(&s.h_in, in_doubles * sizeof(double)) != cudaSuccess ||
            cudaMallocHost(&s.h_out, out_doubles * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            spb_set_error("spb_server_create: could not allocate %d batch slots", cfg.slots);
            return SPB_ERR_OOM;
        }
        SPB_CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
    }
    t_batch = std::thread(&Server::batch_loop, this);
    t_large = std::thread(&Server::large_loop, this);
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
    if (t_large.joinable()) t_large.join();
    cudaSetDevice(device);
    if (small_stream) cudaStreamSynchronize(small_stream);
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto& s : slots) {
        if (s.ev) cudaEventDestroy(s.ev);
        if (s.d_in) cudaFree(s.d_in);
        if (s.d_out) cudaFree(s.d_out);
        if (s.h_in) cudaFreeHost(s.h_in);
        if (s.h_out) cudaFreeHost(s.h_out);
    }
    if (small_stream) cudaStreamDestroy(small_stream);
}

int Server::submit(const double* a, int n, int comps, uint64_t* ticket)
{
    if (!a || !ticket || n < 1 || n > 63) {
        spb_set_error("spb_server_submit: null pointer or n=%d outside 1..63", n);
        return SPB_ERR_INVALID;
    }
    const size_t bytes = sizeof(double) * (size_t)n * n * comps;
    std::unique_lock<std::mutex> lk(mu);
    if (queued_bytes + bytes > cfg.admit_bytes) {
        ++st.rejected;
        spb_set_error("spb_server_submit: admission refused (%zu of %zu queued bytes in use)", queued_bytes,
                      cfg.admit_bytes);
        return SPB_ERR_BUSY;
    }
    const uint64_t id = next_id++;
    Request& r = reqs[id];
    r.n = n;
    r.comps = comps;
    r.a.assign(a, a + (size_t)n * n * comps);
    r.bytes = bytes;
    r.t_submit = wall_seconds();
    queued_bytes += bytes;
    ++st.submitted;
    const bool small = n <= cfg.batch_max_n;
    if (small) small_q[comps - 1][n].push_back(id);
    else large_q.push_back(id);
    lk.unlock();
    (small ? cv_work : cv_large).notify_one();
    *ticket = id;
    return SPB_OK;
}

void Server::finish(uint64_t, Request& r, int status)
{
    r.done = true;
    r.in_flight = false;
    r.status = r.cancelled ? SPB_ERR_CANCELLED : status;
    r.t_done = wall_seconds();
    r.a.clear();
    r.a.shrink_to_fit();
    queued_bytes -= r.bytes;
    if (r.status == SPB_ERR_CANCELLED) ++st.cancelled;
    else ++st.completed;
}

int Server::poll(uint64_t id, spb_request_result* out, bool erase)
{
    std::lock_guard<std::mutex> lk(mu);
    auto it = reqs.find(id);
    if (it == reqs.end()) {
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
    if (it == reqs.end()) return SPB_ERR_INVALID;
    Request& r = it->second;
    if (r.done) return SPB_OK;
    r.cancelled = true;
    if (!r.in_flight) {
        auto& q = r.n <= cfg.batch_max_n ? small_q[r.comps - 1][r.n] : large_q;
        q.erase(std::remove(q.begin(), q.end(), id), q.end());
        finish(id, r, SPB_ERR_CANCELLED);
        cv_done.notify_all();
    }
    return SPB_OK;
}

void Server::stats(spb_server_stats* out)
{
    std::lock_guard<std::mutex> lk(mu);
    *out = st;
    out->queued_bytes = queued_bytes;
}

}  // namespace serve
}  // namespace spb

extern "C" int spb_perm_batch_dev(const double* d_mats, int n, int is_complex, int count, double* d_out,
                                  void* stream);

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
    const size_t per = (size_t)n * n * comps;
    {
        // the requests are marked in flight: their matrices stay put
        std::lock_guard<std::mutex> lk(mu);
        for (int k = 0; k < count; ++k) {
            const Request& r = reqs.at(ids[k]);
            std::memcpy(s.h_in + k * per, r.a.data(), per * sizeof(double));
        }
    }
    if (bucket > count) std::memset(s.h_in + count * per, 0, (bucket - count) * per * sizeof(double));
    SPB_CUDA_TRY(cudaSetDevice(device));
    const bool graphs_on = cfg.use_graphs >= 0;
    auto enqueue = [&]() -> int {
        SPB_CUDA_TRY(cudaMemcpyAsync(s.d_in, s.h_in, bucket * per * sizeof(double), cudaMemcpyHostToDevice,
                                     small_stream));
        int st = spb_perm_batch_dev(s.d_in, n, comps == 2, bucket, s.d_out, small_stream);
        if (st != SPB_OK) return st;
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
            // outside any capture; capture the copy-kernel-copy chain.
            cudaGraph_t g = nullptr;
            SPB_CUDA_TRY(cudaStreamBeginCapture(small_stream, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue();
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
        const int rc = enqueue();
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

}  // namespace serve
}  // namespace spb

namespace spb {
namespace serve {

// Starts one batch if a slot is free and a shape is due: its queue holds a
// full batch, its oldest request waited max_wait_s, or (force) the batch side
// of the GPU is idle, in which case waiting would only add latency.
bool Server::launch_ready(bool force)
{
    int si = -1;
    for (int i = 0; i < (int)slots.size(); ++i)
        if (!slots[i].busy) { si = i; break; }
    if (si < 0) return false;
    std::vector<uint64_t> ids;
    int n = 0, comps = 1;
    {
        std::lock_guard<std::mutex> lk(mu);
        double oldest = 1e300;
        int bc = -1, bn = -1;
        for (int c = 0; c < 2; ++c)
            for (int k = 1; k <= cfg.batch_max_n; ++k) {
                auto& q = small_q[c][k];
                if (q.empty()) continue;
                const double t = reqs.at(q.front()).t_submit;
                if ((int)q.size() >= cfg.max_batch) { oldest = -1; bc = c; bn = k; }
                else if (t < oldest) { oldest = t; bc = c; bn = k; }
            }
        if (bc < 0) return false;
        auto& q = small_q[bc][bn];
        const bool due = force || (int)q.size() >= cfg.max_batch || wall_seconds() - oldest >= cfg.max_wait_s;
        if (!due) return false;
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
        for (uint64_t id : keep) finish(id, reqs.at(id), status);
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
                        reqs.at(id).cancelled = true;
                        finish(id, reqs.at(id), SPB_ERR_CANCELLED);
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

void Server::large_loop()
{
    cudaSetDevice(device);
    for (;;) {
        uint64_t id;
        const double* a;
        int n, comps;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_large.wait(lk, [&] { return stopping || !large_q.empty(); });
            if (stopping) {
                for (uint64_t q : large_q) {
                    reqs.at(q).cancelled = true;
                    finish(q, reqs.at(q), SPB_ERR_CANCELLED);
                }
                large_q.clear();
                cv_done.notify_all();
                return;
            }
            id = large_q.front();
            large_q.pop_front();
            Request& r = reqs.at(id);
            r.in_flight = true;
            a = r.a.data();
            n = r.n;
            comps = r.comps;
        }
        spb_options o;
        spb_default_options(&o);
        o.device = device;
        o.precision = cfg.precision;
        spb_result res;
        const int status = comps == 1 ? spb_perm_dense_f64(a, n, &o, &res) : spb_perm_dense_c128(a, n, &o, &res);
        std::lock_guard<std::mutex> lk(mu);
        Request& r = reqs.at(id);
        r.res[0] = res.value;
        r.res[1] = res.value_lo;
        r.res[2] = res.imag;
        r.res[3] = res.imag_lo;
        finish(id, r, status);
        ++st.large_launches;
        cv_done.notify_all();
    }
}

}  // namespace serve
}  // namespace spb

using spb::serve::Server;

extern "C" int spb_server_create(const spb_server_config* cfg, void** server)
{
    if (!server) return SPB_ERR_INVALID;
    *server = nullptr;
    spb_server_config c;
    std::memset(&c, 0, sizeof(c));
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
