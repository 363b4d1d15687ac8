// Serving loop: continuous batching of CKKS and CGGI requests on one GPU.
//
// Clients submit requests that name device-resident ciphertexts and keys (keys and
// ciphertexts stay in HBM; a request moves no host data).  One worker thread owns
// the GPU side:
//   * arrivals go to a queue per (operation, parameter class);
//   * whenever a stream slot is free, the class whose oldest request has waited
//     longest is batched: up to max_batch requests (CGGI: up to the class's maximum
//     ciphertext count), shrunk until its scratch fits the HBM budget left;
//   * a batch gathers its inputs with device-to-device copies into stream-ordered
//     scratch (the server's own memory pool), runs ONE batched call (vfhe_cuda_ckks_*_batch /
//     vfhe_cuda_cggi_bootstrap_batch semantics), scatters the outputs, frees the
//     scratch on its stream and records an event;
//   * batches on different streams overlap on the device; requests that arrive while
//     batches run are admitted as soon as a slot and budget free up (continuous
//     batching, not a queue drained batch by batch).
// A request's latency is the host steady-clock time from submission to the moment
// the worker sees its batch's completion event.  With max_batch = 1 and one stream the
// same loop is the plain one-call-per-request path.
//
// Results do not depend on batching: every batched kernel computes each ciphertext
// independently and exactly, so a request's output is the same alone or in any mix.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "abi_common.cuh"

namespace vc {
uint64_t ckks_mul_ws_elems(uint64_t N, uint64_t B, uint64_t L);
uint64_t ckks_rot_ws_elems(uint64_t N, uint64_t B, uint64_t L);
int ckks_mul_relin_rescale(IncNtt* t, uint64_t* out, const uint64_t* ct1, const uint64_t* ct2, uint64_t B,
                           const uint32_t* limbs, uint32_t L, uint32_t special, const uint64_t* rlk, uint64_t* ws,
                           cudaStream_t st);
int ckks_rotate(IncNtt* t, uint64_t* out, const uint64_t* ct, uint64_t B, const uint32_t* limbs, uint32_t L,
                uint32_t special, const uint64_t* gens, const uint64_t* const* gks, uint64_t* ws, cudaStream_t st);
uint64_t cggi_ws_elems(uint64_t N, uint64_t B, uint64_t n, uint32_t L0);
int cggi_bootstrap(IncNtt* t, uint64_t* out_a, uint64_t* out_b, const uint64_t* in_a, const uint64_t* in_b,
                   uint64_t B, uint32_t n, const uint32_t* limbs, uint32_t L0, uint32_t special, const uint64_t* bk,
                   const uint64_t* tv, uint64_t torus_base, uint64_t* ws, cudaStream_t st);

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kCkksMul = 0, kCkksRot = 1, kCggi = 2 };

struct CkksClass {
    IncNtt* t;
    uint32_t limbs[kMaxLimbs];
    uint32_t L;
    uint32_t special;
    const uint64_t* rlk;
};

struct CggiClass {
    IncNtt* t;
    uint32_t limbs[4];
    uint32_t L0;
    uint32_t special;
    uint32_t n;
    const uint64_t* bk;
    const uint64_t* tv;
    uint64_t torus_base;
    uint32_t bmax;
    // persistent per-class buffers: the blind rotation is a CUDA graph captured per
    // (buffers, batch size), so its scratch stays put; batch sizes round up to powers
    // of two (zero-padded inputs) to keep the number of graphs small
    uint64_t* ws = nullptr;
    uint64_t* in_a = nullptr;   // [bmax][L0][n]
    uint64_t* in_b = nullptr;   // [bmax][L0]
    uint64_t* out_a = nullptr;  // [bmax][L0][N]
    uint64_t* out_b = nullptr;  // [bmax][L0]
    bool busy = false;
    // torus classes (FP64-FFT programmable bootstrap, then key switch back to n):
    // uint32 LWEs [bmax][n+1] in, extracted [bmax][N+1], [bmax][n+1] out; no padding
    bool torus = false;
    uint32_t N = 0, bs_base_log = 0, bs_levels = 0, ks_base_log = 0, ks_levels = 0;
    const double* bsk_f = nullptr;
    const uint32_t* tv32 = nullptr;
    const uint32_t* ksk = nullptr;
    uint32_t* t_in = nullptr;
    uint32_t* t_mid = nullptr;
    uint32_t* t_out = nullptr;
};

struct Request {
    int64_t id;
    int kind;
    int cls;
    uint64_t* out;
    uint64_t* out_b;
    const uint64_t* in1;
    const uint64_t* in2;
    uint64_t gen;
    const uint64_t* key;
    uint64_t count;
    Clock::time_point t_submit, t_done;
    int status = 0;  // 0 queued/running, 1 done, -1 failed, -2 cancelled
    bool started = false;  // taken into a batch (no longer cancellable)
};

struct Batch {
    int kind;
    int cls;
    std::vector<Request*> reqs;
    int stream;
    cudaEvent_t done = nullptr;
    uint64_t bytes = 0;  // budget held until completion
    Clock::time_point t_start;
    bool stalled = false;  // injected: completion not observed until the deadline
    bool expired = false;  // its requests were failed by the batch deadline
};

// launch() outcome
enum LaunchResult { kLaunched = 0, kLaunchFailed = 1, kOutOfMemory = 2 };

}  // namespace

struct Server {
    uint64_t budget = 0;
    uint64_t used = 0;  // resident + persistent class buffers + in-flight scratch
    int max_batch = 1;
    std::vector<cudaStream_t> streams;
    std::vector<bool> stream_busy;
    std::vector<CkksClass> ckks;
    std::vector<CggiClass> cggi;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> arrivals;
    std::map<std::pair<int, int>, std::deque<Request*>> pending;
    std::vector<Batch*> inflight;
    std::unordered_map<int64_t, Request*> requests;
    int64_t next_id = 0;
    int64_t completed = 0;
    int64_t failed = 0;
    uint64_t batches = 0;
    uint64_t batched_requests = 0;
    bool stop = false;
    bool paused = false;         // admission held (requests stay queued)
    double batch_timeout_ms = 0;  // > 0: fail the requests of a batch not done by then
    // host-side fault injection (tests): the next n batch launches fail, the next n
    // scratch allocations fail, the next n batches' completions go unobserved
    int inject_launch = 0, inject_alloc = 0, inject_stall = 0;
    uint64_t expired_batches = 0, oom_retries = 0, cancelled = 0;
    std::thread worker;
    int device = 0;
    // the server's own stream-ordered pool: batch scratch comes and goes every batch,
    // so freed memory stays in the pool (release threshold = max) instead of being
    // unmapped and mapped again
    cudaMemPool_t pool = nullptr;

    void run();
    int launch(Batch* b);
    void fail_request(Request* r, int status);
    uint64_t batch_bytes(int kind, int cls, const std::vector<Request*>& rs) const;
};

namespace {

uint64_t ckks_ct_elems(const CkksClass& c, uint32_t L) { return 2ULL * L * c.t->pub.N; }

int pow2_at_least(uint64_t x) {
    int b = 0;
    while ((1ULL << b) < x) ++b;
    return b;
}

}  // namespace

uint64_t Server::batch_bytes(int kind, int cls, const std::vector<Request*>& rs) const {
    const uint64_t B = rs.size();
    if (kind == kCggi) return 0;  // persistent class buffers, accounted at registration
    const CkksClass& c = ckks[cls];
    const uint64_t N = c.t->pub.N;
    if (kind == kCkksMul)
        return 8 * (2 * B * ckks_ct_elems(c, c.L) + B * ckks_ct_elems(c, c.L - 1) + ckks_mul_ws_elems(N, B, c.L) +
                    3 * B) + 4096;
    return 8 * (2 * B * ckks_ct_elems(c, c.L) + ckks_rot_ws_elems(N, B, c.L) + 3 * B) + 4096;
}

namespace {

// dst[i] = chunk i (elems u64 at srcs[i]) for i < B; grid-stride over B x elems
__global__ void k_gather(uint64_t* __restrict__ dst, const uint64_t* const* __restrict__ srcs, uint64_t elems,
                         uint64_t B) {
    const uint64_t total = elems * B;
    for (uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * 2; k < total;
         k += (uint64_t)gridDim.x * blockDim.x * 2) {
        const uint64_t i = k / elems, j = k - i * elems;  // elems is even: a pair never crosses chunks
        *reinterpret_cast<ulonglong2*>(dst + k) = *reinterpret_cast<const ulonglong2*>(srcs[i] + j);
    }
}

// chunk i of src to dsts[i]
__global__ void k_scatter(uint64_t* const* __restrict__ dsts, const uint64_t* __restrict__ src, uint64_t elems,
                          uint64_t B) {
    const uint64_t total = elems * B;
    for (uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * 2; k < total;
         k += (uint64_t)gridDim.x * blockDim.x * 2) {
        const uint64_t i = k / elems, j = k - i * elems;
        *reinterpret_cast<ulonglong2*>(dsts[i] + j) = *reinterpret_cast<const ulonglong2*>(src + k);
    }
}

unsigned copy_grid(uint64_t elems) {
    const uint64_t blocks = (elems / 2 + 255) / 256;
    return (unsigned)(blocks < 1 ? 1 : (blocks > 8 * 148 ? 8 * 148 : blocks));
}

}  // namespace

int Server::launch(Batch* b) {
    const char* where = "vfhe_cuda_server";
    cudaStream_t st = streams[b->stream];
    const uint64_t B = b->reqs.size();
    int err = 0;
    if (inject_launch > 0) {  // an injected launch error: nothing is enqueued
        --inject_launch;
        set_error(where, "batch launch failed (injected fault)");
        return kLaunchFailed;
    }
    if (b->kind == kCggi && cggi[b->cls].torus) {
        CggiClass& g = cggi[b->cls];
        const uint64_t n1 = g.n + 1;
        uint64_t total = 0;
        for (Request* r : b->reqs) {
            err = err ? err : cudaMemcpyAsync(g.t_in + total * n1, r->in1, r->count * n1 * 4, cudaMemcpyDeviceToDevice,
                                              st);
            total += r->count;
        }
        if (!err && vfhe_cuda_cggi_fft_bootstrap_batch(g.t_mid, g.t_in, total, g.bsk_f, g.tv32, g.n, g.N,
                                                       g.bs_base_log, g.bs_levels, (uint32_t)g.torus_base, st))
            err = -1;
        if (!err && vfhe_cuda_cggi_fft_keyswitch_batch(g.t_out, g.t_mid, total, g.ksk, g.N, g.n, g.ks_base_log,
                                                       g.ks_levels, st))
            err = -1;
        total = 0;
        for (Request* r : b->reqs) {
            if (!err) err = cudaMemcpyAsync(r->out, g.t_out + total * n1, r->count * n1 * 4, cudaMemcpyDeviceToDevice,
                                            st);
            total += r->count;
        }
        g.busy = true;
    } else if (b->kind == kCggi) {
        CggiClass& g = cggi[b->cls];
        const uint64_t N = g.t->pub.N, L0 = g.L0, n = g.n;
        uint64_t total = 0;
        for (Request* r : b->reqs) {
            err = err ? err : cudaMemcpyAsync(g.in_a + total * L0 * n, r->in1, r->count * L0 * n * 8,
                                              cudaMemcpyDeviceToDevice, st);
            err = err ? err : cudaMemcpyAsync(g.in_b + total * L0, r->in2, r->count * L0 * 8, cudaMemcpyDeviceToDevice,
                                              st);
            total += r->count;
        }
        const uint64_t Bp = 1ULL << pow2_at_least(total);
        if (!err && Bp > total) {
            err = cudaMemsetAsync(g.in_a + total * L0 * n, 0, (Bp - total) * L0 * n * 8, st);
            if (!err) err = cudaMemsetAsync(g.in_b + total * L0, 0, (Bp - total) * L0 * 8, st);
        }
        if (!err && cggi_bootstrap(g.t, g.out_a, g.out_b, g.in_a, g.in_b, Bp, g.n, g.limbs, g.L0, g.special, g.bk, g.tv,
                                   g.torus_base, g.ws, st))
            err = -1;
        total = 0;
        for (Request* r : b->reqs) {
            if (!err) err = cudaMemcpyAsync(r->out, g.out_a + total * L0 * N, r->count * L0 * N * 8,
                                            cudaMemcpyDeviceToDevice, st);
            if (!err) err = cudaMemcpyAsync(r->out_b, g.out_b + total * L0, r->count * L0 * 8,
                                            cudaMemcpyDeviceToDevice, st);
            total += r->count;
        }
        g.busy = true;
    } else {
        const CkksClass& c = ckks[b->cls];
        const uint64_t cte = ckks_ct_elems(c, c.L), octe = ckks_ct_elems(c, c.L - 1);
        void* mem = nullptr;
        if (inject_alloc > 0) {  // an injected scratch-allocation failure
            --inject_alloc;
            return kOutOfMemory;
        }
        err = cudaMallocFromPoolAsync(&mem, b->bytes, pool, st);
        if (err == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return kOutOfMemory;
        }
        if (!err) {
            // [in1 | in2 or out | out (mul) | workspace | pointer tables (3 B)]
            uint64_t* in1 = (uint64_t*)mem;
            uint64_t* in2 = in1 + B * cte;
            uint64_t* out = b->kind == kCkksMul ? in2 + B * cte : in2;
            uint64_t* ws = out + B * (b->kind == kCkksMul ? octe : cte);
            const uint64_t ws_elems = b->kind == kCkksMul ? ckks_mul_ws_elems(c.t->pub.N, B, c.L)
                                                         : ckks_rot_ws_elems(c.t->pub.N, B, c.L);
            uint64_t* tabs = ws + ws_elems;
            std::vector<uint64_t> p1(B), p2(B), po(B);
            for (uint64_t i = 0; i < B; ++i) {
                p1[i] = (uint64_t)b->reqs[i]->in1;
                p2[i] = (uint64_t)b->reqs[i]->in2;
                po[i] = (uint64_t)b->reqs[i]->out;
            }
            err = upload_small(tabs, p1.data(), B, st);
            if (!err && b->kind == kCkksMul) err = upload_small(tabs + B, p2.data(), B, st);
            if (!err) err = upload_small(tabs + 2 * B, po.data(), B, st);
            if (!err) {
                k_gather<<<copy_grid(B * cte), 256, 0, st>>>(in1, (const uint64_t* const*)tabs, cte, B);
                if (b->kind == kCkksMul)
                    k_gather<<<copy_grid(B * cte), 256, 0, st>>>(in2, (const uint64_t* const*)(tabs + B), cte, B);
                note_launch(b->kind == kCkksMul ? 2 : 1);
                err = cudaGetLastError();
            }
            if (b->kind == kCkksMul) {
                if (!err && ckks_mul_relin_rescale(c.t, out, in1, in2, B, c.limbs, c.L, c.special, c.rlk, ws, st))
                    err = -1;
                if (!err) k_scatter<<<copy_grid(B * octe), 256, 0, st>>>((uint64_t* const*)(tabs + 2 * B), out, octe, B);
            } else {
                std::vector<uint64_t> gens(B);
                std::vector<const uint64_t*> keys(B);
                for (uint64_t i = 0; i < B; ++i) {
                    gens[i] = b->reqs[i]->gen;
                    keys[i] = b->reqs[i]->key;
                }
                if (!err && ckks_rotate(c.t, out, in1, B, c.limbs, c.L, c.special, gens.data(), keys.data(), ws, st))
                    err = -1;
                if (!err) k_scatter<<<copy_grid(B * cte), 256, 0, st>>>((uint64_t* const*)(tabs + 2 * B), out, cte, B);
            }
            if (!err) {
                note_launch();
                err = cudaGetLastError();
            }
            const int e2 = cudaFreeAsync(mem, st);
            if (!err) err = e2;
        }
    }
    if (!err) err = cudaEventRecord(b->done, st);
    if (err) {
        if (err != -1) check_cuda(err, where);
        return kLaunchFailed;
    }
    b->t_start = Clock::now();
    if (inject_stall > 0) {
        --inject_stall;
        b->stalled = true;
    }
    return kLaunched;
}

void Server::fail_request(Request* r, int status) {
    r->status = status;
    r->t_done = Clock::now();
    if (status == -2) ++cancelled;
    else ++failed;
}

void Server::run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        while (!arrivals.empty()) {
            Request* r = arrivals.front();
            arrivals.pop_front();
            pending[{r->kind, r->cls}].push_back(r);
        }
        bool progress = false;
        // completions
        for (size_t i = 0; i < inflight.size();) {
            Batch* b = inflight[i];
            const Clock::time_point now = Clock::now();
            // a batch past its deadline: its requests fail now; the batch itself is
            // released only once its work has really finished on the device
            if (batch_timeout_ms > 0 && !b->expired &&
                std::chrono::duration<double, std::milli>(now - b->t_start).count() > batch_timeout_ms) {
                b->expired = true;
                ++expired_batches;
                for (Request* r : b->reqs) fail_request(r, -1);
                set_error("vfhe_cuda_server", "batch deadline exceeded");
                progress = true;
            }
            cudaError_t q = cudaEventQuery(b->done);
            if (b->stalled && !b->expired && q != cudaErrorNotReady) q = cudaErrorNotReady;  // injected
            if (q == cudaErrorNotReady) {
                ++i;
                continue;
            }
            if (!b->expired) {
                for (Request* r : b->reqs) {
                    r->t_done = now;
                    r->status = q == cudaSuccess ? 1 : -1;
                    if (q == cudaSuccess) ++completed;
                    else ++failed;
                }
            }
            if (q != cudaSuccess) check_cuda(q, "vfhe_cuda_server: batch");
            used -= b->bytes;
            stream_busy[b->stream] = false;
            if (b->kind == kCggi) cggi[b->cls].busy = false;
            cudaEventDestroy(b->done);
            delete b;
            inflight[i] = inflight.back();
            inflight.pop_back();
            progress = true;
        }
        if (progress) cv_done.notify_all();
        // admissions: oldest waiting class first
        for (; !paused;) {
            int free_stream = -1;
            for (size_t s = 0; s < streams.size(); ++s)
                if (!stream_busy[s]) {
                    free_stream = (int)s;
                    break;
                }
            if (free_stream < 0) break;
            std::deque<Request*>* best = nullptr;
            std::pair<int, int> best_key{0, 0};
            for (auto& kv : pending) {
                if (kv.second.empty()) continue;
                if (kv.first.first == kCggi && cggi[kv.first.second].busy) continue;
                if (!best || kv.second.front()->t_submit < best->front()->t_submit) {
                    best = &kv.second;
                    best_key = kv.first;
                }
            }
            if (!best) break;
            Batch* b = new Batch();
            b->kind = best_key.first;
            b->cls = best_key.second;
            b->stream = free_stream;
            if (b->kind == kCggi) {
                uint64_t total = 0;
                const uint64_t cap = std::min<uint64_t>(cggi[b->cls].bmax, (uint64_t)max_batch * cggi[b->cls].bmax);
                while (!best->empty() && total + best->front()->count <= cap &&
                       (b->reqs.empty() || max_batch > 1)) {
                    total += best->front()->count;
                    b->reqs.push_back(best->front());
                    best->pop_front();
                }
            } else {
                while (!best->empty() && (int)b->reqs.size() < max_batch) {
                    b->reqs.push_back(best->front());
                    best->pop_front();
                }
                // shrink until the scratch fits the budget left
                while (b->reqs.size() > 1 && used + batch_bytes(b->kind, b->cls, b->reqs) > budget) {
                    best->push_front(b->reqs.back());
                    b->reqs.pop_back();
                }
                b->bytes = batch_bytes(b->kind, b->cls, b->reqs);
                if (used + b->bytes > budget) {
                    for (auto it = b->reqs.rbegin(); it != b->reqs.rend(); ++it) best->push_front(*it);
                    delete b;
                    if (inflight.empty()) {  // can never fit: fail the oldest request
                        Request* r = best->front();
                        best->pop_front();
                        fail_request(r, -1);
                        set_error("vfhe_cuda_server", "request scratch exceeds the HBM budget");
                        cv_done.notify_all();
                    }
                    break;
                }
            }
            if (b->reqs.empty()) {
                delete b;
                break;
            }
            for (Request* r : b->reqs) r->started = true;
            int lr = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess ? launch(b)
                                                                                               : kLaunchFailed;
            if (lr == kOutOfMemory && inflight.empty()) {
                ++oom_retries;  // nothing in flight will free memory: one more attempt now
                lr = launch(b);
            }
            if (lr == kOutOfMemory) {
                // scratch did not fit (or an injected allocation failure): back to the
                // front of the queue, retried when a running batch has freed memory
                ++oom_retries;
                for (auto it = b->reqs.rbegin(); it != b->reqs.rend(); ++it) {
                    (*it)->started = false;
                    best->push_front(*it);
                }
                cudaEventDestroy(b->done);
                delete b;
                if (inflight.empty()) {
                    Request* r = best->front();
                    best->pop_front();
                    fail_request(r, -1);
                    set_error("vfhe_cuda_server", "batch scratch allocation failed");
                    cv_done.notify_all();
                }
                break;
            }
            if (lr != kLaunched) {
                for (Request* r : b->reqs) fail_request(r, -1);
                if (b->done) cudaEventDestroy(b->done);
                delete b;
                cv_done.notify_all();
                continue;
            }
            used += b->bytes;
            stream_busy[free_stream] = true;
            ++batches;
            batched_requests += b->reqs.size();
            inflight.push_back(b);
        }
        bool any_pending = false;
        for (auto& kv : pending) any_pending |= !kv.second.empty();
        if (stop && inflight.empty() && !any_pending && arrivals.empty()) break;
        // nothing left to start: sleep until an arrival, or poll the running batches
        if (inflight.empty() && arrivals.empty())
            cv_work.wait_for(lk, std::chrono::milliseconds(5));
        else if (arrivals.empty()) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
        }
    }
}

}  // namespace vc

using vc::Server;

extern "C" {

void* vfhe_cuda_server_new(uint64_t hbm_budget_bytes, uint32_t nstreams, uint32_t max_batch) {
    if (!vc::ensure_ready()) return nullptr;
    if (nstreams == 0 || nstreams > 64 || max_batch == 0) {
        vc::set_error("vfhe_cuda_server_new", "need 1..64 streams and max_batch >= 1");
        return nullptr;
    }
    Server* s = new Server();
    s->budget = hbm_budget_bytes;
    s->max_batch = (int)max_batch;
    s->device = vc::ctx().device;
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    uint64_t keep = ~0ULL;
    if (!vc::check_cuda(cudaMemPoolCreate(&s->pool, &props), "vfhe_cuda_server_new: pool") ||
        !vc::check_cuda(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep),
                        "vfhe_cuda_server_new: pool")) {
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return nullptr;
    }
    for (uint32_t i = 0; i < nstreams; ++i) {
        cudaStream_t st = nullptr;
        if (!vc::check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "vfhe_cuda_server_new")) {
            for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
            cudaMemPoolDestroy(s->pool);
            delete s;
            return nullptr;
        }
        s->streams.push_back(st);
        s->stream_busy.push_back(false);
    }
    s->worker = std::thread([s] { s->run(); });
    return s;
}

// Stop accepting work, finish everything queued, release the server.
void vfhe_cuda_server_free(void* sv) {
    Server* s = (Server*)sv;
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->paused = false;  // everything queued still runs
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    for (auto& g : s->cggi) {
        cudaFree(g.ws);
        cudaFree(g.in_a);
        cudaFree(g.in_b);
        cudaFree(g.out_a);
        cudaFree(g.out_b);
        cudaFree(g.t_in);
        cudaFree(g.t_mid);
        cudaFree(g.t_out);
    }
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    for (auto& kv : s->requests) delete kv.second;
    delete s;
}

// Bytes of HBM the caller keeps resident for this server's requests (keys and
// ciphertexts); counted against the budget.
int vfhe_cuda_server_note_resident(void* sv, uint64_t bytes) {
    Server* s = (Server*)sv;
    if (!s) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    s->used += bytes;
    return 0;
}

int vfhe_cuda_server_ckks_class(void* sv, void* ntt, const uint32_t* limbs, uint32_t L, uint32_t special,
                                const uint64_t* d_rlk) {
    Server* s = (Server*)sv;
    vc::IncNtt* t = vc::as_ntt(ntt);
    if (!s || !t || !limbs || L < 2 || L + 1 > (uint32_t)vc::kMaxLimbs || special >= t->pub.l) {
        vc::set_error("vfhe_cuda_server_ckks_class", "bad pool, limbs (2 <= L <= 63) or special prime");
        return -1;
    }
    vc::CkksClass c;
    memset(&c, 0, sizeof c);
    c.t = t;
    memcpy(c.limbs, limbs, L * sizeof(uint32_t));
    c.L = L;
    c.special = special;
    c.rlk = d_rlk;
    std::lock_guard<std::mutex> lk(s->mu);
    s->ckks.push_back(c);
    return (int)s->ckks.size() - 1;
}

int vfhe_cuda_server_cggi_class(void* sv, void* ntt, const uint32_t* limbs, uint32_t L0, uint32_t special, uint32_t n,
                                const uint64_t* d_bk, const uint64_t* d_tv, uint64_t torus_base, uint32_t max_count) {
    Server* s = (Server*)sv;
    vc::IncNtt* t = vc::as_ntt(ntt);
    if (!s || !t || !limbs || L0 < 1 || L0 > 2 || n == 0 || max_count == 0 || max_count > 16384) {
        vc::set_error("vfhe_cuda_server_cggi_class", "bad pool, limbs (1 or 2), n or max_count (1..16384)");
        return -1;
    }
    vc::CggiClass g;
    g.t = t;
    memset(g.limbs, 0, sizeof g.limbs);
    memcpy(g.limbs, limbs, L0 * sizeof(uint32_t));
    g.L0 = L0;
    g.special = special;
    g.n = n;
    g.bk = d_bk;
    g.tv = d_tv;
    g.torus_base = torus_base;
    g.bmax = 1u << vc::pow2_at_least(max_count);
    const uint64_t N = t->pub.N;
    const uint64_t ws = 8 * vc::cggi_ws_elems(N, g.bmax, n, L0);
    const uint64_t io = 8 * (uint64_t)g.bmax * L0 * (n + 1 + N + 1);
    void *p0 = nullptr, *p1 = nullptr, *p2 = nullptr, *p3 = nullptr, *p4 = nullptr;
    if (cudaMalloc(&p0, ws) || cudaMalloc(&p1, 8ULL * g.bmax * L0 * n) || cudaMalloc(&p2, 8ULL * g.bmax * L0) ||
        cudaMalloc(&p3, 8ULL * g.bmax * L0 * N) || cudaMalloc(&p4, 8ULL * g.bmax * L0)) {
        cudaFree(p0);
        cudaFree(p1);
        cudaFree(p2);
        cudaFree(p3);
        cudaFree(p4);
        vc::set_error("vfhe_cuda_server_cggi_class", "cudaMalloc of the class buffers failed");
        return -1;
    }
    g.ws = (uint64_t*)p0;
    g.in_a = (uint64_t*)p1;
    g.in_b = (uint64_t*)p2;
    g.out_a = (uint64_t*)p3;
    g.out_b = (uint64_t*)p4;
    std::lock_guard<std::mutex> lk(s->mu);
    s->used += ws + io;
    s->cggi.push_back(g);
    return (int)s->cggi.size() - 1;
}

// Torus CGGI class: programmable bootstraps with the FP64-FFT kernel and the key
// switch back to the input key (vfhe_cuda_cggi_fft_bootstrap_batch, _keyswitch_batch);
// keys stay where the caller put them.  Class ids share the CGGI class list.
int vfhe_cuda_server_torus_class(void* sv, const double* d_bsk_f, const uint32_t* d_tv, const uint32_t* d_ksk,
                                 uint32_t n, uint32_t N, uint32_t bs_base_log, uint32_t bs_levels, uint32_t ks_base_log,
                                 uint32_t ks_levels, uint32_t torus_base, uint32_t max_count) {
    Server* s = (Server*)sv;
    if (!s || !d_bsk_f || !d_tv || !d_ksk || n == 0 || N == 0 || max_count == 0 || max_count > (1u << 20) ||
        torus_base == 0) {
        vc::set_error("vfhe_cuda_server_torus_class", "bad keys, n, N, torus base or max_count (1..2^20)");
        return -1;
    }
    vc::CggiClass g;
    memset(g.limbs, 0, sizeof g.limbs);
    g.t = nullptr;
    g.torus = true;
    g.n = n;
    g.N = N;
    g.bs_base_log = bs_base_log;
    g.bs_levels = bs_levels;
    g.ks_base_log = ks_base_log;
    g.ks_levels = ks_levels;
    g.torus_base = torus_base;
    g.bsk_f = d_bsk_f;
    g.tv32 = d_tv;
    g.ksk = d_ksk;
    g.bmax = max_count;
    const uint64_t io = 4ULL * max_count * (2ULL * (n + 1) + N + 1);
    void *p0 = nullptr, *p1 = nullptr, *p2 = nullptr;
    if (cudaMalloc(&p0, 4ULL * max_count * (n + 1)) || cudaMalloc(&p1, 4ULL * max_count * (N + 1)) ||
        cudaMalloc(&p2, 4ULL * max_count * (n + 1))) {
        cudaFree(p0);
        cudaFree(p1);
        cudaFree(p2);
        vc::set_error("vfhe_cuda_server_torus_class", "cudaMalloc of the class buffers failed");
        return -1;
    }
    g.t_in = (uint32_t*)p0;
    g.t_mid = (uint32_t*)p1;
    g.t_out = (uint32_t*)p2;
    std::lock_guard<std::mutex> lk(s->mu);
    s->used += io;
    s->cggi.push_back(g);
    return (int)s->cggi.size() - 1;
}

namespace {
int64_t submit(Server* s, vc::Request* r) {
    r->t_submit = vc::Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return -1;
        }
        r->id = s->next_id++;
        s->requests[r->id] = r;
        s->arrivals.push_back(r);
    }
    s->cv_work.notify_one();
    return r->id;
}
}  // namespace

// Grow the server's memory pool to `bytes` now (allocate and free once), so batches
// admitted later do not map memory while requests wait.
int vfhe_cuda_server_reserve(void* sv, uint64_t bytes) {
    Server* s = (Server*)sv;
    if (!s) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    void* p = nullptr;
    cudaStream_t st = s->streams[0];
    if (!vc::check_cuda(cudaMallocFromPoolAsync(&p, bytes, s->pool, st), "vfhe_cuda_server_reserve") ||
        !vc::check_cuda(cudaFreeAsync(p, st), "vfhe_cuda_server_reserve") ||
        !vc::check_cuda(cudaStreamSynchronize(st), "vfhe_cuda_server_reserve"))
        return 1;
    return 0;
}

namespace {
bool aligned16(const void* a, const void* b = nullptr, const void* c = nullptr, const void* d = nullptr) {
    return (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)d) & 15) == 0;
}
}  // namespace

// CKKS multiply + relinearise + rescale of two [2][L][N] NTT-domain ciphertexts of class
// `cls` into a [2][L-1][N] coefficient-domain output.  Returns the request id.
int64_t vfhe_cuda_server_submit_ckks_mul(void* sv, int cls, uint64_t* d_out, const uint64_t* d_ct1,
                                         const uint64_t* d_ct2) {
    Server* s = (Server*)sv;
    if (!s || cls < 0 || cls >= (int)s->ckks.size() || !aligned16(d_out, d_ct1, d_ct2)) return -1;
    vc::Request* r = new vc::Request();
    r->kind = vc::kCkksMul;
    r->cls = cls;
    r->out = d_out;
    r->in1 = d_ct1;
    r->in2 = d_ct2;
    return submit(s, r);
}

// CKKS rotation (automorphism by `gen` + key switch with d_gk) of a [2][L][N]
// coefficient-domain ciphertext of class `cls`.
int64_t vfhe_cuda_server_submit_ckks_rotate(void* sv, int cls, uint64_t* d_out, const uint64_t* d_ct, uint64_t gen,
                                            const uint64_t* d_gk) {
    Server* s = (Server*)sv;
    if (!s || cls < 0 || cls >= (int)s->ckks.size() || !aligned16(d_out, d_ct, d_gk)) return -1;
    if ((gen & 1) == 0 || gen >= 2 * s->ckks[cls].t->pub.N) return -1;
    vc::Request* r = new vc::Request();
    r->kind = vc::kCkksRot;
    r->cls = cls;
    r->out = d_out;
    r->in1 = d_ct;
    r->gen = gen;
    r->key = d_gk;
    return submit(s, r);
}

// CGGI16 bootstrap of `count` LWE ciphertexts (d_in_a [count][L0][n], d_in_b
// [count][L0]) into d_out_a [count][L0][N], d_out_b [count][L0].
int64_t vfhe_cuda_server_submit_cggi(void* sv, int cls, uint64_t* d_out_a, uint64_t* d_out_b, const uint64_t* d_in_a,
                                     const uint64_t* d_in_b, uint64_t count) {
    Server* s = (Server*)sv;
    if (!s || cls < 0 || cls >= (int)s->cggi.size() || count == 0 || count > s->cggi[cls].bmax) return -1;
    vc::Request* r = new vc::Request();
    r->kind = vc::kCggi;
    r->cls = cls;
    r->out = d_out_a;
    r->out_b = d_out_b;
    r->in1 = d_in_a;
    r->in2 = d_in_b;
    r->count = count;
    return submit(s, r);
}

// Torus bootstrap of `count` LWEs d_in [count][n+1] (uint32, mask then body) into
// d_out [count][n+1] under the same key, through a torus class.
int64_t vfhe_cuda_server_submit_torus(void* sv, int cls, uint32_t* d_out, const uint32_t* d_in, uint64_t count) {
    Server* s = (Server*)sv;
    if (!s || cls < 0 || cls >= (int)s->cggi.size() || !s->cggi[cls].torus || count == 0 ||
        count > s->cggi[cls].bmax)
        return -1;
    vc::Request* r = new vc::Request();
    r->kind = vc::kCggi;
    r->cls = cls;
    r->out = (uint64_t*)d_out;
    r->in1 = (const uint64_t*)d_in;
    r->count = count;
    return submit(s, r);
}

// Wait for request `id` at most timeout_ms (< 0: no limit).  When it has finished,
// forget it (one successful wait per request) and write its latency (ms).  Returns 0
// when it succeeded, 1 when it failed or the id is unknown, 2 when the time ran out
// (the request is kept: wait again or cancel it), 3 when it was cancelled.
int vfhe_cuda_server_wait_for(void* sv, int64_t id, double timeout_ms, double* latency_ms) {
    Server* s = (Server*)sv;
    if (!s) return 1;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return 1;
    vc::Request* r = it->second;
    auto finished = [r] { return r->status != 0; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, finished);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), finished)) {
        return 2;
    }
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    const int rc = r->status == 1 ? 0 : (r->status == -2 ? 3 : 1);
    s->requests.erase(it);
    delete r;
    return rc;
}

// Block until request `id` finished (no time limit); same results as wait_for.
int vfhe_cuda_server_wait(void* sv, int64_t id, double* latency_ms) {
    return vfhe_cuda_server_wait_for(sv, id, -1.0, latency_ms);
}

// Cancel a request that no batch has taken yet.  Returns 0 when it was cancelled (its
// wait returns 3), 1 when it already runs or finished (it completes normally), -1
// when the id is unknown.
int vfhe_cuda_server_cancel(void* sv, int64_t id) {
    Server* s = (Server*)sv;
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return -1;
    vc::Request* r = it->second;
    if (r->status != 0 || r->started) return 1;
    auto drop = [r](std::deque<vc::Request*>& q) {
        auto pos = std::find(q.begin(), q.end(), r);
        if (pos == q.end()) return false;
        q.erase(pos);
        return true;
    };
    bool found = drop(s->arrivals);
    for (auto& kv : s->pending)
        if (!found) found = drop(kv.second);
    if (!found) return 1;
    s->fail_request(r, -2);
    s->cv_done.notify_all();
    return 0;
}

// Hold (paused = 1) or resume (0) the admission of queued requests into batches;
// running batches finish either way.
int vfhe_cuda_server_pause(void* sv, int paused) {
    Server* s = (Server*)sv;
    if (!s) return 1;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->paused = paused != 0;
    }
    s->cv_work.notify_all();
    return 0;
}

// Batch deadline (ms; 0 = none): the requests of a batch still running after it fail
// with "batch deadline exceeded"; the batch's stream and scratch are released when its
// device work has really finished.
int vfhe_cuda_server_set_batch_timeout(void* sv, double timeout_ms) {
    Server* s = (Server*)sv;
    if (!s || !(timeout_ms >= 0)) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    s->batch_timeout_ms = timeout_ms;
    return 0;
}

// Host-side fault injection, for tests of the failure paths (no GPU fault is made):
//   kind 1: the next `count` batch launches fail before enqueuing anything;
//   kind 2: the next `count` batch scratch allocations fail (the batch is re-queued);
//   kind 3: the next `count` batches' completions go unobserved until the batch
//           deadline (vfhe_cuda_server_set_batch_timeout) fails their requests.
int vfhe_cuda_server_inject_fault(void* sv, int kind, uint32_t count) {
    Server* s = (Server*)sv;
    if (!s || kind < 1 || kind > 3) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    (kind == 1 ? s->inject_launch : kind == 2 ? s->inject_alloc : s->inject_stall) += (int)count;
    return 0;
}

// Failure counters: out[0] batches failed by the deadline, out[1] scratch allocation
// retries, out[2] cancelled requests, out[3] injected faults not yet consumed.
int vfhe_cuda_server_fault_stats(void* sv, uint64_t* out4) {
    Server* s = (Server*)sv;
    if (!s || !out4) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    out4[0] = s->expired_batches;
    out4[1] = s->oom_retries;
    out4[2] = s->cancelled;
    out4[3] = (uint64_t)(s->inject_launch + s->inject_alloc + s->inject_stall);
    return 0;
}

// Counters: out[0] completed, out[1] failed, out[2] batches launched, out[3] requests
// in those batches, out[4] HBM bytes in use (resident + class buffers + in flight).
int vfhe_cuda_server_stats(void* sv, uint64_t* out5) {
    Server* s = (Server*)sv;
    if (!s || !out5) return 1;
    std::lock_guard<std::mutex> lk(s->mu);
    out5[0] = (uint64_t)s->completed;
    out5[1] = (uint64_t)s->failed;
    out5[2] = s->batches;
    out5[3] = s->batched_requests;
    out5[4] = s->used;
    return 0;
}

}  // extern "C"
