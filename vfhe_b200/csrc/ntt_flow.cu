// Two-pass FP64 transforms as one dataflow launch.
//
// A transform of P = 2^(K + K1) points splits into a radix-2^K1 column pass (index bits
// K .. logP-1; every residue crosses HBM with only K1 butterfly stages, so the pass is
// HBM-bound) and a pass of 2^K-point tiles (the other K stages; FP64-bound).  Launched
// one after the other, each kernel leaves the other's resource idle.  Here one
// persistent launch carries both passes: its CTAs take work items by ticket, and the
// ticket order puts the first pass's items of row r + lag just before the second pass's
// items of row r, so on every SM column work and tile work run side by side.
//
// Items are one CTA of work (TileThreads<K> threads): NT adjacent columns of one row,
// or NT / 2^(K-4) tiles of one row.  A second-pass item waits, with a bounded spin, for
// the count of its row's finished first-pass items (release: barrier, fence, atomic
// add; acquire: ld.acquire by thread 0, then a barrier).  Tickets are taken only by
// running CTAs, and every item waits only on items with smaller tickets, so the launch
// makes progress whatever the number of resident CTAs.  A spin that runs out raises
// vc_flow_fault (vfhe_cuda_device_faults) and the launch's abort word, and the item goes
// ahead; every later wait of the launch sees the abort word and returns at once, so a
// launch that went wrong ends after one spin limit (well under a second to a few
// seconds), not one per item.
//
// The per-row counters live in a per-stream device buffer, zeroed by a memset in front
// of each launch.  The dataflow path is not taken for work-list row tables, while a
// stream is being captured, or where the caller allows no allocation and the buffer is
// too small: the column and tile kernels run instead, with identical results.
#include <cuda_runtime.h>

#include <mutex>
#include <unordered_map>

#include "ntt_f64_dev.cuh"

namespace vc {

__device__ int vc_flow_fault;  // nonzero: a dataflow wait gave up

namespace {

constexpr long long kFlowSpins = 1LL << 21;  // at least 2^21 x 64 ns = 0.13 s; items take microseconds

struct FlowPlan {
    long long rows;
    long long lag;      // rows of first-pass tickets issued ahead of the second pass
    long long tickets;  // rows * (np + nc)
    int np;             // first-pass tickets per row
    int nc;             // second-pass tickets per row
    unsigned long long* ticket;
    int* abort;  // set when a wait gave up: the launch's later waits return at once
    int* done;   // per row: finished first-pass tickets
};

// Ticket i -> (pass, row, ticket within the row's tickets of that pass).  Order: the first
// pass of rows [0, lag), then for r = 0, 1, ...: the first pass of row r + lag (while
// such a row exists) followed by the second pass of row r.
__device__ __forceinline__ void flow_item(const FlowPlan& p, long long i, bool& first, long long& row, int& k) {
    const long long head = p.lag * p.np;
    if (i < head) {
        first = true;
        row = i / p.np;
        k = (int)(i - row * p.np);
        return;
    }
    long long j = i - head;
    const long long full = p.rows - p.lag;  // rows r whose block also carries row r + lag
    const long long blk = p.np + p.nc;
    if (j < full * blk) {
        const long long r = j / blk;
        const int kk = (int)(j - r * blk);
        first = kk < p.np;
        row = first ? r + p.lag : r;
        k = first ? kk : kk - p.np;
        return;
    }
    j -= full * blk;
    first = false;
    row = full + j / p.nc;
    k = (int)(j - (row - full) * p.nc);
}

__device__ __forceinline__ void flow_wait(const int* ctr, int need, int* abort) {
    for (long long spin = 0;; ++spin) {
        int v;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
        if (v >= need) return;
        if (spin >= kFlowSpins) {
            atomicExch(abort, 1);
            atomicExch(&vc_flow_fault, 1);
            return;
        }
        if ((spin & 255) == 255 && *(volatile int*)abort) return;
        __nanosleep(64);
    }
}

// a: the first pass's rows (forward: column pass over the input; inverse: tiles over the
// input), b: the second pass's rows (in place on the first pass's output).  Each ticket
// is PER consecutive items of one row (a compile-time count: a run-time loop bound made
// the compiler spill); thread 0 requests the CTA's next ticket as the current one
// starts, so the atomic's round trip overlaps the work.
template <int K, int K1, bool INV, int PER>
__global__ void __launch_bounds__(TileThreads<K>::value, TileMinBlocks<K>::value)
    k_flow_f(const __grid_constant__ RowSet a, const __grid_constant__ RowSet b, const PrimeInfo* __restrict__ primes,
             const FlowPlan p) {
    constexpr int NT = TileThreads<K>::value, TPT = 1 << (K - 4), G = NT / TPT;
    constexpr int PADDED = (1 << K) + (1 << (K - 4));
    constexpr bool GROUP = G > 1;  // several tiles per CTA: each meets at its own barrier
    extern __shared__ __align__(128) double fsm[];
    __shared__ long long s_item;
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    double* sm = fsm + lt * PADDED;
    long long nxt = 0;
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(p.ticket, 1ULL);
    __syncthreads();
    for (;;) {
        const long long i = s_item;
        if (i >= p.tickets) break;  // the same value in every thread
        if (threadIdx.x == 0) nxt = (long long)atomicAdd(p.ticket, 1ULL);
        bool first;
        long long row;
        int k;
        flow_item(p, i, first, row, k);
        if (!first) {
            if (threadIdx.x == 0) flow_wait(p.done + row, p.np, p.abort);
            __syncthreads();
        }
#pragma unroll 1
        for (int s = 0; s < PER; ++s) {
            const long long item = (long long)k * PER + s;
            if (first != INV) {
                // column work: the forward transform's first pass, the inverse's second
                const long long gc = (row << K) + item * NT + threadIdx.x;
                col_one<K1, INV>(INV ? b : a, primes, gc, K);
            } else {
                // tile work: the forward transform's second pass (centred doubles in), the
                // inverse's first (centred doubles out)
                const RowSet& rs = INV ? a : b;
                const Tile r = locate<false>(rs, primes, K, (row << K1) + item * G + lt, 1 << K1);
                if (s) tile_sync<K, GROUP>(lt);  // the previous tile's exchanges are over
                if (INV) tile_inv_one<K, false, false, GROUP>(r, rs, sm, t, true, lt);
                else tile_fwd_one<K, true, false, GROUP>(r, rs, sm, t, true, lt);
            }
        }
        __syncthreads();  // the ticket's stores are issued and every thread has read s_item
        if (threadIdx.x == 0) {
            if (first) {
                __threadfence();
                atomicAdd(p.done + row, 1);
            }
            s_item = nxt;
        }
        __syncthreads();
    }
}

thread_local int g_no_alloc_depth = 0;

struct Scratch {
    void* p = nullptr;
    size_t bytes = 0;
};

// The stream's counter buffer, at least `bytes` long; nullptr when it would have to be
// allocated where allocation is not allowed (stream capture, allocation-free callers).
void* flow_scratch(cudaStream_t st, size_t bytes) {
    static std::mutex mu;
    static std::unordered_map<cudaStream_t, Scratch> bufs;
    std::lock_guard<std::mutex> lk(mu);
    Scratch& s = bufs[st];
    if (s.bytes >= bytes) return s.p;
    if (g_no_alloc_depth > 0) return nullptr;
    if (s.p) {
        // an earlier launch on this stream may still read the old buffer
        if (cudaStreamSynchronize(st) != cudaSuccess) return nullptr;
        cudaFree(s.p);
        s.p = nullptr;
        s.bytes = 0;
    }
    size_t want = 64 * 1024;
    while (want < bytes) want <<= 1;
    if (cudaMalloc(&s.p, want) != cudaSuccess) {
        cudaGetLastError();
        s.p = nullptr;
        return nullptr;
    }
    s.bytes = want;
    return s.p;
}

template <typename Kern>
int resident_blocks(Kern kern, int threads, size_t smem) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find((const void*)kern);
    if (it != cache.end()) return it->second;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cache[(const void*)kern] = nb;
    return nb;
}

template <int K, int K1>
int flow_launch(const RowSet& a, const RowSet& b, const PrimeInfo* d, bool inverse, int per, cudaStream_t st) {
    constexpr int NT = TileThreads<K>::value, TPT = 1 << (K - 4), G = NT / TPT;
    static_assert(G <= (1 << K1), "a tile item holds tiles of one row");
    if (a.table) return kFlowUnavailable;  // work-list rows run in captured graphs or the persistent kernels
    const long long rows = rowset_rows(a);
    if (rows <= 0) return 0;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        return kFlowUnavailable;
    }
    if (cs != cudaStreamCaptureStatusNone) return kFlowUnavailable;
    const size_t ctr_bytes = 16 + sizeof(int) * (size_t)rows;
    void* buf = flow_scratch(st, ctr_bytes);
    if (!buf) return kFlowUnavailable;
    const size_t smem = sizeof(double) * (size_t)G * ((1 << K) + (1 << (K - 4)));
    const int col_items = (1 << K) / NT, tile_items = (1 << K1) / G;
    // items per ticket: the schedule's choice (0: two) within both passes' item counts
    // (four items per ticket spilled 110-190 bytes per thread under the 80-register cap)
    if (per <= 0 || per > 2) per = 2;
    while (per > 1 && (per > col_items || per > tile_items)) per >>= 1;
    void (*kern)(RowSet, RowSet, const PrimeInfo*, FlowPlan);
    if (per == 2) kern = inverse ? k_flow_f<K, K1, true, 2> : k_flow_f<K, K1, false, 2>;
    else kern = inverse ? k_flow_f<K, K1, true, 1> : k_flow_f<K, K1, false, 1>;
    const int nb = resident_blocks(kern, NT, smem);
    if (nb <= 0) return kFlowUnavailable;
    FlowPlan p;
    p.rows = rows;
    p.np = (inverse ? tile_items : col_items) / per;
    p.nc = (inverse ? col_items : tile_items) / per;
    p.tickets = rows * (p.np + p.nc);
    long long grid = (long long)nb * sm_count();
    if (grid > p.tickets) grid = p.tickets;
    // first-pass work of about two CTA generations ahead of the second pass
    const long long lag = (2 * grid + p.np + p.nc - 1) / (p.np + p.nc) + 1;
    p.lag = lag < rows ? lag : rows;
    p.ticket = reinterpret_cast<unsigned long long*>(buf);
    p.abort = reinterpret_cast<int*>(reinterpret_cast<char*>(buf) + 8);
    p.done = reinterpret_cast<int*>(reinterpret_cast<char*>(buf) + 16);
    int e = (int)cudaMemsetAsync(buf, 0, ctr_bytes, st);
    if (e) return e;
    kern<<<(unsigned)grid, NT, smem, st>>>(a, b, d, p);
    note_launch();
    return (int)cudaGetLastError();
}

}  // namespace

bool flow_supported(int K, int K1) {
    if (K < 10 || K > 13 || K1 < 2 || K1 > 4) return false;
    const int G = (K >= 12) ? 1 : (K == 11 ? 2 : 4);
    return G <= (1 << K1);
}

int flow_dispatch(int K, int K1, const RowSet& first, const RowSet& second, const PrimeInfo* d, bool inverse,
                  int per, cudaStream_t st) {
    switch (K * 8 + K1) {
        case 10 * 8 + 2: return flow_launch<10, 2>(first, second, d, inverse, per, st);
        case 10 * 8 + 3: return flow_launch<10, 3>(first, second, d, inverse, per, st);
        case 10 * 8 + 4: return flow_launch<10, 4>(first, second, d, inverse, per, st);
        case 11 * 8 + 2: return flow_launch<11, 2>(first, second, d, inverse, per, st);
        case 11 * 8 + 3: return flow_launch<11, 3>(first, second, d, inverse, per, st);
        case 11 * 8 + 4: return flow_launch<11, 4>(first, second, d, inverse, per, st);
        case 12 * 8 + 2: return flow_launch<12, 2>(first, second, d, inverse, per, st);
        case 12 * 8 + 3: return flow_launch<12, 3>(first, second, d, inverse, per, st);
        case 12 * 8 + 4: return flow_launch<12, 4>(first, second, d, inverse, per, st);
        case 13 * 8 + 2: return flow_launch<13, 2>(first, second, d, inverse, per, st);
        case 13 * 8 + 3: return flow_launch<13, 3>(first, second, d, inverse, per, st);
        case 13 * 8 + 4: return flow_launch<13, 4>(first, second, d, inverse, per, st);
        default: return kFlowUnavailable;
    }
}

FlowNoAlloc::FlowNoAlloc() { ++g_no_alloc_depth; }
FlowNoAlloc::~FlowNoAlloc() { --g_no_alloc_depth; }

int read_flow_fault(int* out) { return (int)cudaMemcpyFromSymbol(out, vc_flow_fault, sizeof(int)); }

int clear_flow_fault() {
    const int zero = 0;
    return (int)cudaMemcpyToSymbol(vc_flow_fault, &zero, sizeof(int));
}

}  // namespace vc
