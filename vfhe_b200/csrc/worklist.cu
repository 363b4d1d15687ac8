// Work list: many independent jobs of uneven ring degree N and limb count L run as
// one CUDA-graph launch.
//
// Job kinds (each is bit-exact with the one-job-per-call entry points, which follow
// the reference's own calls):
//   chain      out = INTT(NTT(a) (x) NTT(b)), (x) the incomplete product of the
//              ring's split degree (rns_polynomial.c:311-356, polynomial_RNSc_to_RNS
//              and back, rns_polynomial.c:582-614);
//   keyswitch  GHS key switch of a rank-1 sample (a, b) in the coefficient domain
//              with one key-switching key (mlwe.c:557-598): digits = limbs of a
//              lifted to limbs + special prime, NTT, -sum digit x key, INTT, round
//              division by the special prime, + b.
//
// Compilation groups the jobs by transform pool (same N, split and prime tables) and
// writes, per group, device-resident row tables: one descriptor per P-point row to
// transform, per limb row to multiply, per (job, limb) to multiply-accumulate and per
// (job, component) to divide.
//
// A run is three persistent cooperative kernels (when every row has 2^8 <= P <= 2^16
// and the split degree is at most 4) whose CTAs walk six phases over the tables of
// every group -- forward column passes and forward tile passes; products and key
// multiply-accumulates; inverse tile passes, inverse column passes and special-prime
// divisions -- with a bounded grid barrier between the phases inside a kernel, so jobs
// of every N and L share each launch and small jobs fill the gaps of large ones.  Three
// kernels instead of one let each keep the register budget (and so the occupancy) its
// phases need.  The fallback (and mode 1) is a CUDA graph of one launch
// per stage per group, groups as independent branches, transform shapes from the tuned
// schedule of (log2 P, rows) (vfhe_cuda_ntt_set_schedule).
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "abi_common.cuh"
#include "fp64mod.cuh"
#include "keyswitch.cuh"
#include "ntt_f64_dev.cuh"

namespace vc {

namespace {

// product of one limb row: S blocks of P slots
struct ProdDesc {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* out;
    const PrimeInfo* pi;
};

// one (job, extended limb) of a key switch: digits d + j*ne*N, key k + j*2*ne*N,
// outputs oa and oa + ne*N
struct MacDesc {
    const uint64_t* d;
    const uint64_t* k;
    uint64_t* oa;
    const PrimeInfo* pi;
    int nd;
    int ne;
};

// one (job, component) of the special-prime division: acc [nl+1][N] -> out [nl][N] (+ pass)
struct DownDesc {
    const uint64_t* acc;
    uint64_t* out;
    const uint64_t* pass;
    const ModDownConsts* mc;
    int nl;
    int pad;
};

constexpr int kWlThreads = 256;

// Product of slot x (all S blocks) of one limb row.
template <int S>
__device__ __forceinline__ void wl_product_one(const ProdDesc& d, long long x, int logP) {
    const PrimeInfo& pi = *d.pi;
    const uint64_t q = pi.q;
    const long long P = 1LL << logP;
    uint64_t av[S], bv[S], res[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        av[j] = d.a[j * P + x];
        bv[j] = d.b[j * P + x];
    }
    if (S == 1 && pi.fp64) {
        // exact FP64 product of canonical operands (uncentred, below 2^50: |t| <= 3q/4)
        const double fa = f_from_u64(av[0]), fb = f_from_u64(bv[0]);
        d.out[x] = f_to_canonical(f_mulmod(fa, fb, __dmul_rn(fb, pi.qinv), pi.qd), pi.qd, pi.qinv, q);
        return;
    }
    const ulonglong2 w = S > 1 ? reinterpret_cast<const ulonglong2*>(pi.twist)[x] : make_ulonglong2(0, 0);
#pragma unroll
    for (int o = 0; o < S; ++o) {
        uint64_t acc = 0, wrap = 0;
#pragma unroll
        for (int j = 0; j < S; ++j) {
            if (j <= o) acc = add_mod(acc, mul_mod(av[j], bv[o - j], pi), q);
            else wrap = add_mod(wrap, mul_mod(av[j], bv[o - j + S], pi), q);
        }
        if (S > 1) acc = add_mod(acc, shoup(wrap, w.x, w.y, q), q);
        res[o] = acc;
    }
#pragma unroll
    for (int o = 0; o < S; ++o) d.out[o * P + x] = res[o];
}

template <int S>
__global__ void __launch_bounds__(kWlThreads) k_wl_product(const ProdDesc* __restrict__ tab, long long chunks,
                                                           int logP) {
    const long long e = blockIdx.x / chunks;
    const long long chunk = blockIdx.x - e * chunks;
    const long long x = chunk * kWlThreads + threadIdx.x;
    if (x >= (1LL << logP)) return;
    wl_product_one<S>(tab[e], x, logP);
}

// -sum_j D_j (*) K_j for one (job, extended limb).  S <= 4: one thread per slot x
// computes all S blocks (mac_slots); larger S: one thread per (block, slot).  idx below
// wl_mac_work(S, N).
__host__ __device__ __forceinline__ long long wl_mac_work(int S, long long N) { return (S == 2 || S == 4) ? N / S : N; }

template <int S>
__device__ __forceinline__ void wl_mac_one(const MacDesc& d, long long idx, long long N) {
    const long long P = N / S;
    const long long dstr = (long long)d.ne * N;
    if (S == 2 || S == 4) {
        mac_slots<(S == 2 ? 2 : 4)>(d.oa, d.oa + dstr, d.d, dstr, d.k, d.k + dstr, 2 * dstr, d.nd, P, idx, *d.pi);
        return;
    }
    const int o = (int)(idx / P);
    const long long x = idx - o * P;
    mac_slot(d.oa, d.oa + dstr, d.d, dstr, d.k, d.k + dstr, 2 * dstr, d.nd, S, P, x, o, *d.pi);
}

template <int S>
__global__ void __launch_bounds__(kWlThreads) k_wl_mac(const MacDesc* __restrict__ tab, long long chunks,
                                                       long long N) {
    const long long e = blockIdx.x / chunks;
    const long long chunk = blockIdx.x - e * chunks;
    const long long idx = chunk * kWlThreads + threadIdx.x;
    if (idx >= wl_mac_work(S, N)) return;
    wl_mac_one<S>(tab[e], idx, N);
}

// Special-prime division of coefficient x of one (job, component).
__device__ __forceinline__ void wl_down_one(const DownDesc& d, long long x, long long N,
                                            const PrimeInfo* __restrict__ primes) {
    const ModDownConsts& mc = *d.mc;
    if (mc.fp64) {
        // exact FP64 form of the loop below (every intermediate an integer below 2^52)
        uint64_t t = d.acc[(long long)d.nl * N + x] + mc.half_p;
        t -= t >= mc.p ? mc.p : 0;
        const double td = f_from_u64(t);
        for (int i = 0; i < d.nl; ++i) {
            const PrimeInfo& pi = primes[mc.prime[i]];
            const double y = __dadd_rn(__dadd_rn(f_from_u64(d.acc[(long long)i * N + x]), mc.half_sp_d[i]), -td);
            double v = f_mulmod(y, mc.inv_sp_d[i], mc.inv_sp_dq[i], pi.qd);
            if (d.pass) v = __dadd_rn(v, f_from_u64(d.pass[(long long)i * N + x]));
            d.out[(long long)i * N + x] = f_to_canonical(v, pi.qd, pi.qinv, pi.q);
        }
        return;
    }
    const uint64_t t = add_mod(d.acc[(long long)d.nl * N + x], mc.half_p, mc.p);
    for (int i = 0; i < d.nl; ++i) {
        const PrimeInfo& pi = primes[mc.prime[i]];
        uint64_t v = add_mod(d.acc[(long long)i * N + x], mc.half_sp[i], pi.q);
        v = sub_mod(v, reduce64(t, pi), pi.q);
        v = shoup(v, mc.inv_sp[i], mc.inv_sp_sh[i], pi.q);
        if (d.pass) v = add_mod(v, d.pass[(long long)i * N + x], pi.q);
        d.out[(long long)i * N + x] = v;
    }
}

__global__ void __launch_bounds__(kWlThreads) k_wl_moddown(const DownDesc* __restrict__ tab, long long chunks,
                                                           long long N, const PrimeInfo* __restrict__ primes) {
    const long long e = blockIdx.x / chunks;
    const long long chunk = blockIdx.x - e * chunks;
    const long long x = chunk * kWlThreads + threadIdx.x;
    if (x >= N) return;
    wl_down_one(tab[e], x, N, primes);
}

// ---- the persistent work-list kernel

// One group's tables as the persistent kernel reads them (device memory).
struct WlGroupPlan {
    RowSet fwd_first;   // column pass (K < logP) or the only tile pass (K == logP)
    RowSet fwd_second;  // tile pass after the column pass
    RowSet inv_first;   // inverse tile pass
    RowSet inv_second;  // inverse column pass (K < logP)
    const ProdDesc* prod;
    const MacDesc* mac;
    const DownDesc* down;
    const PrimeInfo* info;
    long long nprod, nmac, ndown;
    long long N;
    int logP, K, S, logS;
};

struct WlPlan {
    const WlGroupPlan* groups;
    int ngroups;
    unsigned* barrier;              // [0] arrivals, [1] generation
    unsigned long long* phase_ns;   // [7]: start and the end of every phase (global timer), CTA 0
};

__device__ __forceinline__ void wl_stamp(const WlPlan& plan, int k) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        plan.phase_ns[k] = t;
    }
}

constexpr int kWlPThreads = 256;
constexpr long long kWlBarrierSpins = 1LL << 25;  // ~2 s of 64 ns sleeps

__device__ int vc_wl_fault;  // nonzero: a work-list grid barrier gave up waiting

// Grid-wide barrier of a cooperative launch (every CTA is resident, so every CTA
// arrives).  The wait is bounded: if it runs out, the fault flag is raised and the CTA
// carries on (results are then wrong; vfhe_cuda_device_faults reports it).
__device__ __forceinline__ void wl_grid_barrier(unsigned* bar) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > kWlBarrierSpins) {
                    atomicExch(&vc_wl_fault, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// All tiles of one group's tile pass, TPC = 256 / 2^(K-4) tiles per CTA step.  Threads
// whose tile would lie past the end recompute the last tile without storing, so every
// thread reaches every barrier.
template <int K, bool INV, bool TWO>
__device__ __forceinline__ void wl_tiles(const RowSet& rows, double* fsm) {
    constexpr int TPT = 1 << (K - 4), TPC = kWlPThreads / TPT, PADDED = (1 << K) + (1 << (K - 4));
    const int tiles_per_row = 1 << (rows.logP - K);
    const long long ntiles = rows.table_rows * tiles_per_row;
    const long long ngroups = (ntiles + TPC - 1) / TPC;
    const int lt = threadIdx.x / TPT, t = threadIdx.x - lt * TPT;
    double* sm = fsm + lt * PADDED;
    for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const long long tile = grp * TPC + lt;
        const bool valid = tile < ntiles;
        const Tile r = locate<true>(rows, nullptr, K, valid ? tile : ntiles - 1, tiles_per_row);
        if constexpr (INV) tile_inv_one<K, !TWO, false>(r, rows, sm, t, valid);
        else tile_fwd_one<K, TWO, false>(r, rows, sm, t, valid);
        __syncthreads();  // the next step reuses the exchange buffers
    }
}

template <bool INV, bool TWO>
__device__ __forceinline__ void wl_tiles_k(int K, const RowSet& rows, double* fsm) {
    switch (K) {
        case 8: wl_tiles<8, INV, TWO>(rows, fsm); break;
        case 9: wl_tiles<9, INV, TWO>(rows, fsm); break;
        case 10: wl_tiles<10, INV, TWO>(rows, fsm); break;
        case 11: wl_tiles<11, INV, TWO>(rows, fsm); break;
        default: wl_tiles<12, INV, TWO>(rows, fsm); break;
    }
}

template <bool INV>
__device__ __forceinline__ void wl_cols(int K1, const RowSet& rows, int KT) {
    const long long ncols = rows.table_rows << KT;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long gc = (long long)blockIdx.x * blockDim.x + threadIdx.x; gc < ncols; gc += stride) {
        switch (K1) {
            case 1: col_one<1, INV>(rows, nullptr, gc, KT); break;
            case 2: col_one<2, INV>(rows, nullptr, gc, KT); break;
            case 3: col_one<3, INV>(rows, nullptr, gc, KT); break;
            default: col_one<4, INV>(rows, nullptr, gc, KT); break;
        }
    }
}

template <int S>
__device__ __forceinline__ void wl_products_s(const WlGroupPlan& G) {
    const int logP = G.logP;
    const long long total = G.nprod << logP;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
        wl_product_one<S>(G.prod[i >> logP], i & ((1LL << logP) - 1), logP);
}

template <int S>
__device__ __forceinline__ void wl_macs_s(const WlGroupPlan& G) {
    const long long work = wl_mac_work(S, G.N);
    const int lw = 63 - __clzll(work);
    const long long total = G.nmac << lw;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
        wl_mac_one<S>(G.mac[i >> lw], i & (work - 1), G.N);
}

__device__ __forceinline__ void wl_downs(const WlGroupPlan& G) {
    if (!G.ndown) return;
    const int ln = 63 - __clzll(G.N);
    const long long total = G.ndown << ln;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
        wl_down_one(G.down[i >> ln], i & (G.N - 1), G.N, G.info);
}

// The run as three cooperative kernels, each with the register budget its phases need
// (so the memory-bound phases keep enough warps in flight):
//   PART 0: column passes of two-pass pools + one-pass transforms | grid barrier |
//           tile passes of two-pass pools
//   PART 1: products of the chains and multiply-accumulates of the key switches
//   PART 2: inverse tile passes | barrier | inverse column passes of two-pass pools +
//           divisions of one-pass pools | barrier | divisions of two-pass pools
// Resident CTAs per SM asked of the compiler: three for the transform phases (80
// registers; the forward phase spills 388 bytes per thread, yet two CTAs per SM at 128
// registers without spills measured 5% slower), two for the MACs.
template <int PART>
struct WlPartBlocks {
    static constexpr int value = PART == 1 ? 2 : 3;
};

template <int PART>
__global__ void __launch_bounds__(kWlPThreads, WlPartBlocks<PART>::value) k_wl_persistent(const __grid_constant__ WlPlan plan) {
    extern __shared__ __align__(128) double fsm[];
    if constexpr (PART == 0) {
        wl_stamp(plan, 0);
        // column passes of the two-pass pools, and beside them (they depend on no column
        // pass) the whole transforms of the one-pass pools
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K < G.logP && G.fwd_first.table_rows) wl_cols<false>(G.logP - G.K, G.fwd_first, G.K);
        }
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K == G.logP && G.fwd_first.table_rows) wl_tiles_k<false, false>(G.K, G.fwd_first, fsm);
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 1);
        // tile passes of the two-pass pools (reading the column passes' centred doubles)
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K < G.logP && G.fwd_first.table_rows) wl_tiles_k<false, true>(G.K, G.fwd_second, fsm);
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 2);
    } else if constexpr (PART == 1) {
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.nprod) {
                switch (G.S) {
                    case 1: wl_products_s<1>(G); break;
                    case 2: wl_products_s<2>(G); break;
                    default: wl_products_s<4>(G); break;
                }
            }
            if (G.nmac) {
                switch (G.S) {
                    case 1: wl_macs_s<1>(G); break;
                    case 2: wl_macs_s<2>(G); break;
                    default: wl_macs_s<4>(G); break;
                }
            }
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 3);
    } else {
        // inverse tile passes (before a column pass they leave centred doubles)
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (!G.inv_first.table_rows) continue;
            if (G.K < G.logP) wl_tiles_k<true, true>(G.K, G.inv_first, fsm);
            else wl_tiles_k<true, false>(G.K, G.inv_first, fsm);
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 4);
        // inverse column passes of the two-pass pools, and beside them the divisions of
        // the one-pass pools (whose transforms are complete)
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K < G.logP && G.inv_second.table_rows) wl_cols<true>(G.logP - G.K, G.inv_second, G.K);
        }
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K == G.logP) wl_downs(G);
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 5);
        for (int g = 0; g < plan.ngroups; ++g) {
            const WlGroupPlan& G = plan.groups[g];
            if (G.K < G.logP) wl_downs(G);
        }
        wl_grid_barrier(plan.barrier);
        wl_stamp(plan, 6);
    }
}

constexpr size_t kWlPSmem = sizeof(double) * kWlPThreads * 17;  // TPC tiles of 17 TPT doubles, any K

struct Job {
    int kind;  // 0 chain, 1 keyswitch
    IncNtt* t;
    uint64_t* out;
    const uint64_t* a;
    const uint64_t* b;    // chain: second operand; keyswitch: unused (b is a + L N)
    const uint64_t* ksk;  // keyswitch: [L][2][L+1][N]
    uint32_t limbs[kMaxLimbs];
    int L;
    uint32_t special;
};

struct Group {
    IncNtt* t = nullptr;
    std::vector<RowDesc> fwd, inv;
    std::vector<ProdDesc> prod;
    std::vector<MacDesc> mac;
    std::vector<DownDesc> down;
    // device copies
    RowDesc* d_fwd = nullptr;
    RowDesc* d_inv = nullptr;
    ProdDesc* d_prod = nullptr;
    MacDesc* d_mac = nullptr;
    DownDesc* d_down = nullptr;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct WorkList {
    std::vector<Job> jobs;
    std::vector<Group> groups;
    void* dev = nullptr;  // workspace and tables, one allocation
    size_t dev_bytes = 0;
    cudaGraphExec_t exec = nullptr;
    int launches_per_run = 0;
    int mode = 0;  // 0: one persistent launch when the jobs allow it; 1: graph of per-group launches
    // persistent path
    bool persistent = false;
    WlPlan plan = {};
    int grid[3] = {0, 0, 0};  // CTAs of each part (all resident)

    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        persistent = false;
        plan = WlPlan{};
        if (dev) cudaFree(dev);
        dev = nullptr;
        dev_bytes = 0;
        groups.clear();
    }
};

namespace {

const char* kWhere = "vfhe_cuda_worklist";

bool job_rows_ok(const Job& j) {
    const IncNtt* t = j.t;
    if (!t || j.L <= 0 || j.L + 1 > kMaxLimbs) return false;
    for (int i = 0; i < j.L; ++i)
        if (j.limbs[i] >= t->pub.l || !t->info[j.limbs[i]].fp64) return false;
    if (j.kind == 1 && (j.special >= t->pub.l || !t->info[j.special].fp64)) return false;
    // transforms read 16-byte vectors
    const uintptr_t m = (uintptr_t)j.out | (uintptr_t)j.a | (uintptr_t)j.b | (uintptr_t)j.ksk;
    return (m & 15) == 0 && t->logP >= 8 && t->logP <= 17;
}

int compile(WorkList& w) {
    w.release();
    std::map<IncNtt*, size_t> gidx;
    std::vector<std::vector<const Job*>> members;
    for (const Job& j : w.jobs) {
        auto it = gidx.find(j.t);
        if (it == gidx.end()) {
            it = gidx.emplace(j.t, w.groups.size()).first;
            w.groups.emplace_back();
            w.groups.back().t = j.t;
            members.emplace_back();
        }
        members[it->second].push_back(&j);
    }
    // workspace layout (elements): chain tmp [L][N]; keyswitch D [L][L+1][N] + acc [2][L+1][N]
    std::vector<size_t> ws_off(w.jobs.size());
    size_t ws = 0;
    for (size_t i = 0; i < w.jobs.size(); ++i) {
        const Job& j = w.jobs[i];
        const size_t N = j.t->pub.N;
        ws_off[i] = ws;
        ws += j.kind == 0 ? (size_t)j.L * N : (size_t)j.L * (j.L + 1) * N + 2 * (size_t)(j.L + 1) * N;
    }
    size_t nks = 0;
    for (const Job& j : w.jobs) nks += j.kind == 1;
    // device buffer: workspace | moddown constants | tables (sized after the host pass)
    const size_t ws_bytes = align256(ws * 8);
    const size_t mc_bytes = align256(nks * sizeof(ModDownConsts));
    std::vector<ModDownConsts> consts;
    consts.reserve(nks);
    // the table pass needs the buffer's base address, so first count, then allocate, then fill
    size_t tab_bytes = 0;
    for (size_t g = 0; g < w.groups.size(); ++g) {
        size_t nf = 0, np = 0, nm = 0, nd = 0;
        for (const Job* j : members[g]) {
            const size_t s = j->t->pub.split_degree;
            if (j->kind == 0) {
                nf += 2 * j->L * s;
                np += j->L;
            } else {
                nf += (size_t)j->L * (j->L + 1) * s;
                nm += j->L + 1;
                nd += 2;
            }
        }
        size_t ni = 0;
        for (const Job* j : members[g]) ni += (j->kind == 0 ? j->L : 2 * (j->L + 1)) * j->t->pub.split_degree;
        tab_bytes += align256(nf * sizeof(RowDesc)) + align256(ni * sizeof(RowDesc)) +
                     align256(np * sizeof(ProdDesc)) + align256(nm * sizeof(MacDesc)) + align256(nd * sizeof(DownDesc));
    }
    // persistent path: every row between 2^8 and 2^16 points (tile passes of at most
    // 2^12 points after a column pass of radix at most 16), split degree at most 4
    bool persist = w.mode == 0;
    for (const Group& G : w.groups)
        persist = persist && G.t->logP >= 8 && G.t->logP <= 16 && G.t->pub.split_degree <= 4;
    const size_t plan_bytes = persist ? align256(w.groups.size() * sizeof(WlGroupPlan)) + 256 : 0;
    w.dev_bytes = ws_bytes + mc_bytes + tab_bytes + plan_bytes;
    if (!check_cuda(cudaMalloc(&w.dev, w.dev_bytes), kWhere)) {
        w.dev = nullptr;
        return 1;
    }
    uint64_t* wsp = (uint64_t*)w.dev;
    ModDownConsts* d_consts = (ModDownConsts*)((char*)w.dev + ws_bytes);
    char* tab = (char*)w.dev + ws_bytes + mc_bytes;

    std::map<const Job*, size_t> job_index;
    for (size_t i = 0; i < w.jobs.size(); ++i) job_index[&w.jobs[i]] = i;
    for (size_t g = 0; g < w.groups.size(); ++g) {
        Group& G = w.groups[g];
        IncNtt* t = G.t;
        const long long N = (long long)t->pub.N;
        const int s = (int)t->pub.split_degree;
        const long long P = N / s;
        const PrimeInfo* dinfo = t->d_info;
        auto rows = [&](std::vector<RowDesc>& v, const uint64_t* in, uint64_t* out, uint32_t prime) {
            for (int blk = 0; blk < s; ++blk) v.push_back(RowDesc{in + blk * P, out + blk * P, dinfo + prime, 0});
        };
        for (const Job* j : members[g]) {
            uint64_t* tmp = wsp + ws_off[job_index[j]];
            if (j->kind == 0) {
                for (int l = 0; l < j->L; ++l) {
                    rows(G.fwd, j->a + l * N, j->out + l * N, j->limbs[l]);
                    rows(G.fwd, j->b + l * N, tmp + l * N, j->limbs[l]);
                    G.prod.push_back(ProdDesc{j->out + l * N, tmp + l * N, j->out + l * N, dinfo + j->limbs[l]});
                    rows(G.inv, j->out + l * N, j->out + l * N, j->limbs[l]);
                }
            } else {
                const int nl = j->L, ne = nl + 1;
                uint32_t ext[kMaxLimbs];
                for (int i = 0; i < nl; ++i) ext[i] = j->limbs[i];
                ext[nl] = j->special;
                uint64_t* D = tmp;
                uint64_t* acc = D + (long long)nl * ne * N;
                for (int d = 0; d < nl; ++d)
                    for (int e = 0; e < ne; ++e) rows(G.fwd, j->a + d * N, D + ((long long)d * ne + e) * N, ext[e]);
                for (int e = 0; e < ne; ++e)
                    G.mac.push_back(MacDesc{D + e * N, j->ksk + e * N, acc + e * N, dinfo + ext[e], nl, ne});
                for (int c = 0; c < 2; ++c)
                    for (int e = 0; e < ne; ++e)
                        rows(G.inv, acc + ((long long)c * ne + e) * N, acc + ((long long)c * ne + e) * N, ext[e]);
                const size_t ci = consts.size();
                consts.push_back(moddown_consts(t, j->limbs, nl, j->special));
                G.down.push_back(DownDesc{acc, j->out, nullptr, d_consts + ci, nl, 0});
                G.down.push_back(DownDesc{acc + (long long)ne * N, j->out + (long long)nl * N, j->a + (long long)nl * N,
                                          d_consts + ci, nl, 0});
            }
        }
        auto place = [&](auto& v, auto*& dptr) {
            using T = typename std::decay<decltype(v)>::type::value_type;
            dptr = (T*)tab;
            tab += align256(v.size() * sizeof(T));
        };
        place(G.fwd, G.d_fwd);
        place(G.inv, G.d_inv);
        place(G.prod, G.d_prod);
        place(G.mac, G.d_mac);
        place(G.down, G.d_down);
    }
    // upload constants and tables (once per compile)
    if (nks && !check_cuda(cudaMemcpy(d_consts, consts.data(), nks * sizeof(ModDownConsts), cudaMemcpyHostToDevice),
                           kWhere))
        return 1;
    for (Group& G : w.groups) {
        if ((!G.fwd.empty() && !check_cuda(cudaMemcpy(G.d_fwd, G.fwd.data(), G.fwd.size() * sizeof(RowDesc),
                                                      cudaMemcpyHostToDevice), kWhere)) ||
            (!G.inv.empty() && !check_cuda(cudaMemcpy(G.d_inv, G.inv.data(), G.inv.size() * sizeof(RowDesc),
                                                      cudaMemcpyHostToDevice), kWhere)) ||
            (!G.prod.empty() && !check_cuda(cudaMemcpy(G.d_prod, G.prod.data(), G.prod.size() * sizeof(ProdDesc),
                                                       cudaMemcpyHostToDevice), kWhere)) ||
            (!G.mac.empty() && !check_cuda(cudaMemcpy(G.d_mac, G.mac.data(), G.mac.size() * sizeof(MacDesc),
                                                      cudaMemcpyHostToDevice), kWhere)) ||
            (!G.down.empty() && !check_cuda(cudaMemcpy(G.d_down, G.down.data(), G.down.size() * sizeof(DownDesc),
                                                       cudaMemcpyHostToDevice), kWhere)))
            return 1;
    }
    // a pageable upload on the legacy stream may return before its DMA lands, and the
    // kernels that read it run on non-blocking streams: wait for the legacy stream
    if (!check_cuda(cudaStreamSynchronize(0), kWhere)) return 1;

    if (persist) {
        // the group plans and the barrier words sit at the end of the buffer
        WlGroupPlan* d_plans = (WlGroupPlan*)((char*)w.dev + ws_bytes + mc_bytes + tab_bytes);
        unsigned* d_bar = (unsigned*)((char*)d_plans + plan_bytes - 256);
        std::vector<WlGroupPlan> plans(w.groups.size());
        for (size_t g = 0; g < w.groups.size(); ++g) {
            const Group& Gr = w.groups[g];
            IncNtt* t = Gr.t;
            WlGroupPlan& P = plans[g];
            memset(&P, 0, sizeof P);
            P.logP = t->logP;
            // tile bits: the tuned schedule's for this (P, rows) class when it fits the
            // persistent kernel (tiles of 2^8..2^12 after a column pass of radix <= 16)
            const NttSchedule sc = get_ntt_schedule(t->logP, (long long)std::max(Gr.fwd.size(), Gr.inv.size()));
            int K = t->logP <= 12 ? t->logP : 12;
            if (sc.tile_bits >= 8 && sc.tile_bits <= 12 && sc.tile_bits <= t->logP && t->logP - sc.tile_bits <= 4 &&
                sc.ctas_per_sm != -1)
                K = sc.tile_bits;
            P.K = K;
            P.S = (int)t->pub.split_degree;
            P.logS = 0;
            while ((1 << P.logS) < P.S) ++P.logS;
            P.N = (long long)t->pub.N;
            P.info = t->d_info;
            auto table_set = [&](RowSet& rs, const RowDesc* tab, size_t n, int reduce, int src_is_dst) {
                memset(&rs, 0, sizeof rs);
                rs.logP = t->logP;
                rs.split = P.S;
                rs.fp64 = 1;
                rs.reduce_input = reduce;
                rs.table = tab;
                rs.table_rows = (long long)n;
                rs.table_src_is_dst = src_is_dst;
            };
            table_set(P.fwd_first, Gr.d_fwd, Gr.fwd.size(), 1, 0);
            table_set(P.fwd_second, Gr.d_fwd, Gr.fwd.size(), 0, 1);
            table_set(P.inv_first, Gr.d_inv, Gr.inv.size(), 0, 0);
            table_set(P.inv_second, Gr.d_inv, Gr.inv.size(), 0, 1);
            P.prod = Gr.d_prod;
            P.nprod = (long long)Gr.prod.size();
            P.mac = Gr.d_mac;
            P.nmac = (long long)Gr.mac.size();
            P.down = Gr.d_down;
            P.ndown = (long long)Gr.down.size();
        }
        int nb = 0;
        int err = (int)cudaMemcpy(d_plans, plans.data(), plans.size() * sizeof(WlGroupPlan), cudaMemcpyHostToDevice);
        if (!err) err = (int)cudaMemset(d_bar, 0, 256);
        if (!err) err = (int)cudaStreamSynchronize(0);  // the plans and barrier words are in place
        int nbp[3] = {0, 0, 0};
        if (!err) err = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp[0], k_wl_persistent<0>, kWlPThreads, kWlPSmem);
        if (!err) err = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp[1], k_wl_persistent<1>, kWlPThreads, kWlPSmem);
        if (!err) err = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp[2], k_wl_persistent<2>, kWlPThreads, kWlPSmem);
        nb = std::min(nbp[0], std::min(nbp[1], nbp[2]));
        if (!err && nb >= 1) {
            for (int k = 0; k < 3; ++k) w.grid[k] = nbp[k] * sm_count();
            w.plan.groups = d_plans;
            w.plan.ngroups = (int)plans.size();
            w.plan.barrier = d_bar;
            w.plan.phase_ns = (unsigned long long*)((char*)d_bar + 64);
            w.persistent = true;
            w.launches_per_run = 3;
            return 0;
        }
        cudaGetLastError();  // the per-group graph below serves instead
    }

    // capture: one branch per group, forked from and joined into one capture stream
    const int G = (int)w.groups.size();
    std::vector<cudaStream_t> gs(G, nullptr);
    std::vector<cudaEvent_t> joins(G, nullptr);
    cudaStream_t cs = nullptr;
    cudaEvent_t fork = nullptr;
    int err = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (!err) err = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (int g = 0; g < G && !err; ++g) {
        err = cudaStreamCreateWithFlags(&gs[g], cudaStreamNonBlocking);
        if (!err) err = cudaEventCreateWithFlags(&joins[g], cudaEventDisableTiming);
    }
    if (!err) err = prepare_ntt_kernels();
    const uint64_t counted0 = launch_counter();
    cudaGraph_t graph = nullptr;
    if (!err) err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (!err) {
        int cerr = cudaEventRecord(fork, cs);
        for (int g = 0; g < G && !cerr; ++g) {
            Group& Gr = w.groups[g];
            IncNtt* t = Gr.t;
            cudaStream_t q = gs[g];
            const long long N = (long long)t->pub.N;
            const int s = (int)t->pub.split_degree;
            cerr = cudaStreamWaitEvent(q, fork, 0);
            RowSet rs;
            memset(&rs, 0, sizeof rs);
            rs.logP = t->logP;
            rs.split = s;
            rs.fp64 = 1;
            rs.reduce_input = 1;
            rs.table = Gr.d_fwd;
            rs.table_rows = (long long)Gr.fwd.size();
            if (!cerr && rs.table_rows) cerr = launch_ntt(rs, t->d_info, false, q);
            if (!cerr && !Gr.prod.empty()) {
                const long long P = N / s;
                const long long chunks = (P + kWlThreads - 1) / kWlThreads;
                const unsigned grid = (unsigned)(chunks * (long long)Gr.prod.size());
                switch (s) {
                    case 1: k_wl_product<1><<<grid, kWlThreads, 0, q>>>(Gr.d_prod, chunks, t->logP); break;
                    case 2: k_wl_product<2><<<grid, kWlThreads, 0, q>>>(Gr.d_prod, chunks, t->logP); break;
                    case 4: k_wl_product<4><<<grid, kWlThreads, 0, q>>>(Gr.d_prod, chunks, t->logP); break;
                    case 8: k_wl_product<8><<<grid, kWlThreads, 0, q>>>(Gr.d_prod, chunks, t->logP); break;
                    case 16: k_wl_product<16><<<grid, kWlThreads, 0, q>>>(Gr.d_prod, chunks, t->logP); break;
                    default: cerr = (int)cudaErrorInvalidValue;
                }
                if (!cerr) cerr = (int)cudaGetLastError();
                note_launch();
            }
            if (!cerr && !Gr.mac.empty()) {
                const long long work = (s == 2 || s == 4) ? N / s : N;  // threads per entry
                const long long chunks = (work + kWlThreads - 1) / kWlThreads;
                const unsigned grid = (unsigned)(chunks * (long long)Gr.mac.size());
                switch (s) {
                    case 1: k_wl_mac<1><<<grid, kWlThreads, 0, q>>>(Gr.d_mac, chunks, N); break;
                    case 2: k_wl_mac<2><<<grid, kWlThreads, 0, q>>>(Gr.d_mac, chunks, N); break;
                    case 4: k_wl_mac<4><<<grid, kWlThreads, 0, q>>>(Gr.d_mac, chunks, N); break;
                    case 8: k_wl_mac<8><<<grid, kWlThreads, 0, q>>>(Gr.d_mac, chunks, N); break;
                    default: k_wl_mac<16><<<grid, kWlThreads, 0, q>>>(Gr.d_mac, chunks, N); break;
                }
                cerr = (int)cudaGetLastError();
                note_launch();
            }
            RowSet ri = rs;
            ri.reduce_input = 0;
            ri.table = Gr.d_inv;
            ri.table_rows = (long long)Gr.inv.size();
            if (!cerr && ri.table_rows) cerr = launch_ntt(ri, t->d_info, true, q);
            if (!cerr && !Gr.down.empty()) {
                const long long chunks = (N + kWlThreads - 1) / kWlThreads;
                k_wl_moddown<<<(unsigned)(chunks * (long long)Gr.down.size()), kWlThreads, 0, q>>>(Gr.d_down, chunks,
                                                                                                  N, t->d_info);
                cerr = (int)cudaGetLastError();
                note_launch();
            }
            if (!cerr) cerr = cudaEventRecord(joins[g], q);
            if (!cerr) cerr = cudaStreamWaitEvent(cs, joins[g], 0);
        }
        const int e2 = cudaStreamEndCapture(cs, &graph);
        err = cerr ? cerr : e2;
    }
    const uint64_t captured = launch_counter() - counted0;
    forget_launches(captured);
    if (!err) err = cudaGraphInstantiate(&w.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    for (int g = 0; g < G; ++g) {
        if (gs[g]) cudaStreamDestroy(gs[g]);
        if (joins[g]) cudaEventDestroy(joins[g]);
    }
    if (fork) cudaEventDestroy(fork);
    if (cs) cudaStreamDestroy(cs);
    if (err) {
        check_cuda(err, kWhere);
        w.exec = nullptr;
        return 1;
    }
    w.launches_per_run = (int)captured;
    return 0;
}

}  // namespace

int read_wl_fault(int* out) {
    return (int)cudaMemcpyFromSymbol(out, vc_wl_fault, sizeof(int));
}

int clear_wl_fault() {
    const int zero = 0;
    return (int)cudaMemcpyToSymbol(vc_wl_fault, &zero, sizeof(int));
}

}  // namespace vc

using vc::WorkList;

extern "C" {

void* vfhe_cuda_worklist_new(void) { return new WorkList(); }

void vfhe_cuda_worklist_free(void* wl) {
    WorkList* w = (WorkList*)wl;
    if (!w) return;
    w->release();
    delete w;
}

int vfhe_cuda_worklist_add_chain(void* wl, void* ntt, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                                 const uint32_t* limbs, uint32_t nlimbs) {
    WorkList* w = (WorkList*)wl;
    if (!w || !limbs || nlimbs == 0 || nlimbs > (uint32_t)vc::kMaxLimbs - 1) {
        vc::set_error("vfhe_cuda_worklist_add_chain", "bad work list or limb list");
        return 1;
    }
    vc::Job j;
    memset(&j, 0, sizeof j);
    j.kind = 0;
    j.t = vc::as_ntt(ntt);
    j.out = d_out;
    j.a = d_a;
    j.b = d_b;
    j.L = (int)nlimbs;
    memcpy(j.limbs, limbs, nlimbs * sizeof(uint32_t));
    if (!vc::job_rows_ok(j)) {
        vc::set_error("vfhe_cuda_worklist_add_chain",
                      "limbs must be below 2^50 and inside the pool, rows 16-byte aligned, 2^8 <= P <= 2^17");
        return 1;
    }
    w->release();
    w->jobs.push_back(j);
    return 0;
}

int vfhe_cuda_worklist_add_keyswitch(void* wl, void* ntt, uint64_t* d_out, const uint64_t* d_ct,
                                     const uint32_t* limbs, uint32_t nlimbs, uint32_t special, const uint64_t* d_ksk) {
    WorkList* w = (WorkList*)wl;
    if (!w || !limbs || nlimbs == 0 || nlimbs > (uint32_t)vc::kMaxLimbs - 1) {
        vc::set_error("vfhe_cuda_worklist_add_keyswitch", "bad work list or limb list");
        return 1;
    }
    vc::Job j;
    memset(&j, 0, sizeof j);
    j.kind = 1;
    j.t = vc::as_ntt(ntt);
    j.out = d_out;
    j.a = d_ct;
    j.ksk = d_ksk;
    j.L = (int)nlimbs;
    j.special = special;
    memcpy(j.limbs, limbs, nlimbs * sizeof(uint32_t));
    if (!vc::job_rows_ok(j)) {
        vc::set_error("vfhe_cuda_worklist_add_keyswitch",
                      "limbs must be below 2^50 and inside the pool, rows 16-byte aligned, 2^8 <= P <= 2^17");
        return 1;
    }
    w->release();
    w->jobs.push_back(j);
    return 0;
}

int vfhe_cuda_worklist_compile(void* wl) {
    if (!vc::ensure_ready()) return 1;
    WorkList* w = (WorkList*)wl;
    if (!w || w->jobs.empty()) {
        vc::set_error("vfhe_cuda_worklist_compile", "empty work list");
        return 1;
    }
    return vc::compile(*w);
}

int vfhe_cuda_worklist_run(void* wl, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    WorkList* w = (WorkList*)wl;
    if (!w || w->jobs.empty()) {
        vc::set_error("vfhe_cuda_worklist_run", "empty work list");
        return 1;
    }
    if (!w->exec && !w->persistent && vc::compile(*w)) return 1;
    cudaStream_t st = (cudaStream_t)stream_;
    if (w->persistent) {
        // a cooperative launch: every CTA is resident, so the grid barriers between the
        // phases cannot wait on a CTA that has not started
        if (!vc::check_cuda(cudaMemsetAsync(w->plan.barrier, 0, 2 * sizeof(unsigned), st), "vfhe_cuda_worklist_run"))
            return 1;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        for (int part = 0; part < 3; ++part) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)w->grid[part], 1, 1);
            cfg.blockDim = dim3(vc::kWlPThreads, 1, 1);
            cfg.dynamicSmemBytes = vc::kWlPSmem;
            cfg.stream = st;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t le = part == 0   ? cudaLaunchKernelEx(&cfg, vc::k_wl_persistent<0>, w->plan)
                                   : part == 1 ? cudaLaunchKernelEx(&cfg, vc::k_wl_persistent<1>, w->plan)
                                               : cudaLaunchKernelEx(&cfg, vc::k_wl_persistent<2>, w->plan);
            if (!vc::check_cuda(le, "vfhe_cuda_worklist_run")) return 1;
        }
        vc::note_launch(3);
        return 0;
    }
    if (!vc::check_cuda(cudaGraphLaunch(w->exec, st), "vfhe_cuda_worklist_run")) return 1;
    vc::note_launch(w->launches_per_run);
    return 0;
}

int vfhe_cuda_worklist_set_mode(void* wl, int mode) {
    WorkList* w = (WorkList*)wl;
    if (!w || mode < 0 || mode > 1) {
        vc::set_error("vfhe_cuda_worklist_set_mode", "mode is 0 (three persistent launches) or 1 (graph of launches)");
        return 1;
    }
    if (mode != w->mode) w->release();
    w->mode = mode;
    return 0;
}

int vfhe_cuda_worklist_phase_ms(void* wl, double* out6) {
    WorkList* w = (WorkList*)wl;
    if (!w || !out6 || !w->persistent) return 1;
    unsigned long long t[7];
    if (!vc::check_cuda(cudaMemcpy(t, w->plan.phase_ns, sizeof t, cudaMemcpyDeviceToHost), "vfhe_cuda_worklist_phase_ms"))
        return 1;
    for (int k = 0; k < 6; ++k) out6[k] = (double)(t[k + 1] - t[k]) * 1e-6;
    return 0;
}

int vfhe_cuda_worklist_is_persistent(void* wl) {
    WorkList* w = (WorkList*)wl;
    return w && w->persistent ? 1 : 0;
}

uint64_t vfhe_cuda_worklist_device_bytes(void* wl) {
    WorkList* w = (WorkList*)wl;
    return w ? (uint64_t)w->dev_bytes : 0;
}

int vfhe_cuda_worklist_launches(void* wl) {
    WorkList* w = (WorkList*)wl;
    return w ? w->launches_per_run : 0;
}

}  // extern "C"
