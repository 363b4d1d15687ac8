// Register-blocked NTT with FP64 butterflies (primes q < 2^50).
//
// Same schedule as ntt_rb.cu (16 residues per thread, 4-bit fields, padded shared
// memory, column pass for transforms above 2^13); the butterflies run on the FP64 pipe
// using the exact arithmetic of fp64mod.cuh.  Residues are centred doubles between
// passes; the row buffer itself carries those doubles between the two passes of a
// split transform and holds canonical uint64 residues at the end.
//
// Range schedule (every modular product needs its input below 2^52 in magnitude):
//   forward (CT: x +- w y): each stage adds at most 3q/4, so passes of <= 4 stages
//     starting from |x| <= q stay below 4q; all residues are reduced at pass end;
//   inverse (GS: x + y, w (x - y)): sums double, so the sum outputs are reduced after
//     every second stage and at pass end; products are always <= 3q/4.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "bulk.cuh"
#include "fp64mod.cuh"
#include "ntt.cuh"
#include "ntt_f64_dev.cuh"

namespace vc {

namespace {

// ---- bulk asynchronous tile loads (persistent kernels)
//
// A persistent CTA keeps two tile buffers: while it transforms the tiles in one, the
// bulk-copy engine fills the other with its next group's input (bulk.cuh).  A wait
// that gives up records the fault in vc_tile_fault.

__device__ int vc_tile_fault;  // nonzero: a tile copy wait gave up

__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    vc::mbar_wait_bounded(bar, parity, &vc_tile_fault);
}

// Thread 0: request the input of tile group `grp` into buf (tiles at buf + l * padded).
template <int K, bool TABLE>
__device__ __forceinline__ void issue_group(const RowSet& rows, const PrimeInfo* primes, long long grp,
                                            int tiles_per_cta, int tiles_per_row, double* buf, uint64_t* bar) {
    constexpr int TILE = 1 << K, PADDED = TILE + (TILE >> 4);
    mbar_expect_tx(bar, (uint32_t)(tiles_per_cta * TILE * 8));
    for (int l = 0; l < tiles_per_cta; ++l) {
        const Tile rr = locate<TABLE>(rows, primes, K, grp * tiles_per_cta + l, tiles_per_row);
        bulk_load(buf + l * PADDED, rr.src, TILE * 8, bar);
    }
}

// Forward transform of the low K bits of each row.  IN_D: the row holds centred
// doubles from the column pass; otherwise canonical (or foreign, with reduce_input)
// uint64 residues.  Output: canonical uint64.
// PERSIST: a grid of a few CTAs per SM walks the ngroups groups of tiles_per_cta tiles
// (every thread of a CTA makes the same number of trips), loading each group's input
// with bulk asynchronous copies into one of two shared buffers while the previous
// group computes; otherwise CTA b takes group b, reads its input straight from global
// memory, and the compiler keeps the lean straight-line register allocation.
template <int K, bool IN_D, bool PERSIST, bool TABLE>
__global__ void __launch_bounds__(TileThreads<K>::value, TileMinBlocks<K>::value) k_tile_fwd_f(const __grid_constant__ RowSet rows,
                                                                     const PrimeInfo* __restrict__ primes,
                                                                     int tiles_per_cta, int tiles_per_row,
                                                                     long long ngroups) {
    constexpr int TPT = 1 << (K - 4);
    constexpr int PADDED = (1 << K) + (1 << (K - 4));
    extern __shared__ __align__(128) double fsm[];
    __shared__ uint64_t bars[2];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    double* bufs[2] = {fsm, fsm + (PERSIST ? tiles_per_cta * PADDED : 0)};
    if (PERSIST) {
        if (threadIdx.x == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            if ((long long)blockIdx.x < ngroups)
                issue_group<K, TABLE>(rows, primes, blockIdx.x, tiles_per_cta, tiles_per_row, bufs[0], &bars[0]);
        }
        __syncthreads();
    }
    int trip = 0;
    for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x, ++trip) {
    const int cur = PERSIST ? (trip & 1) : 0;
    double* sm = bufs[cur] + lt * PADDED;
    if (PERSIST) {
        const long long nxt = grp + gridDim.x;
        if (threadIdx.x == 0 && nxt < ngroups) {
            // the other buffer's last generic writes (exchanges) precede this async write
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_group<K, TABLE>(rows, primes, nxt, tiles_per_cta, tiles_per_row, bufs[cur ^ 1], &bars[cur ^ 1]);
        }
        mbar_wait_bounded(&bars[cur], (uint32_t)((trip >> 1) & 1));
    }
    const long long tile = grp * tiles_per_cta + lt;
    const Tile r = locate<TABLE>(rows, primes, K, tile, tiles_per_row);
    tile_fwd_one<K, IN_D, PERSIST>(r, rows, sm, t, true);
    if (!PERSIST) break;
    __syncthreads();  // the next trip rewrites shared memory
    }
}

// Inverse transform of the low K bits.  FINAL (K == logP): P^-1 folded in, canonical
// output; otherwise centred doubles are written for the column pass.
template <int K, bool FINAL, bool PERSIST, bool TABLE>
__global__ void __launch_bounds__(TileThreads<K>::value, TileMinBlocks<K>::value) k_tile_inv_f(const __grid_constant__ RowSet rows,
                                                                     const PrimeInfo* __restrict__ primes,
                                                                     int tiles_per_cta, int tiles_per_row,
                                                                     long long ngroups) {
    constexpr int TPT = 1 << (K - 4);
    constexpr int PADDED = (1 << K) + (1 << (K - 4));
    extern __shared__ __align__(128) double fsm[];
    __shared__ uint64_t bars[2];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    double* bufs[2] = {fsm, fsm + (PERSIST ? tiles_per_cta * PADDED : 0)};
    if (PERSIST) {
        if (threadIdx.x == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            if ((long long)blockIdx.x < ngroups)
                issue_group<K, TABLE>(rows, primes, blockIdx.x, tiles_per_cta, tiles_per_row, bufs[0], &bars[0]);
        }
        __syncthreads();
    }
    int trip = 0;
    for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x, ++trip) {
    const int cur = PERSIST ? (trip & 1) : 0;
    double* sm = bufs[cur] + lt * PADDED;
    if (PERSIST) {
        const long long nxt = grp + gridDim.x;
        if (threadIdx.x == 0 && nxt < ngroups) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_group<K, TABLE>(rows, primes, nxt, tiles_per_cta, tiles_per_row, bufs[cur ^ 1], &bars[cur ^ 1]);
        }
        mbar_wait_bounded(&bars[cur], (uint32_t)((trip >> 1) & 1));
    }
    const long long tile = grp * tiles_per_cta + lt;
    const Tile r = locate<TABLE>(rows, primes, K, tile, tiles_per_row);
    tile_inv_one<K, FINAL, PERSIST>(r, rows, sm, t, true);
    if (!PERSIST) break;
    __syncthreads();  // the next trip rewrites shared memory
    }
}

// Column pass over bits [KT, logP), KT the tile bits of the second pass: thread c
// owns j = m * 2^KT + c, m < 2^K1.
// Forward (first pass): canonical/foreign uint64 in, centred doubles out.
// Inverse (last pass): centred doubles in, canonical uint64 out.
// Up to radix 16 the kernel fits 64 registers, so four 256-thread CTAs share an SM.
template <int K1, bool INV>
__global__ void __launch_bounds__(256, (K1 >= 5 ? 2 : 4)) k_col_f(const __grid_constant__ RowSet rows,
                                               const PrimeInfo* __restrict__ primes, long long ncols, int KT) {
    const long long gc = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gc >= ncols) return;  // no barriers in this kernel
    col_one<K1, INV>(rows, primes, gc, KT);
}

// Largest dynamic shared memory the tile kernels may be given (200 KiB of the 227).
constexpr size_t kTileSmemMax = 200 * 1024;

// ---- fused split transforms on a thread-block cluster
//
// A row of P = 2^(K + K1) residues is held by a cluster of C = 2^K1 CTAs, CTA r owning
// the contiguous block [r 2^K, (r + 1) 2^K) in its shared memory.  The radix-2^K1
// column stages (index bits K .. logP-1) pair elements of the same in-block position
// across the C blocks, so each CTA runs them on a 1/C share of the positions with
// loads and stores into the other CTAs' shared memory (distributed shared memory);
// the low K bits are then the usual register-blocked tile passes, fed from shared
// memory.  The row crosses HBM once in and once out, instead of twice each way for
// the column kernel + tile kernel pair, and it is one launch.
namespace cgx = cooperative_groups;

template <int K, int K1, bool TABLE>
__global__ void __launch_bounds__(TileThreads<K>::value) k_fused_fwd_f(const __grid_constant__ RowSet rows,
                                                                      const PrimeInfo* __restrict__ primes) {
    constexpr int TPT = 1 << (K - 4), TILE = 1 << K, C = 1 << K1;
    extern __shared__ __align__(128) double fsm[];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int rank = (int)cluster.block_rank();
    const long long row = blockIdx.x / C;
    const int t = threadIdx.x;
    const Tile r = locate<TABLE>(rows, primes, K, row * C + rank, C);
    const PrimeInfo& pi = *r.pi;
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.fwd_d);
    c.lt = reinterpret_cast<const double2*>(pi.fwd_lane);
    c.mt = reinterpret_cast<const double2*>(pi.fwd_mid);
    c.lazy = fwd_lazy(pi);
    const int logP = rows.logP;
    const bool red = rows.reduce_input != 0;
    // phase 1: this CTA's block, natural order, as residues in doubles
#pragma unroll
    for (int m = 0; m < 16; ++m) fsm[t + TPT * m] = load_in(r.src + t + TPT * m, false, red, c);
    cluster.sync();
    // phase 2: column stages on positions [rank TILE/C, (rank + 1) TILE/C)
    {
        double* blk[C];
#pragma unroll
        for (int m = 0; m < C; ++m) blk[m] = cluster.map_shared_rank(fsm, m);
        double2 w[K1 * C / 2];  // stage bb's twiddles (at most C/2) do not depend on the position
#pragma unroll
        for (int bb = K1 - 1; bb >= 0; --bb)
#pragma unroll
            for (int m = 0; m < C; ++m)
                if (!(m & (1 << bb))) w[(K1 - 1 - bb) * (C / 2) + (m >> (bb + 1))] =
                    __ldg(&c.tw[(1 << (logP - K - 1 - bb)) + (m >> (bb + 1))]);
        for (int j = rank * (TILE / C) + t; j < (rank + 1) * (TILE / C); j += TPT) {
            double x[C];
#pragma unroll
            for (int m = 0; m < C; ++m) x[m] = blk[m][j];
#pragma unroll
            for (int bb = K1 - 1; bb >= 0; --bb) {
#pragma unroll
                for (int m = 0; m < C; ++m) {
                    if (m & (1 << bb)) continue;
                    const double2 ww = w[(K1 - 1 - bb) * (C / 2) + (m >> (bb + 1))];
                    const double v = f_mulmod(x[m | (1 << bb)], ww.x, ww.y, c.q);
                    const double u = x[m];
                    x[m] = __dadd_rn(u, v);
                    x[m | (1 << bb)] = __dsub_rn(u, v);
                }
            }
#pragma unroll
            for (int m = 0; m < C; ++m) blk[m][j] = f_reduce(x[m], c.q, c.qinv);
        }
    }
    cluster.sync();
    // phase 3: the tile passes over the low K bits of this block
    const int hi = rank;
    double x[16];
    constexpr int L1 = K - 4;
    constexpr int L2 = (K - 8) > 0 ? (K - 8) : 0;
    constexpr int L3 = (K - 12) > 0 ? (K - 12) : 0;
    PassTw<L1, K - 1, L1> tw1;
    f_fwd_tw<K, L1, K - 1, L1>(tw1, t, hi, logP, c);
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = fsm[own<L1>(t, m)];
    __syncthreads();  // every value is in registers before the exchanges reuse the buffer
    f_fwd_bits<K, L1, K - 1, L1>(x, tw1, c);
    PassTw<L2, L1 - 1, L2> tw2;
    f_fwd_tw<K, L2, L1 - 1, L2>(tw2, t, hi, logP, c);
    fput<L1>(fsm, x, t);
    __syncthreads();
    fget<L2>(x, fsm, t);
    f_fwd_bits<K, L2, L1 - 1, L2>(x, tw2, c);
    if constexpr (L2 > 0) {
        PassTw<L3, L2 - 1, L3> tw3;
        f_fwd_tw<K, L3, L2 - 1, L3>(tw3, t, hi, logP, c);
        __syncthreads();
        fput<L2>(fsm, x, t);
        __syncthreads();
        fget<L3>(x, fsm, t);
        f_fwd_bits<K, L3, L2 - 1, L3>(x, tw3, c);
        if constexpr (L3 > 0) {
            PassTw<0, L3 - 1, 0> tw4;
            f_fwd_tw<K, 0, L3 - 1, 0>(tw4, t, hi, logP, c);
            __syncthreads();
            fput<L3>(fsm, x, t);
            __syncthreads();
            fget<0>(x, fsm, t);
            f_fwd_bits<K, 0, L3 - 1, 0>(x, tw4, c);
        }
    }
    store16_canonical(r.dst + 16 * t, x, c.q, c.qinv, pi.q);
}

template <int K, int K1, bool TABLE>
__global__ void __launch_bounds__(TileThreads<K>::value) k_fused_inv_f(const __grid_constant__ RowSet rows,
                                                                      const PrimeInfo* __restrict__ primes) {
    constexpr int TPT = 1 << (K - 4), TILE = 1 << K, C = 1 << K1;
    extern __shared__ __align__(128) double fsm[];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int rank = (int)cluster.block_rank();
    const long long row = blockIdx.x / C;
    const int t = threadIdx.x;
    const Tile r = locate<TABLE>(rows, primes, K, row * C + rank, C);
    const PrimeInfo& pi = *r.pi;
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.inv_d);
    c.lt = reinterpret_cast<const double2*>(pi.inv_lane);
    c.mt = reinterpret_cast<const double2*>(pi.inv_mid);
    const int logP = rows.logP, hi = rank;
    // phase 1: inverse tile passes over the low K bits of this block
    double x[16];
    constexpr int F1 = 4 < (K - 4) ? 4 : (K - 4);
    constexpr int F2 = 8 < (K - 4) ? 8 : (K - 4);
    constexpr int F3 = 12 < (K - 4) ? 12 : (K - 4);
    load16_u64(x, r.src + 16 * t);
    PassTw<0, 0, 3> tw1;
    f_inv_tw<K, 0, 0, 3, false>(tw1, t, hi, logP, c);
    f_inv_bits<K, 0, 0, 3, false>(x, tw1, c, pi);
    if constexpr (K <= 8) {
        PassTw<F1, 4, K - 1> tw2;
        f_inv_tw<K, F1, 4, K - 1, false>(tw2, t, hi, logP, c);
        fput<0>(fsm, x, t);
        __syncthreads();
        fget<F1>(x, fsm, t);
        f_inv_bits<K, F1, 4, K - 1, false>(x, tw2, c, pi);
    } else {
        PassTw<F1, 4, 7> tw2;
        f_inv_tw<K, F1, 4, 7, false>(tw2, t, hi, logP, c);
        fput<0>(fsm, x, t);
        __syncthreads();
        fget<F1>(x, fsm, t);
        f_inv_bits<K, F1, 4, 7, false>(x, tw2, c, pi);
        if constexpr (K <= 12) {
            PassTw<F2, 8, K - 1> tw3;
            f_inv_tw<K, F2, 8, K - 1, false>(tw3, t, hi, logP, c);
            __syncthreads();
            fput<F1>(fsm, x, t);
            __syncthreads();
            fget<F2>(x, fsm, t);
            f_inv_bits<K, F2, 8, K - 1, false>(x, tw3, c, pi);
        } else {
            PassTw<F2, 8, 11> tw3;
            f_inv_tw<K, F2, 8, 11, false>(tw3, t, hi, logP, c);
            __syncthreads();
            fput<F1>(fsm, x, t);
            __syncthreads();
            fget<F2>(x, fsm, t);
            f_inv_bits<K, F2, 8, 11, false>(x, tw3, c, pi);
            PassTw<F3, 12, K - 1> tw4;
            f_inv_tw<K, F3, 12, K - 1, false>(tw4, t, hi, logP, c);
            __syncthreads();
            fput<F2>(fsm, x, t);
            __syncthreads();
            fget<F3>(x, fsm, t);
            f_inv_bits<K, F3, 12, K - 1, false>(x, tw4, c, pi);
        }
    }
    constexpr int LAST = K - 4;
    __syncthreads();  // the exchanges are over: the block goes back in natural order
#pragma unroll
    for (int m = 0; m < 16; ++m) fsm[own<LAST>(t, m)] = x[m];
    cluster.sync();
    // phase 2: inverse column stages (P^-1 folded into the last), canonical results
    {
        double* blk[C];
#pragma unroll
        for (int m = 0; m < C; ++m) blk[m] = cluster.map_shared_rank(fsm, m);
        for (int j = rank * (TILE / C) + t; j < (rank + 1) * (TILE / C); j += TPT) {
            double y[C];
#pragma unroll
            for (int m = 0; m < C; ++m) y[m] = blk[m][j];
#pragma unroll
            for (int bb = 0; bb < K1; ++bb) {
                const int base = (1 << logP) >> (bb + K + 1);
                const bool last = bb == K1 - 1;
#pragma unroll
                for (int m = 0; m < C; ++m) {
                    if (m & (1 << bb)) continue;
                    const double u = y[m], v = y[m | (1 << bb)];
                    if (last) {
                        y[m] = f_mulmod(__dadd_rn(u, v), pi.pinv_d, pi.pinv_q, c.q);
                        y[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), pi.ilast_d, pi.ilast_q, c.q);
                    } else {
                        const double2 w = __ldg(&c.tw[base + (m >> (bb + 1))]);
                        y[m] = __dadd_rn(u, v);
                        y[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), w.x, w.y, c.q);
                    }
                }
                if (!last && (bb & 1)) {
#pragma unroll
                    for (int m = 0; m < C; ++m)
                        if (!(m & (1 << bb))) y[m] = f_reduce(y[m], c.q, c.qinv);
                }
            }
#pragma unroll
            for (int m = 0; m < C; ++m)
                reinterpret_cast<uint64_t*>(blk[m])[j] = f_to_canonical(y[m], c.q, c.qinv, pi.q);
        }
    }
    cluster.sync();
    // phase 3: this CTA's block to global memory
    const uint64_t* done = reinterpret_cast<const uint64_t*>(fsm);
#pragma unroll
    for (int m = 0; m < 16; ++m) r.dst[t + TPT * m] = done[t + TPT * m];
}

template <typename KernelT>
int set_smem(KernelT kern, size_t bytes) {
    if (bytes <= 48 * 1024) return 0;
    // one attribute call per kernel: raised straight to the maximum, then remembered
    static std::mutex mu;
    static std::vector<const void*> done;
    std::lock_guard<std::mutex> lk(mu);
    for (const void* k : done)
        if (k == (const void*)kern) return 0;
    const int e = (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemMax);
    if (!e) done.push_back((const void*)kern);
    return e;
}

// mode: 0 forward (canonical in), 1 forward (doubles in), 2 inverse final, 3 inverse to doubles
template <int K>
int tile_launch(const RowSet& rows, const PrimeInfo* d_primes, int mode, int tiles_per_row, const NttSchedule& sc,
                cudaStream_t st) {
    constexpr int TPT = 1 << (K - 4);
    const long long ntiles = rowset_rows(rows) * tiles_per_row;
    int tiles_per_cta = TPT >= 256 ? 1 : 256 / TPT;
    // a tuned tiles-per-CTA is taken when it fits the kernel's launch bound and shared memory
    if (sc.tiles_per_cta > 0 && TPT * sc.tiles_per_cta <= TileThreads<K>::value &&
        (sc.tiles_per_cta & (sc.tiles_per_cta - 1)) == 0 &&
        sizeof(double) * (size_t)sc.tiles_per_cta * ((1 << K) + (1 << (K - 4))) <= kTileSmemMax)
        tiles_per_cta = sc.tiles_per_cta;
    // the tile groups must cover the tiles exactly: no thread may leave before a barrier
    while (tiles_per_cta > 1 && (ntiles % tiles_per_cta) != 0) tiles_per_cta >>= 1;
    const long long ngroups = ntiles / tiles_per_cta;
    long long grid = ngroups;
    if (sc.ctas_per_sm > 0) {
        const long long cap = (long long)sc.ctas_per_sm * sm_count();
        if (cap < grid) grid = cap;
    }
    if (grid > 0x7fffffffLL) grid = 0x7fffffffLL;
    const bool persist = grid < ngroups;
    // persistent CTAs double-buffer their tiles
    const size_t smem = sizeof(double) * (size_t)tiles_per_cta * ((1 << K) + (1 << (K - 4))) * (persist ? 2 : 1);
    const int threads = TPT * tiles_per_cta;
    int e = 0;
#define VC_TILE_LAUNCH(KERN)                                                                              \
    do {                                                                                                  \
        e = set_smem(KERN, smem);                                                                         \
        if (!e) KERN<<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row, ngroups); \
    } while (0)
    const bool table = rows.table != nullptr;
    switch (mode * 4 + (persist ? 2 : 0) + (table ? 1 : 0)) {
        case 0: VC_TILE_LAUNCH((k_tile_fwd_f<K, false, false, false>)); break;
        case 1: VC_TILE_LAUNCH((k_tile_fwd_f<K, false, false, true>)); break;
        case 2: VC_TILE_LAUNCH((k_tile_fwd_f<K, false, true, false>)); break;
        case 3: VC_TILE_LAUNCH((k_tile_fwd_f<K, false, true, true>)); break;
        case 4: VC_TILE_LAUNCH((k_tile_fwd_f<K, true, false, false>)); break;
        case 5: VC_TILE_LAUNCH((k_tile_fwd_f<K, true, false, true>)); break;
        case 6: VC_TILE_LAUNCH((k_tile_fwd_f<K, true, true, false>)); break;
        case 7: VC_TILE_LAUNCH((k_tile_fwd_f<K, true, true, true>)); break;
        case 8: VC_TILE_LAUNCH((k_tile_inv_f<K, true, false, false>)); break;
        case 9: VC_TILE_LAUNCH((k_tile_inv_f<K, true, false, true>)); break;
        case 10: VC_TILE_LAUNCH((k_tile_inv_f<K, true, true, false>)); break;
        case 11: VC_TILE_LAUNCH((k_tile_inv_f<K, true, true, true>)); break;
        case 12: VC_TILE_LAUNCH((k_tile_inv_f<K, false, false, false>)); break;
        case 13: VC_TILE_LAUNCH((k_tile_inv_f<K, false, false, true>)); break;
        case 14: VC_TILE_LAUNCH((k_tile_inv_f<K, false, true, false>)); break;
        default: VC_TILE_LAUNCH((k_tile_inv_f<K, false, true, true>)); break;
    }
#undef VC_TILE_LAUNCH
    if (e) return e;
    note_launch();
    return (int)cudaGetLastError();
}

template <int K1>
int col_launch(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, int KT, cudaStream_t st) {
    const long long ncols = rowset_rows(rows) << KT;
    const long long grid = (ncols + 255) / 256;
    if (inverse) k_col_f<K1, true><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols, KT);
    else k_col_f<K1, false><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols, KT);
    note_launch();
    return (int)cudaGetLastError();
}

template <int K, int K1, bool TABLE>
int fused_launch_t(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t st) {
    constexpr int TPT = 1 << (K - 4), C = 1 << K1;
    const size_t smem = sizeof(double) * (size_t)((1 << K) + (1 << (K - 4)));
    const long long nrows = rowset_rows(rows);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nrows * C), 1, 1);
    cfg.blockDim = dim3(TPT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int e;
    if (inverse) {
        e = set_smem(k_fused_inv_f<K, K1, TABLE>, smem);
        if (!e) e = (int)cudaLaunchKernelEx(&cfg, k_fused_inv_f<K, K1, TABLE>, rows, d_primes);
    } else {
        e = set_smem(k_fused_fwd_f<K, K1, TABLE>, smem);
        if (!e) e = (int)cudaLaunchKernelEx(&cfg, k_fused_fwd_f<K, K1, TABLE>, rows, d_primes);
    }
    if (e) return e;
    note_launch();
    return (int)cudaGetLastError();
}

template <int K, int K1>
int fused_launch(const RowSet& rows, const PrimeInfo* d, bool inverse, cudaStream_t st) {
    return rows.table ? fused_launch_t<K, K1, true>(rows, d, inverse, st)
                      : fused_launch_t<K, K1, false>(rows, d, inverse, st);
}

// fused cluster transform for K in 11..13 and K1 in 1..3 (cluster of 2..8 CTAs)
int fused_dispatch(int K, int K1, const RowSet& rows, const PrimeInfo* d, bool inverse, cudaStream_t st) {
    switch (K * 4 + K1) {
        case 11 * 4 + 1: return fused_launch<11, 1>(rows, d, inverse, st);
        case 11 * 4 + 2: return fused_launch<11, 2>(rows, d, inverse, st);
        case 11 * 4 + 3: return fused_launch<11, 3>(rows, d, inverse, st);
        case 12 * 4 + 1: return fused_launch<12, 1>(rows, d, inverse, st);
        case 12 * 4 + 2: return fused_launch<12, 2>(rows, d, inverse, st);
        case 12 * 4 + 3: return fused_launch<12, 3>(rows, d, inverse, st);
        case 13 * 4 + 1: return fused_launch<13, 1>(rows, d, inverse, st);
        case 13 * 4 + 2: return fused_launch<13, 2>(rows, d, inverse, st);
        case 13 * 4 + 3: return fused_launch<13, 3>(rows, d, inverse, st);
        default: return (int)cudaErrorInvalidValue;
    }
}

int tile_dispatch(int K, const RowSet& rows, const PrimeInfo* d, int mode, int tpr, const NttSchedule& sc,
                  cudaStream_t st) {
    switch (K) {
        case 8: return tile_launch<8>(rows, d, mode, tpr, sc, st);
        case 9: return tile_launch<9>(rows, d, mode, tpr, sc, st);
        case 10: return tile_launch<10>(rows, d, mode, tpr, sc, st);
        case 11: return tile_launch<11>(rows, d, mode, tpr, sc, st);
        case 12: return tile_launch<12>(rows, d, mode, tpr, sc, st);
        case 13: return tile_launch<13>(rows, d, mode, tpr, sc, st);
        default: return (int)cudaErrorInvalidValue;
    }
}

int col_dispatch(int K1, const RowSet& rows, const PrimeInfo* d, bool inverse, int KT, cudaStream_t st) {
    switch (K1) {
        case 1: return col_launch<1>(rows, d, inverse, KT, st);
        case 2: return col_launch<2>(rows, d, inverse, KT, st);
        case 3: return col_launch<3>(rows, d, inverse, KT, st);
        case 4: return col_launch<4>(rows, d, inverse, KT, st);
        case 5: return col_launch<5>(rows, d, inverse, KT, st);
        default: return (int)cudaErrorInvalidValue;
    }
}

NttSchedule g_sched[kSchedMaxLogP + 1][kSchedRowBuckets];

template <int K, bool P, bool T>
int prepare_kp() {
    int e = set_smem(k_tile_fwd_f<K, false, P, T>, kTileSmemMax);
    if (!e) e = set_smem(k_tile_fwd_f<K, true, P, T>, kTileSmemMax);
    if (!e) e = set_smem(k_tile_inv_f<K, true, P, T>, kTileSmemMax);
    if (!e) e = set_smem(k_tile_inv_f<K, false, P, T>, kTileSmemMax);
    return e;
}

template <int K, int K1>
int prepare_fused() {
    int e = set_smem(k_fused_fwd_f<K, K1, false>, kTileSmemMax);
    if (!e) e = set_smem(k_fused_fwd_f<K, K1, true>, kTileSmemMax);
    if (!e) e = set_smem(k_fused_inv_f<K, K1, false>, kTileSmemMax);
    if (!e) e = set_smem(k_fused_inv_f<K, K1, true>, kTileSmemMax);
    return e;
}

template <int K>
int prepare_k() {
    int e = prepare_kp<K, false, false>();
    if (!e) e = prepare_kp<K, false, true>();
    if (!e) e = prepare_kp<K, true, false>();
    if (!e) e = prepare_kp<K, true, true>();
    if constexpr (K >= 11) {
        if (!e) e = prepare_fused<K, 1>();
        if (!e) e = prepare_fused<K, 2>();
        if (!e) e = prepare_fused<K, 3>();
    }
    return e;
}

}  // namespace

int read_tile_fault(int* out) {
    return (int)cudaMemcpyFromSymbol(out, vc_tile_fault, sizeof(int));
}

int clear_tile_fault() {
    const int zero = 0;
    return (int)cudaMemcpyToSymbol(vc_tile_fault, &zero, sizeof(int));
}

int prepare_chain_kernels();

int prepare_ntt_kernels() {
    int e = prepare_ckks_kernels();
    if (!e) e = prepare_chain_kernels();
    if (!e) e = prepare_k<8>();
    if (!e) e = prepare_k<9>();
    if (!e) e = prepare_k<10>();
    if (!e) e = prepare_k<11>();
    if (!e) e = prepare_k<12>();
    if (!e) e = prepare_k<13>();
    return e;
}

bool set_ntt_schedule(int logP, int rows_log2, const NttSchedule& s) {
    if (logP < 8 || logP > kSchedMaxLogP || rows_log2 < 0 || rows_log2 >= kSchedRowBuckets) return false;
    if (s.tile_bits != 0 && (s.tile_bits < 8 || s.tile_bits > 13 || s.tile_bits > logP || logP - s.tile_bits > 5))
        return false;
    if (s.tiles_per_cta < 0 || s.tiles_per_cta > 64 || s.ctas_per_sm < -2 || s.ctas_per_sm > 64) return false;
    if (s.ctas_per_sm == -1) {  // fused cluster transform: K in 11..13, logP - K in 1..3
        const int K = s.tile_bits;
        if (K < 11 || K > 13 || logP - K < 1 || logP - K > 3) return false;
    }
    if (s.ctas_per_sm == -2 && !flow_supported(s.tile_bits, logP - s.tile_bits)) return false;  // dataflow launch
    g_sched[logP][rows_log2] = s;
    return true;
}

NttSchedule get_ntt_schedule(int logP, long long nrows) {
    NttSchedule s = {0, 0, 0};
    if (logP < 8 || logP > kSchedMaxLogP || nrows <= 0) return s;
    int b = 0;
    while (b + 1 < kSchedRowBuckets && (2LL << b) <= nrows) ++b;  // floor(log2 nrows)
    return g_sched[logP][b];
}

// FP64-butterfly transform of every row (8 <= logP <= 17, all primes below 2^50).
int launch_ntt_f64(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream) {
    const int logP = rows.logP;
    if (logP < 8 || logP > 17) return -1;
    const NttSchedule sc = get_ntt_schedule(logP, rowset_rows(rows));
    int K = sc.tile_bits ? sc.tile_bits : (logP <= 13 ? logP : 12);
    if (K > logP || logP - K > 5) K = logP <= 13 ? logP : 12;
    if (K == logP) return tile_dispatch(logP, rows, d_primes, inverse ? 2 : 0, 1, sc, stream);
    const int K1 = logP - K;
    if (sc.ctas_per_sm == -1 && K >= 11 && K <= 13 && K1 >= 1 && K1 <= 3)
        return fused_dispatch(K, K1, rows, d_primes, inverse, stream);
    RowSet second = rows;
    for (int i = 0; i < rows.nlimbs; ++i) second.in[i] = rows.out[i];
    second.in_batch_stride = rows.batch_stride;
    second.reduce_input = 0;
    second.table_src_is_dst = 1;
    int e;
    if (sc.ctas_per_sm == -2 && flow_supported(K, K1)) {
        e = flow_dispatch(K, K1, rows, second, d_primes, inverse, sc.tiles_per_cta, stream);
        if (e != kFlowUnavailable) return e;
    }
    if (!inverse) {
        e = col_dispatch(K1, rows, d_primes, false, K, stream);
        if (e) return e;
        return tile_dispatch(K, second, d_primes, 1, 1 << K1, sc, stream);
    }
    e = tile_dispatch(K, rows, d_primes, 3, 1 << K1, sc, stream);
    if (e) return e;
    return col_dispatch(K1, second, d_primes, true, K, stream);
}

// The tile pass of an inverse transform whose schedule is a plain tile pass + column
// pass with at most `max_k1` column bits: the rows are left as centred doubles for a
// caller that fuses the column pass (and what follows it) into its own kernel.  Returns
// kTilePassUnavailable, having enqueued nothing, for any other schedule.
int launch_ntt_f64_inverse_tiles(const RowSet& rows, const PrimeInfo* d_primes, int max_k1, int* K1_out, int* KT_out,
                                 cudaStream_t stream) {
    const int logP = rows.logP;
    if (!ntt_f64_eligible(rows)) return kTilePassUnavailable;
    const NttSchedule sc = get_ntt_schedule(logP, rowset_rows(rows));
    int K = sc.tile_bits ? sc.tile_bits : (logP <= 13 ? logP : 12);
    if (K > logP || logP - K > 5) K = logP <= 13 ? logP : 12;
    const int K1 = logP - K;
    if (K1 < 1 || K1 > max_k1 || sc.ctas_per_sm < 0) return kTilePassUnavailable;
    *K1_out = K1;
    *KT_out = K;
    return tile_dispatch(K, rows, d_primes, 3, 1 << K1, sc, stream);
}

}  // namespace vc
