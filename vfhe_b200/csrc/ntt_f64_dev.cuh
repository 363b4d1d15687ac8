// Device building blocks of the FP64 transforms (primes q < 2^50), shared by the
// transform kernels of ntt_f64.cu and the persistent work-list kernel of worklist.cu:
// index maps, twiddle loads, butterfly passes, shared-memory exchanges, and the work of
// one tile (forward / inverse, 16 residues per thread) or one column of a column pass.
//
// Range schedule (every modular product needs its input below 2^52 in magnitude):
//   forward (CT: x +- w y): each stage adds at most 3q/4, so passes of <= 4 stages
//     starting from |x| <= q stay below 4q; all residues are reduced at pass end;
//   inverse (GS: x + y, w (x - y)): sums double, so the sum outputs are reduced after
//     every second stage and at pass end; products are always <= 3q/4.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp64mod.cuh"
#include "ntt.cuh"

namespace vc {

namespace {

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

template <int LO>
__device__ __forceinline__ int own(int t, int m) {
    return ((t >> LO) << (LO + 4)) | (m << LO) | (t & ((1 << LO) - 1));
}

struct FCtx {
    double q, qinv;
    const double2* tw;
    const double2* lt;  // lane-major twiddles of bits 0..3 (PrimeInfo::fwd_lane / inv_lane)
    const double2* mt;  // the same for bits 2..5 by 64-residue group (fwd_mid / inv_mid)
    bool lazy = false;  // forward: skip the reductions between passes (fwd_lazy)
};

// A forward transform of a prime q < 2^47 needs no reduction between its load and its
// final canonical store: each stage adds at most |t| <= q/2 + q|y| 2^-54 <= 0.69q to a
// value (centred twiddles, |y| < 2^52), so after at most 20 stages every value stays
// below 0.5q + 20 * 0.69q < 14.3q < 2^51 and every step stays exact.
__device__ __forceinline__ bool fwd_lazy(const PrimeInfo& pi) { return pi.q < (1ULL << 47); }

// Position of slot (bit b, h) of 16-residue block g in a lane-major twiddle table.
__device__ __forceinline__ int lane_tw_index(int g, int b, int h) {
    return (((g >> 5) * 15 + ((1 << (3 - b)) - 1) + h) << 5) + (g & 31);
}

// A thread's 16 consecutive residues (p = row + 16 t): 32-byte accesses when the row is
// 32-byte aligned (a warp then touches each sector once per instruction), else 16-byte.
__device__ __forceinline__ void load16_u64(double (&x)[16], const uint64_t* p) {
    if ((reinterpret_cast<uintptr_t>(p) & 31) == 0) {
#pragma unroll
        for (int m = 0; m < 16; m += 4) {
            uint64_t a, b, c, d;
            // ordered like an ordinary load: rows may be transformed in place
            asm volatile("ld.global.v4.u64 {%0, %1, %2, %3}, [%4];"
                         : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
                         : "l"(p + m)
                         : "memory");
            x[m] = f_from_u64(a);
            x[m + 1] = f_from_u64(b);
            x[m + 2] = f_from_u64(c);
            x[m + 3] = f_from_u64(d);
        }
    } else {
        const ulonglong2* in = reinterpret_cast<const ulonglong2*>(p);
#pragma unroll
        for (int m = 0; m < 16; m += 2) {
            const ulonglong2 v = in[m / 2];
            x[m] = f_from_u64(v.x);
            x[m + 1] = f_from_u64(v.y);
        }
    }
}

// Canonical residues of x[0..15] to p[0..15] (same access widths as load16_u64).
__device__ __forceinline__ void store16_canonical(uint64_t* p, const double (&x)[16], double q, double qinv,
                                                  uint64_t qi) {
    if ((reinterpret_cast<uintptr_t>(p) & 31) == 0) {
#pragma unroll
        for (int m = 0; m < 16; m += 4) {
            const uint64_t a = f_to_canonical(x[m], q, qinv, qi), b = f_to_canonical(x[m + 1], q, qinv, qi);
            const uint64_t c = f_to_canonical(x[m + 2], q, qinv, qi), d = f_to_canonical(x[m + 3], q, qinv, qi);
            asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p + m), "l"(a), "l"(b), "l"(c), "l"(d)
                         : "memory");
        }
    } else {
        ulonglong2* out = reinterpret_cast<ulonglong2*>(p);
#pragma unroll
        for (int m = 0; m < 16; m += 2) {
            ulonglong2 v;
            v.x = f_to_canonical(x[m], q, qinv, qi);
            v.y = f_to_canonical(x[m + 1], q, qinv, qi);
            out[m / 2] = v;
        }
    }
}

// Twiddles of one pass.  In the field at LO, the butterfly of residue m at tile bit
// b = LO + bb uses index (... + (i >> (b+1))), which depends on m only through
// h = m >> (bb+1): stage bb needs 2^(3-bb) twiddles, a 4-stage pass 15.  Descending
// (forward) stages are stored first-stage-first; ascending (inverse) the same way.
template <int LO, int BFROM, int BTO>
struct PassTw {
    __host__ __device__ static constexpr int count() {
        int n = 0;
        for (int b = BFROM;; b += (BTO >= BFROM ? 1 : -1)) {
            n += 1 << (3 - (b - LO));
            if (b == BTO) break;
        }
        return n;
    }
    // offset of stage b's twiddles
    __host__ __device__ static constexpr int offset(int bq) {
        int n = 0;
        for (int b = BFROM; b != bq; b += (BTO >= BFROM ? 1 : -1)) n += 1 << (3 - (b - LO));
        return n;
    }
    double2 w[count()];
};

template <int K, int LO, int BHI, int BLO>
__device__ __forceinline__ void f_fwd_tw(PassTw<LO, BHI, BLO>& T, int t, int hi, int logP, const FCtx& c) {
#pragma unroll
    for (int b = BHI; b >= BLO; --b) {
        const int bb = b - LO;
        if constexpr (LO == 0) {
            // one twiddle per thread and slot: the lane-major copy keeps the warp's loads contiguous
            const int g = (hi << (K - 4)) + t;
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BHI, BLO>::offset(b) + h] = __ldg(&c.lt[lane_tw_index(g, b, h)]);
        } else if constexpr (LO == 2 && K >= 6) {
            // four threads per 64-residue group: a warp's loads are 8 consecutive pairs
            const int g = (hi << (K - 6)) + (t >> 2);
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BHI, BLO>::offset(b) + h] = __ldg(&c.mt[lane_tw_index(g, bb, h)]);
        } else {
            const int base = (1 << (logP - 1 - b)) + (hi << (K - b - 1));
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BHI, BLO>::offset(b) + h] =
                    __ldg(&c.tw[base + (own<LO>(t, h << (bb + 1)) >> (b + 1))]);
        }
    }
}

template <int K, int LO, int BHI, int BLO>
__device__ __forceinline__ void f_fwd_bits(double (&x)[16], const PassTw<LO, BHI, BLO>& T, const FCtx& c) {
#pragma unroll
    for (int b = BHI; b >= BLO; --b) {
        const int bb = b - LO;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & (1 << bb)) continue;
            const double2 w = T.w[PassTw<LO, BHI, BLO>::offset(b) + (m >> (bb + 1))];
            const double v = f_mulmod(x[m | (1 << bb)], w.x, w.y, c.q);
            const double u = x[m];
            x[m] = __dadd_rn(u, v);
            x[m | (1 << bb)] = __dsub_rn(u, v);
        }
    }
    // The pass at bit 0 is the transform's last and is followed by f_to_canonical, whose
    // own reduction takes its outputs (|x| < 4q < 2^52) directly.
    if constexpr (LO != 0) {
        if (!c.lazy) {
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = f_reduce(x[m], c.q, c.qinv);
        }
    }
}

// Inverse stages at bits BLO..BHI of the field at LO.  FINAL: the global last bit folds
// P^-1 (constants pinv and ilast, centred with their fl(./q) companions).
template <int K, int LO, int BLO, int BHI, bool FINAL>
__device__ __forceinline__ void f_inv_tw(PassTw<LO, BLO, BHI>& T, int t, int hi, int logP, const FCtx& c) {
#pragma unroll
    for (int b = BLO; b <= BHI; ++b) {
        if (FINAL && b == BHI) break;  // the last stage uses the P^-1 constants
        const int bb = b - LO;
        if constexpr (LO == 0) {
            const int g = (hi << (K - 4)) + t;
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BLO, BHI>::offset(b) + h] = __ldg(&c.lt[lane_tw_index(g, b, h)]);
        } else if constexpr (LO == 2 && K >= 6) {
            const int g = (hi << (K - 6)) + (t >> 2);
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BLO, BHI>::offset(b) + h] = __ldg(&c.mt[lane_tw_index(g, bb, h)]);
        } else {
            const int base = ((1 << logP) >> (b + 1)) + (hi << (K - b - 1));
#pragma unroll
            for (int h = 0; h < (1 << (3 - bb)); ++h)
                T.w[PassTw<LO, BLO, BHI>::offset(b) + h] =
                    __ldg(&c.tw[base + (own<LO>(t, h << (bb + 1)) >> (b + 1))]);
        }
    }
}

template <int K, int LO, int BLO, int BHI, bool FINAL>
__device__ __forceinline__ void f_inv_bits(double (&x)[16], const PassTw<LO, BLO, BHI>& T, const FCtx& c,
                                           const PrimeInfo& pi) {
#pragma unroll
    for (int b = BLO; b <= BHI; ++b) {
        const int bb = b - LO;
        const int j = b - BLO;  // stage index within this pass
        const bool last = FINAL && b == BHI;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & (1 << bb)) continue;
            const double u = x[m], v = x[m | (1 << bb)];
            if (last) {
                x[m] = f_mulmod(__dadd_rn(u, v), pi.pinv_d, pi.pinv_q, c.q);
                x[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), pi.ilast_d, pi.ilast_q, c.q);
            } else {
                const double2 w = T.w[PassTw<LO, BLO, BHI>::offset(b) + (m >> (bb + 1))];
                x[m] = __dadd_rn(u, v);
                x[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), w.x, w.y, c.q);
            }
        }
        // sums (m with bit bb clear) have doubled: bring them back after every second
        // stage and at the end of the pass
        if (!last && ((j & 1) || b == BHI)) {
#pragma unroll
            for (int m = 0; m < 16; ++m)
                if (!(m & (1 << bb))) x[m] = f_reduce(x[m], c.q, c.qinv);
        }
    }
}

template <int LO>
__device__ __forceinline__ void fput(double* sm, const double (&x)[16], int t) {
#pragma unroll
    for (int m = 0; m < 16; ++m) sm[pad(own<LO>(t, m))] = x[m];
}

template <int LO>
__device__ __forceinline__ void fget(double (&x)[16], const double* sm, int t) {
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = sm[pad(own<LO>(t, m))];
}

struct Tile {
    const uint64_t* src;
    uint64_t* dst;
    const PrimeInfo* pi;
    int hi;
};

template <bool TABLE>
__device__ __forceinline__ Tile locate(const RowSet& rows, const PrimeInfo* primes, int K, long long tile,
                                       int tiles_per_row) {
    const long long row = tile / tiles_per_row;
    const int hi = (int)(tile - row * tiles_per_row);
    Tile r;
    r.hi = hi;
    if constexpr (TABLE) {
        const RowDesc d = rows.table[row];
        const long long off = (long long)hi << K;
        r.src = (rows.table_src_is_dst ? d.out : d.in) + off;
        r.dst = d.out + off;
        r.pi = d.pi;
        return r;
    }
    const int per_poly = rows.nlimbs * rows.split;
    const long long b = row / per_poly;
    const int rem = (int)(row - b * per_poly);
    const int slot = rem / rows.split;
    const int blk = rem - slot * rows.split;
    const long long off = ((long long)blk << rows.logP) + ((long long)hi << K);
    r.src = rows.in[slot] + b * rows.in_batch_stride + off;
    r.dst = rows.out[slot] + b * rows.batch_stride + off;
    r.pi = primes + rows.prime[slot];
    return r;
}

template <int K>
struct TileThreads {
    static constexpr int value = (1 << (K - 4)) > 256 ? (1 << (K - 4)) : 256;
};

// Resident CTAs per SM asked of the compiler for the tile kernels: three 256-thread
// CTAs (at most 85 registers) measured ~4% faster than the unconstrained 64-register
// build at 2^16 points; the 512-thread tiles keep their own choice.
template <int K>
struct TileMinBlocks {
    static constexpr int value = TileThreads<K>::value >= 512 ? 1 : 3;
};

__device__ __forceinline__ double load_in(const uint64_t* p, bool in_double, bool reduce, const FCtx& c) {
    const uint64_t raw = *p;
    if (in_double) return __longlong_as_double((long long)raw);
    double v = f_from_u64(raw);
    return reduce ? f_reduce(v, c.q, c.qinv) : v;
}

// Barrier of one tile's threads.  GROUP: the CTA holds several independent tiles, and
// each tile's 2^(K-4) threads (a multiple of 32) meet at their own named barrier 1 + grp,
// so one tile's exchanges never wait for another's; otherwise the whole CTA meets.
template <int K, bool GROUP>
__device__ __forceinline__ void tile_sync(int grp) {
    if constexpr (GROUP) {
        static_assert((1 << (K - 4)) % 32 == 0, "a named barrier counts whole warps");
        asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "n"(1 << (K - 4)) : "memory");
    } else {
        __syncthreads();
    }
}

// Forward transform of the low K bits of tile r of a 2^logP-point row (16 residues per
// thread t; the tile's padded exchange buffer at sm); red: reduce each input modulo the
// row's prime on load.  STAGED: the input was copied into sm by a bulk copy; otherwise
// it is read from r.src.  tile_fwd_regs leaves the result in x (x[m] at index 16 t + m
// of the tile, |x| < 2^51, not reduced); tile_fwd_one stores it canonically to r.dst
// when `store` is set (a thread whose tile only pads out a group computes without
// storing).  GROUP, grp: the tile's threads synchronise at named barrier 1 + grp
// (tile_sync).
template <int K, bool IN_D, bool STAGED, bool GROUP = false>
__device__ __forceinline__ void tile_fwd_regs(const Tile& r, int logP, bool red, double* sm, int t, double (&x)[16],
                                              int grp = 0) {
    const PrimeInfo& pi = *r.pi;
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.fwd_d);
    c.lt = reinterpret_cast<const double2*>(pi.fwd_lane);
    c.mt = reinterpret_cast<const double2*>(pi.fwd_mid);
    c.lazy = fwd_lazy(pi);
    const int hi = r.hi;

    constexpr int L1 = K - 4;
    constexpr int L2 = (K - 8) > 0 ? (K - 8) : 0;
    constexpr int L3 = (K - 12) > 0 ? (K - 12) : 0;
    // each pass's twiddles are requested before the exchange that precedes the pass,
    // so their latency overlaps the barrier
    PassTw<L1, K - 1, L1> tw1;
    f_fwd_tw<K, L1, K - 1, L1>(tw1, t, hi, logP, c);
    if (STAGED) {
        const uint64_t* staged = reinterpret_cast<const uint64_t*>(sm);
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = load_in(staged + own<L1>(t, m), IN_D, red, c);
        tile_sync<K, GROUP>(grp);  // every input is in registers before the exchanges reuse the buffer
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = load_in(r.src + own<L1>(t, m), IN_D, red, c);
    }
    f_fwd_bits<K, L1, K - 1, L1>(x, tw1, c);
    PassTw<L2, L1 - 1, L2> tw2;
    f_fwd_tw<K, L2, L1 - 1, L2>(tw2, t, hi, logP, c);
    fput<L1>(sm, x, t);
    tile_sync<K, GROUP>(grp);
    fget<L2>(x, sm, t);
    f_fwd_bits<K, L2, L1 - 1, L2>(x, tw2, c);
    if constexpr (L2 > 0) {
        PassTw<L3, L2 - 1, L3> tw3;
        f_fwd_tw<K, L3, L2 - 1, L3>(tw3, t, hi, logP, c);
        tile_sync<K, GROUP>(grp);
        fput<L2>(sm, x, t);
        tile_sync<K, GROUP>(grp);
        fget<L3>(x, sm, t);
        f_fwd_bits<K, L3, L2 - 1, L3>(x, tw3, c);
        if constexpr (L3 > 0) {
            PassTw<0, L3 - 1, 0> tw4;
            f_fwd_tw<K, 0, L3 - 1, 0>(tw4, t, hi, logP, c);
            tile_sync<K, GROUP>(grp);
            fput<L3>(sm, x, t);
            tile_sync<K, GROUP>(grp);
            fget<0>(x, sm, t);
            f_fwd_bits<K, 0, L3 - 1, 0>(x, tw4, c);
        }
    }
}

template <int K, bool IN_D, bool STAGED, bool GROUP = false>
__device__ __forceinline__ void tile_fwd_one(const Tile& r, const RowSet& rows, double* sm, int t, bool store,
                                             int grp = 0) {
    double x[16];
    tile_fwd_regs<K, IN_D, STAGED, GROUP>(r, rows.logP, rows.reduce_input != 0, sm, t, x, grp);
    if (store) store16_canonical(r.dst + 16 * t, x, r.pi->qd, r.pi->qinv, r.pi->q);
}

// Inverse passes of the low K bits of one tile whose 16 residues per thread t are in x
// (x[m] at index 16 t + m, |x| < q; the forward passes leave this layout).  FINAL
// (K == logP): P^-1 folded in.  On return x[m] is at index own<K - 4>(t, m) of the tile.
template <int K, bool FINAL, bool GROUP = false>
__device__ __forceinline__ void tile_inv_regs(const PrimeInfo& pi, int logP, int hi, double* sm, int t,
                                              double (&x)[16], int grp = 0) {
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.inv_d);
    c.lt = reinterpret_cast<const double2*>(pi.inv_lane);
    c.mt = reinterpret_cast<const double2*>(pi.inv_mid);

    constexpr int F1 = 4 < (K - 4) ? 4 : (K - 4);
    constexpr int F2 = 8 < (K - 4) ? 8 : (K - 4);
    constexpr int F3 = 12 < (K - 4) ? 12 : (K - 4);
    PassTw<0, 0, 3> tw1;
    f_inv_tw<K, 0, 0, 3, false>(tw1, t, hi, logP, c);
    f_inv_bits<K, 0, 0, 3, false>(x, tw1, c, pi);
    if constexpr (K <= 8) {
        PassTw<F1, 4, K - 1> tw2;
        f_inv_tw<K, F1, 4, K - 1, FINAL>(tw2, t, hi, logP, c);
        fput<0>(sm, x, t);
        tile_sync<K, GROUP>(grp);
        fget<F1>(x, sm, t);
        f_inv_bits<K, F1, 4, K - 1, FINAL>(x, tw2, c, pi);
    } else {
        PassTw<F1, 4, 7> tw2;
        f_inv_tw<K, F1, 4, 7, false>(tw2, t, hi, logP, c);
        fput<0>(sm, x, t);
        tile_sync<K, GROUP>(grp);
        fget<F1>(x, sm, t);
        f_inv_bits<K, F1, 4, 7, false>(x, tw2, c, pi);
        if constexpr (K <= 12) {
            PassTw<F2, 8, K - 1> tw3;
            f_inv_tw<K, F2, 8, K - 1, FINAL>(tw3, t, hi, logP, c);
            tile_sync<K, GROUP>(grp);
            fput<F1>(sm, x, t);
            tile_sync<K, GROUP>(grp);
            fget<F2>(x, sm, t);
            f_inv_bits<K, F2, 8, K - 1, FINAL>(x, tw3, c, pi);
        } else {
            PassTw<F2, 8, 11> tw3;
            f_inv_tw<K, F2, 8, 11, false>(tw3, t, hi, logP, c);
            tile_sync<K, GROUP>(grp);
            fput<F1>(sm, x, t);
            tile_sync<K, GROUP>(grp);
            fget<F2>(x, sm, t);
            f_inv_bits<K, F2, 8, 11, false>(x, tw3, c, pi);
            PassTw<F3, 12, K - 1> tw4;
            f_inv_tw<K, F3, 12, K - 1, FINAL>(tw4, t, hi, logP, c);
            tile_sync<K, GROUP>(grp);
            fput<F2>(sm, x, t);
            tile_sync<K, GROUP>(grp);
            fget<F3>(x, sm, t);
            f_inv_bits<K, F3, 12, K - 1, FINAL>(x, tw4, c, pi);
        }
    }
}

// Inverse transform of the low K bits of tile r.  FINAL (K == logP): P^-1 folded in,
// canonical output; otherwise centred doubles for the column pass.  STAGED and store as
// for tile_fwd_one.
template <int K, bool FINAL, bool STAGED, bool GROUP = false>
__device__ __forceinline__ void tile_inv_one(const Tile& r, const RowSet& rows, double* sm, int t, bool store,
                                             int grp = 0) {
    const PrimeInfo& pi = *r.pi;
    double x[16];
    if (STAGED) {
        const ulonglong2* in = reinterpret_cast<const ulonglong2*>(reinterpret_cast<const uint64_t*>(sm) + 16 * t);
#pragma unroll
        for (int m = 0; m < 16; m += 2) {
            const ulonglong2 v = in[m / 2];
            x[m] = f_from_u64(v.x);
            x[m + 1] = f_from_u64(v.y);
        }
    } else {
        load16_u64(x, r.src + 16 * t);
    }
    if (STAGED) tile_sync<K, GROUP>(grp);  // every input is in registers before the exchanges reuse the buffer
    tile_inv_regs<K, FINAL, GROUP>(pi, rows.logP, r.hi, sm, t, x, grp);
    constexpr int LAST = K - 4;
    if (!store) return;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        uint64_t* p = r.dst + own<LAST>(t, m);
        if (FINAL) *p = f_to_canonical(x[m], pi.qd, pi.qinv, pi.q);
        else *p = (uint64_t)__double_as_longlong(x[m]);
    }
}

// The inverse column stages (index bits KT .. KT + K1 - 1, the transform's last, P^-1
// folded into the final stage) of one column whose x[m] sits at index m 2^KT + column:
// centred doubles from the tile pass in, centred values |x| < 2^51 out.
template <int K1>
__device__ __forceinline__ void col_inv_regs(double (&x)[1 << K1], const PrimeInfo& pi, int logP, int KT) {
    constexpr int R = 1 << K1;
    const double q = pi.qd, qinv = pi.qinv;
    const double2* tw = reinterpret_cast<const double2*>(pi.inv_d);
#pragma unroll
    for (int bb = 0; bb < K1; ++bb) {
        const int base = (1 << logP) >> (bb + KT + 1);
        const bool last = bb == K1 - 1;
#pragma unroll
        for (int m = 0; m < R; ++m) {
            if (m & (1 << bb)) continue;
            const double u = x[m], v = x[m | (1 << bb)];
            if (last) {
                x[m] = f_mulmod(__dadd_rn(u, v), pi.pinv_d, pi.pinv_q, q);
                x[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), pi.ilast_d, pi.ilast_q, q);
            } else {
                const double2 w = __ldg(&tw[base + (m >> (bb + 1))]);
                x[m] = __dadd_rn(u, v);
                x[m | (1 << bb)] = f_mulmod(__dsub_rn(u, v), w.x, w.y, q);
            }
        }
        if (!last && (bb & 1)) {
#pragma unroll
            for (int m = 0; m < R; ++m)
                if (!(m & (1 << bb))) x[m] = f_reduce(x[m], q, qinv);
        }
    }
}

// Column-pass work of column gc (see k_col_f below).
template <int K1, bool INV>
__device__ __forceinline__ void col_one(const RowSet& rows, const PrimeInfo* __restrict__ primes, long long gc,
                                        int KT) {
    constexpr int R = 1 << K1;
    const long long row = gc >> KT;
    const int cc = (int)(gc & ((1 << KT) - 1));
    const uint64_t* src;
    uint64_t* dst;
    const PrimeInfo* pp;
    if (rows.table) {
        const RowDesc d = rows.table[row];
        src = (rows.table_src_is_dst ? d.out : d.in) + cc;
        dst = d.out + cc;
        pp = d.pi;
    } else {
        const int per_poly = rows.nlimbs * rows.split;
        const long long b = row / per_poly;
        const int rem = (int)(row - b * per_poly);
        const int slot = rem / rows.split;
        const int blk = rem - slot * rows.split;
        const long long off = ((long long)blk << rows.logP) + cc;
        src = rows.in[slot] + b * rows.in_batch_stride + off;
        dst = rows.out[slot] + b * rows.batch_stride + off;
        pp = primes + rows.prime[slot];
    }
    const PrimeInfo& pi = *pp;
    const double q = pi.qd, qinv = pi.qinv;
    const int logP = rows.logP;
    double x[R];
    if (!INV) {
        const double2* tw = reinterpret_cast<const double2*>(pi.fwd_d);
        const bool lazy = fwd_lazy(pi);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            double v = f_from_u64(src[(long long)m << KT]);
            x[m] = rows.reduce_input ? f_reduce(v, q, qinv) : v;
        }
#pragma unroll
        for (int bb = K1 - 1; bb >= 0; --bb) {
            const int base = 1 << (logP - KT - 1 - bb);
#pragma unroll
            for (int m = 0; m < R; ++m) {
                if (m & (1 << bb)) continue;
                const double2 w = __ldg(&tw[base + (m >> (bb + 1))]);
                const double v = f_mulmod(x[m | (1 << bb)], w.x, w.y, q);
                const double u = x[m];
                x[m] = __dadd_rn(u, v);
                x[m | (1 << bb)] = __dsub_rn(u, v);
            }
            // at most four stages between reductions (|x| < 4q)
            if (bb == K1 - 4 && bb > 0 && !lazy) {
#pragma unroll
                for (int m = 0; m < R; ++m) x[m] = f_reduce(x[m], q, qinv);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m)
            dst[(long long)m << KT] = (uint64_t)__double_as_longlong(lazy ? x[m] : f_reduce(x[m], q, qinv));
    } else {
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = __longlong_as_double((long long)src[(long long)m << KT]);
        col_inv_regs<K1>(x, pi, logP, KT);
#pragma unroll
        for (int m = 0; m < R; ++m) dst[(long long)m << KT] = f_to_canonical(x[m], q, qinv, pi.q);
    }
}

}  // namespace

}  // namespace vc
