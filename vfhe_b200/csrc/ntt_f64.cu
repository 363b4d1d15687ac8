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
#include <cuda_runtime.h>

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
};

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
__device__ __forceinline__ void f_fwd_tw(PassTw<LO, BHI, BLO>& T, int t, int hi, int logP, const double2* tw) {
#pragma unroll
    for (int b = BHI; b >= BLO; --b) {
        const int bb = b - LO;
        const int base = (1 << (logP - 1 - b)) + (hi << (K - b - 1));
#pragma unroll
        for (int h = 0; h < (1 << (3 - bb)); ++h)
            T.w[PassTw<LO, BHI, BLO>::offset(b) + h] = __ldg(&tw[base + (own<LO>(t, h << (bb + 1)) >> (b + 1))]);
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
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = f_reduce(x[m], c.q, c.qinv);
}

// Inverse stages at bits BLO..BHI of the field at LO.  FINAL: the global last bit folds
// P^-1 (constants pinv and ilast, centred with their fl(./q) companions).
template <int K, int LO, int BLO, int BHI, bool FINAL>
__device__ __forceinline__ void f_inv_tw(PassTw<LO, BLO, BHI>& T, int t, int hi, int logP, const double2* tw) {
#pragma unroll
    for (int b = BLO; b <= BHI; ++b) {
        if (FINAL && b == BHI) break;  // the last stage uses the P^-1 constants
        const int bb = b - LO;
        const int base = ((1 << logP) >> (b + 1)) + (hi << (K - b - 1));
#pragma unroll
        for (int h = 0; h < (1 << (3 - bb)); ++h)
            T.w[PassTw<LO, BLO, BHI>::offset(b) + h] = __ldg(&tw[base + (own<LO>(t, h << (bb + 1)) >> (b + 1))]);
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

__device__ __forceinline__ Tile locate(const RowSet& rows, const PrimeInfo* primes, int K, long long tile,
                                       int tiles_per_row) {
    const long long row = tile / tiles_per_row;
    const int hi = (int)(tile - row * tiles_per_row);
    const int per_poly = rows.nlimbs * rows.split;
    const long long b = row / per_poly;
    const int rem = (int)(row - b * per_poly);
    const int slot = rem / rows.split;
    const int blk = rem - slot * rows.split;
    const long long off = ((long long)blk << rows.logP) + ((long long)hi << K);
    Tile r;
    r.src = rows.in[slot] + b * rows.in_batch_stride + off;
    r.dst = rows.out[slot] + b * rows.batch_stride + off;
    r.pi = primes + rows.prime[slot];
    r.hi = hi;
    return r;
}

template <int K>
struct TileThreads {
    static constexpr int value = (1 << (K - 4)) > 256 ? (1 << (K - 4)) : 256;
};

__device__ __forceinline__ double load_in(const uint64_t* p, bool in_double, bool reduce, const FCtx& c) {
    const uint64_t raw = *p;
    if (in_double) return __longlong_as_double((long long)raw);
    double v = f_from_u64(raw);
    return reduce ? f_reduce(v, c.q, c.qinv) : v;
}

// Forward transform of the low K bits of each row.  IN_D: the row holds centred
// doubles from the column pass; otherwise canonical (or foreign, with reduce_input)
// uint64 residues.  Output: canonical uint64.
template <int K, bool IN_D>
__global__ void __launch_bounds__(TileThreads<K>::value) k_tile_fwd_f(const __grid_constant__ RowSet rows,
                                                                     const PrimeInfo* __restrict__ primes,
                                                                     int tiles_per_cta, int tiles_per_row) {
    constexpr int TPT = 1 << (K - 4);
    extern __shared__ double fsm[];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    const long long tile = (long long)blockIdx.x * tiles_per_cta + lt;  // always exists
    double* sm = fsm + lt * ((1 << K) + (1 << (K - 4)));
    const Tile r = locate(rows, primes, K, tile, tiles_per_row);
    const PrimeInfo& pi = *r.pi;
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.fwd_d);
    const int logP = rows.logP, hi = r.hi;
    double x[16];

    constexpr int L1 = K - 4;
    constexpr int L2 = (K - 8) > 0 ? (K - 8) : 0;
    constexpr int L3 = (K - 12) > 0 ? (K - 12) : 0;
    const bool red = rows.reduce_input != 0;
    // each pass's twiddles are requested before the exchange that precedes the pass,
    // so their latency overlaps the barrier
    PassTw<L1, K - 1, L1> tw1;
    f_fwd_tw<K, L1, K - 1, L1>(tw1, t, hi, logP, c.tw);
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = load_in(r.src + own<L1>(t, m), IN_D, red, c);
    f_fwd_bits<K, L1, K - 1, L1>(x, tw1, c);
    PassTw<L2, L1 - 1, L2> tw2;
    f_fwd_tw<K, L2, L1 - 1, L2>(tw2, t, hi, logP, c.tw);
    fput<L1>(sm, x, t);
    __syncthreads();
    fget<L2>(x, sm, t);
    f_fwd_bits<K, L2, L1 - 1, L2>(x, tw2, c);
    if constexpr (L2 > 0) {
        PassTw<L3, L2 - 1, L3> tw3;
        f_fwd_tw<K, L3, L2 - 1, L3>(tw3, t, hi, logP, c.tw);
        __syncthreads();
        fput<L2>(sm, x, t);
        __syncthreads();
        fget<L3>(x, sm, t);
        f_fwd_bits<K, L3, L2 - 1, L3>(x, tw3, c);
        if constexpr (L3 > 0) {
            PassTw<0, L3 - 1, 0> tw4;
            f_fwd_tw<K, 0, L3 - 1, 0>(tw4, t, hi, logP, c.tw);
            __syncthreads();
            fput<L3>(sm, x, t);
            __syncthreads();
            fget<0>(x, sm, t);
            f_fwd_bits<K, 0, L3 - 1, 0>(x, tw4, c);
        }
    }
    ulonglong2* out = reinterpret_cast<ulonglong2*>(r.dst + 16 * t);
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
        ulonglong2 v;
        v.x = f_to_canonical(x[m], c.q, c.qinv, pi.q);
        v.y = f_to_canonical(x[m + 1], c.q, c.qinv, pi.q);
        out[m / 2] = v;
    }
}

// Inverse transform of the low K bits.  FINAL (K == logP): P^-1 folded in, canonical
// output; otherwise centred doubles are written for the column pass.
template <int K, bool FINAL>
__global__ void __launch_bounds__(TileThreads<K>::value) k_tile_inv_f(const __grid_constant__ RowSet rows,
                                                                     const PrimeInfo* __restrict__ primes,
                                                                     int tiles_per_cta, int tiles_per_row) {
    constexpr int TPT = 1 << (K - 4);
    extern __shared__ double fsm[];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    const long long tile = (long long)blockIdx.x * tiles_per_cta + lt;
    double* sm = fsm + lt * ((1 << K) + (1 << (K - 4)));
    const Tile r = locate(rows, primes, K, tile, tiles_per_row);
    const PrimeInfo& pi = *r.pi;
    FCtx c;
    c.q = pi.qd;
    c.qinv = pi.qinv;
    c.tw = reinterpret_cast<const double2*>(pi.inv_d);
    const int logP = rows.logP, hi = r.hi;
    double x[16];

    constexpr int F1 = 4 < (K - 4) ? 4 : (K - 4);
    constexpr int F2 = 8 < (K - 4) ? 8 : (K - 4);
    constexpr int F3 = 12 < (K - 4) ? 12 : (K - 4);
    const ulonglong2* in = reinterpret_cast<const ulonglong2*>(r.src + 16 * t);
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
        const ulonglong2 v = in[m / 2];
        x[m] = f_from_u64(v.x);
        x[m + 1] = f_from_u64(v.y);
    }
    PassTw<0, 0, 3> tw1;
    f_inv_tw<K, 0, 0, 3, false>(tw1, t, hi, logP, c.tw);
    f_inv_bits<K, 0, 0, 3, false>(x, tw1, c, pi);
    if constexpr (K <= 8) {
        PassTw<F1, 4, K - 1> tw2;
        f_inv_tw<K, F1, 4, K - 1, FINAL>(tw2, t, hi, logP, c.tw);
        fput<0>(sm, x, t);
        __syncthreads();
        fget<F1>(x, sm, t);
        f_inv_bits<K, F1, 4, K - 1, FINAL>(x, tw2, c, pi);
    } else {
        PassTw<F1, 4, 7> tw2;
        f_inv_tw<K, F1, 4, 7, false>(tw2, t, hi, logP, c.tw);
        fput<0>(sm, x, t);
        __syncthreads();
        fget<F1>(x, sm, t);
        f_inv_bits<K, F1, 4, 7, false>(x, tw2, c, pi);
        if constexpr (K <= 12) {
            PassTw<F2, 8, K - 1> tw3;
            f_inv_tw<K, F2, 8, K - 1, FINAL>(tw3, t, hi, logP, c.tw);
            __syncthreads();
            fput<F1>(sm, x, t);
            __syncthreads();
            fget<F2>(x, sm, t);
            f_inv_bits<K, F2, 8, K - 1, FINAL>(x, tw3, c, pi);
        } else {
            PassTw<F2, 8, 11> tw3;
            f_inv_tw<K, F2, 8, 11, false>(tw3, t, hi, logP, c.tw);
            __syncthreads();
            fput<F1>(sm, x, t);
            __syncthreads();
            fget<F2>(x, sm, t);
            f_inv_bits<K, F2, 8, 11, false>(x, tw3, c, pi);
            PassTw<F3, 12, K - 1> tw4;
            f_inv_tw<K, F3, 12, K - 1, FINAL>(tw4, t, hi, logP, c.tw);
            __syncthreads();
            fput<F2>(sm, x, t);
            __syncthreads();
            fget<F3>(x, sm, t);
            f_inv_bits<K, F3, 12, K - 1, FINAL>(x, tw4, c, pi);
        }
    }
    constexpr int LAST = K - 4;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        uint64_t* p = r.dst + own<LAST>(t, m);
        if (FINAL) *p = f_to_canonical(x[m], c.q, c.qinv, pi.q);
        else *p = (uint64_t)__double_as_longlong(x[m]);
    }
}

// Column pass over bits [12, logP): thread c owns j = m * 4096 + c, m < 2^K1.
// Forward (first pass): canonical/foreign uint64 in, centred doubles out.
// Inverse (last pass): centred doubles in, canonical uint64 out.
template <int K1, bool INV>
__global__ void __launch_bounds__(256) k_col_f(const __grid_constant__ RowSet rows,
                                               const PrimeInfo* __restrict__ primes, long long ncols) {
    constexpr int R = 1 << K1;
    const long long gc = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gc >= ncols) return;  // no barriers in this kernel
    const long long row = gc >> 12;
    const int cc = (int)(gc & 4095);
    const int per_poly = rows.nlimbs * rows.split;
    const long long b = row / per_poly;
    const int rem = (int)(row - b * per_poly);
    const int slot = rem / rows.split;
    const int blk = rem - slot * rows.split;
    const long long off = ((long long)blk << rows.logP) + cc;
    const uint64_t* src = rows.in[slot] + b * rows.in_batch_stride + off;
    uint64_t* dst = rows.out[slot] + b * rows.batch_stride + off;
    const PrimeInfo& pi = primes[rows.prime[slot]];
    const double q = pi.qd, qinv = pi.qinv;
    const int logP = rows.logP;
    double x[R];
    if (!INV) {
        const double2* tw = reinterpret_cast<const double2*>(pi.fwd_d);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            double v = f_from_u64(src[(long long)m << 12]);
            x[m] = rows.reduce_input ? f_reduce(v, q, qinv) : v;
        }
#pragma unroll
        for (int bb = K1 - 1; bb >= 0; --bb) {
            const int base = 1 << (logP - 13 - bb);
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
            if (bb == K1 - 4 && bb > 0) {
#pragma unroll
                for (int m = 0; m < R; ++m) x[m] = f_reduce(x[m], q, qinv);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m)
            dst[(long long)m << 12] = (uint64_t)__double_as_longlong(f_reduce(x[m], q, qinv));
    } else {
        const double2* tw = reinterpret_cast<const double2*>(pi.inv_d);
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = __longlong_as_double((long long)src[(long long)m << 12]);
#pragma unroll
        for (int bb = 0; bb < K1; ++bb) {
            const int base = (1 << logP) >> (bb + 13);
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
#pragma unroll
        for (int m = 0; m < R; ++m) dst[(long long)m << 12] = f_to_canonical(x[m], q, qinv, pi.q);
    }
}

template <typename KernelT>
int set_smem(KernelT kern, size_t bytes) {
    if (bytes <= 48 * 1024) return 0;
    return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// mode: 0 forward (canonical in), 1 forward (doubles in), 2 inverse final, 3 inverse to doubles
template <int K>
int tile_launch(const RowSet& rows, const PrimeInfo* d_primes, int mode, int tiles_per_row, cudaStream_t st) {
    constexpr int TPT = 1 << (K - 4);
    const long long nrows = (long long)rows.batch * rows.nlimbs * rows.split;
    const long long ntiles = nrows * tiles_per_row;
    int tiles_per_cta = TPT >= 256 ? 1 : 256 / TPT;
    while (tiles_per_cta > 1 && (ntiles % tiles_per_cta) != 0) tiles_per_cta >>= 1;
    const long long grid = ntiles / tiles_per_cta;
    const size_t smem = sizeof(double) * (size_t)tiles_per_cta * ((1 << K) + (1 << (K - 4)));
    const int threads = TPT * tiles_per_cta;
    int e = 0;
    switch (mode) {
        case 0:
            e = set_smem(k_tile_fwd_f<K, false>, smem);
            if (!e) k_tile_fwd_f<K, false><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row);
            break;
        case 1:
            e = set_smem(k_tile_fwd_f<K, true>, smem);
            if (!e) k_tile_fwd_f<K, true><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row);
            break;
        case 2:
            e = set_smem(k_tile_inv_f<K, true>, smem);
            if (!e) k_tile_inv_f<K, true><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row);
            break;
        default:
            e = set_smem(k_tile_inv_f<K, false>, smem);
            if (!e) k_tile_inv_f<K, false><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row);
            break;
    }
    if (e) return e;
    note_launch();
    return (int)cudaGetLastError();
}

template <int K1>
int col_launch(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t st) {
    const long long ncols = (long long)rows.batch * rows.nlimbs * rows.split * 4096;
    const long long grid = (ncols + 255) / 256;
    if (inverse) k_col_f<K1, true><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols);
    else k_col_f<K1, false><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols);
    note_launch();
    return (int)cudaGetLastError();
}

int tile_dispatch(int K, const RowSet& rows, const PrimeInfo* d, int mode, int tpr, cudaStream_t st) {
    switch (K) {
        case 8: return tile_launch<8>(rows, d, mode, tpr, st);
        case 9: return tile_launch<9>(rows, d, mode, tpr, st);
        case 10: return tile_launch<10>(rows, d, mode, tpr, st);
        case 11: return tile_launch<11>(rows, d, mode, tpr, st);
        case 12: return tile_launch<12>(rows, d, mode, tpr, st);
        case 13: return tile_launch<13>(rows, d, mode, tpr, st);
        default: return (int)cudaErrorInvalidValue;
    }
}

int col_dispatch(int K1, const RowSet& rows, const PrimeInfo* d, bool inverse, cudaStream_t st) {
    switch (K1) {
        case 2: return col_launch<2>(rows, d, inverse, st);
        case 3: return col_launch<3>(rows, d, inverse, st);
        case 4: return col_launch<4>(rows, d, inverse, st);
        case 5: return col_launch<5>(rows, d, inverse, st);
        default: return (int)cudaErrorInvalidValue;
    }
}

}  // namespace

// FP64-butterfly transform of every row (8 <= logP <= 17, all primes below 2^50).
int launch_ntt_f64(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream) {
    const int logP = rows.logP;
    if (logP < 8 || logP > 17) return -1;
    if (logP <= 13) return tile_dispatch(logP, rows, d_primes, inverse ? 2 : 0, 1, stream);
    const int K1 = logP - 12;
    RowSet second = rows;
    for (int i = 0; i < rows.nlimbs; ++i) second.in[i] = rows.out[i];
    second.in_batch_stride = rows.batch_stride;
    second.reduce_input = 0;
    int e;
    if (!inverse) {
        e = col_dispatch(K1, rows, d_primes, false, stream);
        if (e) return e;
        return tile_dispatch(12, second, d_primes, 1, 1 << K1, stream);
    }
    e = tile_dispatch(12, rows, d_primes, 3, 1 << K1, stream);
    if (e) return e;
    return col_dispatch(K1, second, d_primes, true, stream);
}

}  // namespace vc
