// Register-blocked NTT kernels (the fast path of launch_ntt).
//
// Same transforms as ntt.cu (conventions in ntt.cuh); a different schedule:
//   * a tile of 2^K residues (8 <= K <= 14) is transformed by 2^(K-4) threads that
//     each own 16 residues; up to four butterfly stages run in registers between
//     shared-memory exchanges (a 2^14 transform: 4 register passes, 3 exchanges);
//   * in a pass whose 4-bit field starts at bit LO, thread t owns the residues
//     i = (t >> LO) << (LO + 4) | m << LO | (t mod 2^LO), m < 16, and runs the stages
//     of that field's bits that are still pending;
//   * shared memory is padded (word i lives at i + i/16), which keeps every pass's
//     8-byte accesses at two wavefronts per warp (no bank conflicts);
//   * a thread loads only the twiddles its butterflies need (<= 15 per 32 butterflies);
//   * transforms larger than 2^14 split into a column pass over the index bits >= 12
//     (each thread transforms one column in registers) and 2^12-point tiles.
#include <cuda_runtime.h>
#include <stdlib.h>

#include "ntt.cuh"

namespace vc {

namespace {

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

template <int LO>
__device__ __forceinline__ int own(int t, int m) {
    return ((t >> LO) << (LO + 4)) | (m << LO) | (t & ((1 << LO) - 1));
}

// Forward (CT) butterflies at tile bits BHI down to BLO, field at LO.  Twiddle of the
// butterfly at tile bit b of tile `hi`: fwd[(1 << s) + (hi << (K-b-1)) + (i >> (b+1))]
// with s = logP - 1 - b.  Residues stay in [0, 4q).
template <int K, int LO, int BHI, int BLO>
__device__ __forceinline__ void fwd_bits(uint64_t (&x)[16], int t, int hi, int logP,
                                         const ulonglong2* __restrict__ tw, uint64_t q, uint64_t q2) {
#pragma unroll
    for (int b = BHI; b >= BLO; --b) {
        const int bb = b - LO;
        const int base = (1 << (logP - 1 - b)) + (hi << (K - b - 1));
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & (1 << bb)) continue;
            const ulonglong2 w = __ldg(&tw[base + (own<LO>(t, m) >> (b + 1))]);
            const uint64_t u = csub(x[m], q2);
            const uint64_t v = shoup_lazy(x[m | (1 << bb)], w.x, w.y, q);
            x[m] = u + v;
            x[m | (1 << bb)] = u + q2 - v;
        }
    }
}

// Inverse (GS) butterflies at tile bits BLO up to BHI, field at LO.  Twiddle:
// inv[(P >> (b+1)) + (hi << (K-b-1)) + (i >> (b+1))].  Residues stay in [0, 2q);
// with FINAL the last bit (global bit logP - 1) folds P^-1 in and ends canonical.
template <int K, int LO, int BLO, int BHI, bool FINAL>
__device__ __forceinline__ void inv_bits(uint64_t (&x)[16], int t, int hi, int logP,
                                         const ulonglong2* __restrict__ tw, const PrimeInfo& pi) {
    const uint64_t q = pi.q, q2 = pi.two_q;
#pragma unroll
    for (int b = BLO; b <= BHI; ++b) {
        const int bb = b - LO;
        const int base = ((1 << logP) >> (b + 1)) + (hi << (K - b - 1));
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & (1 << bb)) continue;
            const uint64_t u = x[m], v = x[m | (1 << bb)];
            if (FINAL && b == BHI) {
                x[m] = shoup(u + v, pi.p_inv, pi.p_inv_sh, q);
                x[m | (1 << bb)] = shoup(u + q2 - v, pi.inv_last, pi.inv_last_sh, q);
            } else {
                const ulonglong2 w = __ldg(&tw[base + (own<LO>(t, m) >> (b + 1))]);
                x[m] = csub(u + v, q2);
                x[m | (1 << bb)] = shoup_lazy(u + q2 - v, w.x, w.y, q);
            }
        }
    }
}

template <int LO>
__device__ __forceinline__ void put(uint64_t* sm, const uint64_t (&x)[16], int t) {
#pragma unroll
    for (int m = 0; m < 16; ++m) sm[pad(own<LO>(t, m))] = x[m];
}

template <int LO>
__device__ __forceinline__ void get(uint64_t (&x)[16], const uint64_t* sm, int t) {
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = sm[pad(own<LO>(t, m))];
}

struct Tile {
    const uint64_t* src;
    uint64_t* dst;
    const PrimeInfo* pi;
    int hi;
};

// Tile `tile` of the launch: tiles_per_row consecutive 2^K-point tiles per row.
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

// Forward transform of the low K bits of each row (the whole row when K == logP).
// Inputs in [0, 4q) (optionally reduced from another prime's residues); outputs canonical.
// Largest CTA a 2^K tile launch uses (tiles are packed up to 256 threads per CTA).
template <int K>
struct TileThreads {
    static constexpr int value = (1 << (K - 4)) > 256 ? (1 << (K - 4)) : 256;
};

template <int K>
__global__ void __launch_bounds__(TileThreads<K>::value) k_tile_fwd(const __grid_constant__ RowSet rows,
                                                      const PrimeInfo* __restrict__ primes, int tiles_per_cta,
                                                      int tiles_per_row, long long ntiles) {
    constexpr int TPT = 1 << (K - 4);
    extern __shared__ uint64_t smem[];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    // the launcher makes tiles_per_cta divide ntiles, so every tile of every CTA exists
    // and all threads reach every barrier
    const long long tile = (long long)blockIdx.x * tiles_per_cta + lt;
    uint64_t* sm = smem + lt * ((1 << K) + (1 << (K - 4)));
    const Tile r = locate(rows, primes, K, tile, tiles_per_row);
    const PrimeInfo& pi = *r.pi;
    const uint64_t q = pi.q, q2 = pi.two_q;
    const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.fwd);
    const int logP = rows.logP, hi = r.hi;
    uint64_t x[16];

    constexpr int L1 = K - 4;
    constexpr int L2 = (K - 8) > 0 ? (K - 8) : 0;
    constexpr int L3 = (K - 12) > 0 ? (K - 12) : 0;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        uint64_t v = r.src[own<L1>(t, m)];
        x[m] = rows.reduce_input ? reduce64(v, pi) : v;
    }
    fwd_bits<K, L1, K - 1, L1>(x, t, hi, logP, tw, q, q2);
    put<L1>(sm, x, t);
    __syncthreads();
    get<L2>(x, sm, t);
    fwd_bits<K, L2, L1 - 1, L2>(x, t, hi, logP, tw, q, q2);
    if constexpr (L2 > 0) {
        __syncthreads();
        put<L2>(sm, x, t);
        __syncthreads();
        get<L3>(x, sm, t);
        fwd_bits<K, L3, L2 - 1, L3>(x, t, hi, logP, tw, q, q2);
        if constexpr (L3 > 0) {
            __syncthreads();
            put<L3>(sm, x, t);
            __syncthreads();
            get<0>(x, sm, t);
            fwd_bits<K, 0, L3 - 1, 0>(x, t, hi, logP, tw, q, q2);
        }
    }
    // the final field is [0, 4): this thread holds residues 16t .. 16t + 15
    ulonglong2* out = reinterpret_cast<ulonglong2*>(r.dst + 16 * t);
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
        ulonglong2 v;
        v.x = csub(csub(x[m], q2), q);
        v.y = csub(csub(x[m + 1], q2), q);
        out[m / 2] = v;
    }
}

// Inverse transform of the low K bits of each row; with FINAL (K == logP) the P^-1
// scale is folded in and outputs are canonical, otherwise they stay in [0, 2q).
template <int K, bool FINAL>
__global__ void __launch_bounds__(TileThreads<K>::value) k_tile_inv(const __grid_constant__ RowSet rows,
                                                      const PrimeInfo* __restrict__ primes, int tiles_per_cta,
                                                      int tiles_per_row, long long ntiles) {
    constexpr int TPT = 1 << (K - 4);
    extern __shared__ uint64_t smem[];
    const int lt = threadIdx.x / TPT;
    const int t = threadIdx.x - lt * TPT;
    const long long tile = (long long)blockIdx.x * tiles_per_cta + lt;
    uint64_t* sm = smem + lt * ((1 << K) + (1 << (K - 4)));
    const Tile r = locate(rows, primes, K, tile, tiles_per_row);
    const PrimeInfo& pi = *r.pi;
    const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.inv);
    const int logP = rows.logP, hi = r.hi;
    uint64_t x[16];

    // fields: [0,4), [4,8) ... the last one is [K-4, K)
    constexpr int F1 = 4 < (K - 4) ? 4 : (K - 4);
    constexpr int F2 = 8 < (K - 4) ? 8 : (K - 4);
    constexpr int F3 = 12 < (K - 4) ? 12 : (K - 4);
    const ulonglong2* in = reinterpret_cast<const ulonglong2*>(r.src + 16 * t);
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
        const ulonglong2 v = in[m / 2];
        x[m] = v.x;
        x[m + 1] = v.y;
    }
    inv_bits<K, 0, 0, 3, false>(x, t, hi, logP, tw, pi);
    put<0>(sm, x, t);
    __syncthreads();
    get<F1>(x, sm, t);
    if constexpr (K <= 8) {
        inv_bits<K, F1, 4, K - 1, FINAL>(x, t, hi, logP, tw, pi);
    } else {
        inv_bits<K, F1, 4, 7, false>(x, t, hi, logP, tw, pi);
        __syncthreads();
        put<F1>(sm, x, t);
        __syncthreads();
        get<F2>(x, sm, t);
        if constexpr (K <= 12) {
            inv_bits<K, F2, 8, K - 1, FINAL>(x, t, hi, logP, tw, pi);
        } else {
            inv_bits<K, F2, 8, 11, false>(x, t, hi, logP, tw, pi);
            __syncthreads();
            put<F2>(sm, x, t);
            __syncthreads();
            get<F3>(x, sm, t);
            inv_bits<K, F3, 12, K - 1, FINAL>(x, t, hi, logP, tw, pi);
        }
    }
    constexpr int LAST = K - 4;
#pragma unroll
    for (int m = 0; m < 16; ++m) r.dst[own<LAST>(t, m)] = x[m];
}

// Column pass over the index bits [12, logP) of rows with 15 <= logP <= 17: thread c
// transforms the 2^K1 residues j = m * 4096 + c (K1 = logP - 12) entirely in registers.
template <int K1, bool INV>
__global__ void __launch_bounds__(256) k_col(const __grid_constant__ RowSet rows,
                                             const PrimeInfo* __restrict__ primes, long long ncols) {
    constexpr int R = 1 << K1;
    const long long gc = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gc >= ncols) return;
    const long long row = gc >> 12;
    const int c = (int)(gc & 4095);
    const int per_poly = rows.nlimbs * rows.split;
    const long long b = row / per_poly;
    const int rem = (int)(row - b * per_poly);
    const int slot = rem / rows.split;
    const int blk = rem - slot * rows.split;
    const long long off = ((long long)blk << rows.logP) + c;
    const uint64_t* src = rows.in[slot] + b * rows.in_batch_stride + off;
    uint64_t* dst = rows.out[slot] + b * rows.batch_stride + off;
    const PrimeInfo& pi = primes[rows.prime[slot]];
    const uint64_t q = pi.q, q2 = pi.two_q;
    const int logP = rows.logP;
    uint64_t x[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        uint64_t v = src[(long long)m << 12];
        x[m] = (!INV && rows.reduce_input) ? reduce64(v, pi) : v;
    }
    if (!INV) {
        const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.fwd);
#pragma unroll
        for (int bb = K1 - 1; bb >= 0; --bb) {
            const int b = bb + 12;
            const int base = 1 << (logP - 1 - b);
#pragma unroll
            for (int m = 0; m < R; ++m) {
                if (m & (1 << bb)) continue;
                const ulonglong2 w = __ldg(&tw[base + (m >> (bb + 1))]);
                const uint64_t u = csub(x[m], q2);
                const uint64_t v = shoup_lazy(x[m | (1 << bb)], w.x, w.y, q);
                x[m] = u + v;
                x[m | (1 << bb)] = u + q2 - v;
            }
        }
    } else {
        const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.inv);
#pragma unroll
        for (int bb = 0; bb < K1; ++bb) {
            const int b = bb + 12;
            const int base = (1 << logP) >> (b + 1);
#pragma unroll
            for (int m = 0; m < R; ++m) {
                if (m & (1 << bb)) continue;
                const uint64_t u = x[m], v = x[m | (1 << bb)];
                if (bb == K1 - 1) {
                    x[m] = shoup(u + v, pi.p_inv, pi.p_inv_sh, q);
                    x[m | (1 << bb)] = shoup(u + q2 - v, pi.inv_last, pi.inv_last_sh, q);
                } else {
                    const ulonglong2 w = __ldg(&tw[base + (m >> (bb + 1))]);
                    x[m] = csub(u + v, q2);
                    x[m | (1 << bb)] = shoup_lazy(u + q2 - v, w.x, w.y, q);
                }
            }
        }
    }
#pragma unroll
    for (int m = 0; m < R; ++m) dst[(long long)m << 12] = x[m];
}

template <typename KernelT>
int set_smem(KernelT kern, size_t bytes) {
    if (bytes <= 48 * 1024) return 0;
    return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int K>
int tile_launch(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, bool final_pass, int tiles_per_row,
                cudaStream_t st) {
    constexpr int TPT = 1 << (K - 4);
    const long long nrows = (long long)rows.batch * rows.nlimbs * rows.split;
    const long long ntiles = nrows * tiles_per_row;
    // tiles per CTA: up to 256 threads' worth, and a divisor of ntiles (a power of two),
    // so that no CTA holds a missing tile
    int tiles_per_cta = TPT >= 256 ? 1 : 256 / TPT;
    while (tiles_per_cta > 1 && (ntiles % tiles_per_cta) != 0) tiles_per_cta >>= 1;
    const long long grid = ntiles / tiles_per_cta;
    const size_t smem = sizeof(uint64_t) * (size_t)tiles_per_cta * ((1 << K) + (1 << (K - 4)));
    const int threads = TPT * tiles_per_cta;
    int e;
    if (!inverse) {
        e = set_smem(k_tile_fwd<K>, smem);
        if (e) return e;
        k_tile_fwd<K><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row, ntiles);
    } else if (final_pass) {
        e = set_smem(k_tile_inv<K, true>, smem);
        if (e) return e;
        k_tile_inv<K, true><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row,
                                                                   ntiles);
    } else {
        e = set_smem(k_tile_inv<K, false>, smem);
        if (e) return e;
        k_tile_inv<K, false><<<(unsigned)grid, threads, smem, st>>>(rows, d_primes, tiles_per_cta, tiles_per_row,
                                                                    ntiles);
    }
    note_launch();
    return (int)cudaGetLastError();
}

template <int K1>
int col_launch(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t st) {
    const long long nrows = (long long)rows.batch * rows.nlimbs * rows.split;
    const long long ncols = nrows * 4096;
    const long long grid = (ncols + 255) / 256;
    if (inverse) k_col<K1, true><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols);
    else k_col<K1, false><<<(unsigned)grid, 256, 0, st>>>(rows, d_primes, ncols);
    note_launch();
    return (int)cudaGetLastError();
}

int tile_dispatch(int K, const RowSet& rows, const PrimeInfo* d, bool inverse, bool final_pass, int tpr,
                  cudaStream_t st) {
    switch (K) {
        case 8: return tile_launch<8>(rows, d, inverse, final_pass, tpr, st);
        case 9: return tile_launch<9>(rows, d, inverse, final_pass, tpr, st);
        case 10: return tile_launch<10>(rows, d, inverse, final_pass, tpr, st);
        case 11: return tile_launch<11>(rows, d, inverse, final_pass, tpr, st);
        case 12: return tile_launch<12>(rows, d, inverse, final_pass, tpr, st);
        case 13: return tile_launch<13>(rows, d, inverse, final_pass, tpr, st);
        case 14: return tile_launch<14>(rows, d, inverse, final_pass, tpr, st);
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

// Register-blocked transform of every row of `rows` (8 <= logP <= 17).  Returns -1 when
// the size is outside that range so the caller can use the generic kernel.
int launch_ntt_rb(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream) {
    const int logP = rows.logP;
    if (logP < 8 || logP > 17) return -1;
    // Largest transform done by one tile.  A 2^14 tile needs 1024 threads and so at most
    // 64 registers per thread, which spills; measured on B200 a 4-point column pass plus
    // 2^12-point tiles is 1.5x faster, so the default is 2^13.
    static int single_max = -1;
    if (single_max < 0) {
        const char* s = getenv("VFHE_CUDA_NTT_SINGLE_MAX");
        single_max = s ? atoi(s) : 13;
        if (single_max < 13 || single_max > 14) single_max = 13;
    }
    if (logP <= single_max) return tile_dispatch(logP, rows, d_primes, inverse, true, 1, stream);
    const int K1 = logP - 12;
    RowSet second = rows;
    for (int i = 0; i < rows.nlimbs; ++i) second.in[i] = rows.out[i];
    second.in_batch_stride = rows.batch_stride;
    second.reduce_input = 0;
    int e;
    if (!inverse) {
        e = col_dispatch(K1, rows, d_primes, false, stream);
        if (e) return e;
        return tile_dispatch(12, second, d_primes, false, true, 1 << K1, stream);
    }
    e = tile_dispatch(12, rows, d_primes, true, false, 1 << K1, stream);
    if (e) return e;
    return col_dispatch(K1, second, d_primes, true, stream);
}

}  // namespace vc
