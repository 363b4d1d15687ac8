// CGGI bootstrap over the 32-bit torus with FP64 complex-FFT external products.
//
// The algorithm is the published TFHE bootstrap (Chillotti, Gama, Georgieva,
// Izabachene, J. Cryptology 33, 2020) with the reference's CGGI16 orchestration
// (modules/fhe/python/src/vfhe/fhe/cggi16.py:46-128: rotation with a half-box
// offset, CMUX(acc, acc X^a_i) per LWE coefficient, extraction at coefficient 0),
// then a base-2^kb LWE key switch back to the input key.  Conventions are those of
// oracle/cggi_torus_oracle.c (the exact-integer checker): uint32 torus, GLWE phase
// b - a S, signed gadget digits, GGSW row (component c, level l) at c * levels + l.
//
// Negacyclic products through a half-size complex FFT: a real polynomial p of N
// coefficients folds to z_j = (p_j + i p_{j+M}) zeta^j, M = N/2, zeta = e^{i pi/N};
// the M-point DFT with kernel e^{+2 pi i/M} evaluates p at the odd roots zeta^{4k+1},
// so pointwise products of spectra are spectra of negacyclic products.  Forward:
// decimation in frequency (natural in, bit-reversed out); inverse: decimation in
// time with the conjugate kernel (bit-reversed in, natural out) and 1/M; no
// permutation pass.  Key spectra come from the same forward code, so both operands
// are in the same bit-reversed order.
//
// Precision: digits |d| <= 2^(g-1) (64 at base 2^7), key values as signed 32-bit,
// 2 levels-by-components rows x N terms: sums below 2^50; FP64 (53-bit) FFTs then
// round each coefficient to the nearest integer, usually exact; the tests measure
// the maximum deviation from the exact integer product.
//
// One persistent launch runs whole blind rotations: each CTA owns one LWE at a time,
// keeps the accumulator and the spectra in shared memory for all n CMUX steps, and
// reads step i's key spectra (same for every CTA, so they stay in L2) directly.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "engine.cuh"

namespace vc {

namespace {

constexpr int kMaxLevels = 4;

// twiddles e^{2 pi i k / M} (k < M/2) and the twist zeta^j (j < M), per N
struct FourierTables {
    int N = 0;
    double2* d_tw = nullptr;
    double2* d_twist = nullptr;
};

std::mutex g_ft_mu;
std::vector<FourierTables> g_ft;

const FourierTables* fourier_tables(int N) {
    std::lock_guard<std::mutex> lk(g_ft_mu);
    for (auto& t : g_ft)
        if (t.N == N) return &t;
    const int M = N / 2;
    std::vector<double2> tw(M / 2), twist(M);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < M / 2; ++k) {
        const long double ang = 2.0L * pi * (long double)k / (long double)M;
        tw[k] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    for (int j = 0; j < M; ++j) {
        const long double ang = pi * (long double)j / (long double)N;
        twist[j] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    FourierTables t;
    t.N = N;
    if (cudaMalloc(&t.d_tw, sizeof(double2) * (M / 2)) != cudaSuccess ||
        cudaMalloc(&t.d_twist, sizeof(double2) * M) != cudaSuccess ||
        cudaMemcpy(t.d_tw, tw.data(), sizeof(double2) * (M / 2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(t.d_twist, twist.data(), sizeof(double2) * M, cudaMemcpyHostToDevice) != cudaSuccess)
        return nullptr;
    g_ft.push_back(t);
    return &g_ft.back();
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -a.y * b.y), __fma_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(__fma_rn(a.x, b.x, a.y * b.y), __fma_rn(a.y, b.x, -a.x * b.y));
}

// Digit `want` of the signed decomposition of v rounded to its top base_log * levels
// bits (digit 0 most significant), without materialising the others
__device__ __forceinline__ int digit_of(uint32_t v, int base_log, int levels, int want) {
    const int total = base_log * levels;
    uint64_t r = ((uint64_t)v + (1ULL << (31 - total))) >> (32 - total);
    r &= total >= 32 ? 0xFFFFFFFFULL : ((1ULL << total) - 1);
    const int half = 1 << (base_log - 1), full = 1 << base_log;
    int out = 0;
    for (int l = levels - 1; l >= 0; --l) {
        int x = (int)(r & (uint64_t)(full - 1));
        r >>= base_log;
        if (x >= half) {
            x -= full;
            r += 1;
        }
        if (l == want) out = x;
    }
    return out;
}

__device__ __forceinline__ int modswitch(uint32_t v, int logN2) {
    return (int)((((uint64_t)v + (1ULL << (31 - logN2))) >> (32 - logN2)) & ((1ULL << logN2) - 1));
}

// acc X^e at coefficient k (negacyclic, 0 <= e < 2N)
template <int N>
__device__ __forceinline__ uint32_t rot_at(const uint32_t* p, int k, int e) {
    int s = k - e;
    s = s < 0 ? s + 2 * N : s;
    return s < N ? p[s] : (uint32_t)(0u - p[s - N]);
}

// ---- register-blocked radix-8 FFT passes
//
// An M-point transform (M = 2^LOGM) of one array is done by M/8 threads holding 8
// values each.  Pass p covers index bits [LO, LO + NST): thread t holds the elements
// pidx<LO>(t, k), k < 8 (k supplies bits LO..LO+2), so all butterflies of the pass are
// in registers; passes exchange through shared memory with an XOR swizzle that keeps
// every pass's accesses free of bank conflicts.  Forward: LOGM/3 full passes from the
// top bits, then one partial pass (LOGM mod 3 stages) at bit 0; the inverse runs the
// same passes in reverse.  The final forward pass leaves element f = 8t + k in thread
// t, which is also the order of the key spectra in memory (position k * M/8 + t), so
// the multiply-accumulate reads both coalesced.

template <int LO>
__device__ __forceinline__ int pidx(int t, int k) {
    return ((t >> LO) << (LO + 3)) | (k << LO) | (t & ((1 << LO) - 1));
}

__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

template <int LOGM, int P>
struct PassOf {
    static constexpr int FULL = LOGM / 3;
    static constexpr int LO = P < FULL ? LOGM - 3 * (P + 1) : 0;
    static constexpr int NST = P < FULL ? 3 : LOGM % 3;
};

template <int LOGM>
struct Passes {
    static constexpr int count = (LOGM + 2) / 3;
};

// decimation-in-frequency stages of one pass (kernel e^{+2 pi i / M})
template <int LOGM, int LO, int NST>
__device__ __forceinline__ void dif(double2 (&v)[8], int t, const double2* __restrict__ tw) {
#pragma unroll
    for (int s = NST - 1; s >= 0; --s) {
        const int bit = 1 << s;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & bit) continue;
            const int j = pidx<LO>(t, k) & ((1 << (LO + s)) - 1);
            const double2 w = __ldg(&tw[j << (LOGM - 1 - LO - s)]);
            const double2 u = v[k], x = v[k | bit];
            v[k] = make_double2(u.x + x.x, u.y + x.y);
            v[k | bit] = cmul(make_double2(u.x - x.x, u.y - x.y), w);
        }
    }
}

// decimation-in-time stages of one pass (kernel e^{-2 pi i / M})
template <int LOGM, int LO, int NST>
__device__ __forceinline__ void dit(double2 (&v)[8], int t, const double2* __restrict__ tw) {
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        const int bit = 1 << s;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & bit) continue;
            const int j = pidx<LO>(t, k) & ((1 << (LO + s)) - 1);
            const double2 w = __ldg(&tw[j << (LOGM - 1 - LO - s)]);
            const double2 u = v[k], x = cmulc(v[k | bit], w);
            v[k] = make_double2(u.x + x.x, u.y + x.y);
            v[k | bit] = make_double2(u.x - x.x, u.y - x.y);
        }
    }
}

template <int LO>
__device__ __forceinline__ void put8(double2* a, const double2 (&v)[8], int t) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[swz(pidx<LO>(t, k))] = v[k];
}

template <int LO>
__device__ __forceinline__ void get8(double2 (&v)[8], const double2* a, int t) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = a[swz(pidx<LO>(t, k))];
}

// forward passes P .. count-1 of array a (pass P-1 left its values at a); barriers are
// taken by every thread of the block (active == false threads skip the work only)
template <int LOGM, int P>
__device__ __forceinline__ void fwd_rest(double2* a, int t, bool active, const double2* tw) {
    if constexpr (P < Passes<LOGM>::count) {
        using Q = PassOf<LOGM, P>;
        double2 v[8];
        if (active) {
            get8<Q::LO>(v, a, t);
            dif<LOGM, Q::LO, Q::NST>(v, t, tw);
        }
        __syncthreads();  // all reads of the previous layout done
        if (active) put8<Q::LO>(a, v, t);
        __syncthreads();
        fwd_rest<LOGM, P + 1>(a, t, active, tw);
    }
}

// inverse passes P down to 1 (pass P+1 left its values at a); pass 0 is done by the caller
template <int LOGM, int P>
__device__ __forceinline__ void inv_rest(double2* a, int t, bool active, const double2* tw) {
    if constexpr (P >= 1) {
        using Q = PassOf<LOGM, P>;
        double2 v[8];
        if (active) {
            get8<Q::LO>(v, a, t);
            dit<LOGM, Q::LO, Q::NST>(v, t, tw);
        }
        __syncthreads();
        if (active) put8<Q::LO>(a, v, t);
        __syncthreads();
        inv_rest<LOGM, P - 1>(a, t, active, tw);
    }
}

template <int N>
struct Smem {
    static constexpr int M = N / 2;
    // acc[2][N] uint32 | spec[2 L][M] double2 | outs[2][M] double2
    static constexpr size_t bytes(int levels) {
        return sizeof(uint32_t) * 2 * N + sizeof(double2) * (2 * levels * M + 2 * M);
    }
};

// One external product on the block's GLWE: digits of the source (MODE 0: acc X^ai -
// acc, from shared acc; MODE 1: the GLWE `src` in global memory), forward transforms,
// multiply-accumulate with the GGSW spectra `key` (key order), inverse transforms;
// MODE 0 adds the rounded result into acc, MODE 1 writes it to `dst` and the largest
// distance of an unrounded coefficient to its integer to *frac.
template <int LOGM, int LEVELS, int MODE>
__device__ __forceinline__ void ext_product(uint32_t* acc, double2* spec, double2* outs, const double2* __restrict__ key,
                                            int ai, int base_log, const uint32_t* __restrict__ src,
                                            uint32_t* __restrict__ dst, double* frac, const double2* __restrict__ tw,
                                            const double2* __restrict__ twist) {
    constexpr int M = 1 << LOGM, N = 2 * M, TPA = M / 8, R = 2 * LEVELS;
    constexpr int NP = Passes<LOGM>::count;
    const int arr = threadIdx.x / TPA, t = threadIdx.x - arr * TPA;
    // forward pass 0 straight from the digits (element j = t + k M/8)
    {
        using Q = PassOf<LOGM, 0>;
        const int c = arr / LEVELS, l = arr - c * LEVELS;
        double2* a = spec + arr * M;
        // the folded, twisted digits go to this thread's own pass-0 slots first (one at a
        // time, to keep register pressure low), then come back as the pass's registers
#pragma unroll 1
        for (int k = 0; k < 8; ++k) {
            const int j = pidx<Q::LO>(t, k);
            uint32_t lo, hi;
            if (MODE == 0) {
                const uint32_t* pc = acc + c * N;
                lo = rot_at<N>(pc, j, ai) - pc[j];
                hi = rot_at<N>(pc, j + M, ai) - pc[j + M];
            } else {
                lo = src[c * N + j];
                hi = src[c * N + j + M];
            }
            a[swz(j)] = cmul(make_double2((double)digit_of(lo, base_log, LEVELS, l),
                                          (double)digit_of(hi, base_log, LEVELS, l)),
                             __ldg(&twist[j]));
        }
        double2 v[8];
        get8<Q::LO>(v, a, t);
        dif<LOGM, Q::LO, Q::NST>(v, t, tw);
        put8<Q::LO>(a, v, t);
    }
    __syncthreads();
    fwd_rest<LOGM, 1>(spec + arr * M, t, true, tw);
    // multiply-accumulate fused into inverse pass NP-1 (threads of the two outputs)
    const bool inv = threadIdx.x < 2 * TPA;
    const int oc = inv ? arr : 0;
    {
        using Q = PassOf<LOGM, NP - 1>;
        if (inv) {
            double2* o = outs + oc * M;
            // products go to this thread's own slots first (one element at a time)
#pragma unroll 1
            for (int k = 0; k < 8; ++k) {
                const int f = pidx<Q::LO>(t, k);
                double2 acc2 = make_double2(0.0, 0.0);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const double2 kv = __ldg(&key[(r * 2 + oc) * M + k * TPA + t]);
                    const double2 dv = spec[r * M + swz(f)];
                    acc2.x = __fma_rn(dv.x, kv.x, __fma_rn(-dv.y, kv.y, acc2.x));
                    acc2.y = __fma_rn(dv.x, kv.y, __fma_rn(dv.y, kv.x, acc2.y));
                }
                o[swz(f)] = acc2;
            }
            double2 v[8];
            get8<Q::LO>(v, o, t);
            dit<LOGM, Q::LO, Q::NST>(v, t, tw);
            put8<Q::LO>(o, v, t);
        }
        __syncthreads();
    }
    inv_rest<LOGM, NP - 2>(outs + oc * M, t, inv, tw);
    // inverse pass 0: untwist, unfold, round (element j = t + k M/8)
    {
        using Q = PassOf<LOGM, 0>;
        double worst = 0.0;
        if (inv) {
            double2 v[8];
            get8<Q::LO>(v, outs + oc * M, t);
            dit<LOGM, Q::LO, Q::NST>(v, t, tw);
            const double inv_m = 1.0 / (double)M;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = pidx<Q::LO>(t, k);
                const double2 z = cmulc(v[k], __ldg(&twist[j]));
                const double re = z.x * inv_m, im = z.y * inv_m;
                const long long lo = __double2ll_rn(re), hi = __double2ll_rn(im);
                if (MODE == 0) {
                    acc[oc * N + j] += (uint32_t)lo;
                    acc[oc * N + j + M] += (uint32_t)hi;
                } else {
                    dst[oc * N + j] = (uint32_t)lo;
                    dst[oc * N + j + M] = (uint32_t)hi;
                    worst = fmax(worst, fmax(fabs(re - (double)lo), fabs(im - (double)hi)));
                }
            }
        }
        if (MODE == 1) {
            // block maximum through the spectra buffer (no longer needed)
            double* red = reinterpret_cast<double*>(spec);
            __syncthreads();
            red[threadIdx.x] = worst;
            __syncthreads();
            if (threadIdx.x == 0) {
                double m = 0.0;
                for (int i = 0; i < (int)blockDim.x; ++i) m = fmax(m, red[i]);
                *frac = m;
            }
        }
        __syncthreads();
    }
}

// CTAs per SM the register budget is sized for (about 64K / (threads x 2) registers
// per thread bounds the allocation the compiler may use)
template <int LOGM, int LEVELS>
struct BootMinCtas {
    static constexpr int threads = 2 * LEVELS * (1 << LOGM) / 8;
    static constexpr int value = threads >= 512 ? 1 : (threads >= 256 ? 2 : 4);
};

// Blind rotation + sample extraction of B LWEs (in: [B][n+1], mask then body) into
// out [B][N+1] (extracted mask, body).  bsk_f: [n][2 levels][2][M] spectra in key order.
// Block: 2 levels x M/8 threads; persistent over the LWEs.
template <int LOGM, int LEVELS>
__global__ void __launch_bounds__(2 * LEVELS * (1 << LOGM) / 8, BootMinCtas<LOGM, LEVELS>::value) k_cggi_fft_bootstrap(
    uint32_t* __restrict__ out, const uint32_t* __restrict__ in, long long B, const double2* __restrict__ bsk_f,
    const uint32_t* __restrict__ tv, int n, int base_log, uint32_t offset, const double2* __restrict__ g_tw,
    const double2* __restrict__ g_twist) {
    constexpr int M = 1 << LOGM, N = 2 * M, R = 2 * LEVELS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    double2* spec = reinterpret_cast<double2*>(acc + 2 * N);
    double2* outs = spec + R * M;
    constexpr int logN2 = LOGM + 2;
    for (long long lwe = blockIdx.x; lwe < B; lwe += gridDim.x) {
        const uint32_t* a = in + lwe * (long long)(n + 1);
        const int rb = modswitch(a[n] + offset, logN2);
        const int e0 = (2 * N - rb) & (2 * N - 1);
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            acc[k] = 0;
            acc[N + k] = rot_at<N>(tv, k, e0);
        }
        __syncthreads();
        for (int i = 0; i < n; ++i) {
            const int ai = modswitch(__ldg(a + i), logN2);
            ext_product<LOGM, LEVELS, 0>(acc, spec, outs, bsk_f + (long long)i * R * 2 * M, ai, base_log, nullptr,
                                         nullptr, nullptr, g_tw, g_twist);
        }
        uint32_t* o = out + lwe * (long long)(N + 1);
        for (int k = threadIdx.x; k < N; k += blockDim.x) o[k] = k == 0 ? acc[0] : (uint32_t)(0u - acc[N - k]);
        if (threadIdx.x == 0) o[N] = acc[N];
        __syncthreads();
    }
}

// out[B][2N] = ExtProd(ggsw_f, c[B][2N]) rounded; frac[b] = largest distance of an
// unrounded coefficient to its integer.  Same code path as a blind-rotation step.
template <int LOGM, int LEVELS>
__global__ void __launch_bounds__(2 * LEVELS * (1 << LOGM) / 8) k_cggi_fft_extprod(
    uint32_t* __restrict__ out, const uint32_t* __restrict__ c, const double2* __restrict__ ggsw_f, int base_log,
    const double2* __restrict__ g_tw, const double2* __restrict__ g_twist, double* __restrict__ frac) {
    constexpr int M = 1 << LOGM, N = 2 * M, R = 2 * LEVELS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    double2* spec = reinterpret_cast<double2*>(acc + 2 * N);
    double2* outs = spec + R * M;
    double dummy;
    ext_product<LOGM, LEVELS, 1>(acc, spec, outs, ggsw_f, 0, base_log, c + (long long)blockIdx.x * 2 * N,
                                 out + (long long)blockIdx.x * 2 * N, frac ? frac + blockIdx.x : &dummy, g_tw,
                                 g_twist);
}

// Spectra of rows of N signed 32-bit coefficients (torus values read as int32), in key
// order: out[r][k * M/8 + t] = spectrum element 8 t + k.  One block of M/8 threads per row.
template <int LOGM>
__global__ void __launch_bounds__((1 << LOGM) / 8) k_rows_to_fourier(double2* __restrict__ outp,
                                                                   const uint32_t* __restrict__ rows,
                                                                   const double2* __restrict__ g_tw,
                                                                   const double2* __restrict__ g_twist) {
    constexpr int M = 1 << LOGM, TPA = M / 8, NP = Passes<LOGM>::count;
    __shared__ double2 x[M];
    const int t = threadIdx.x;
    const uint32_t* p = rows + (long long)blockIdx.x * 2 * M;
    {
        using Q = PassOf<LOGM, 0>;
        double2 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int j = pidx<Q::LO>(t, k);
            v[k] = cmul(make_double2((double)(int32_t)p[j], (double)(int32_t)p[j + M]), __ldg(&g_twist[j]));
        }
        dif<LOGM, Q::LO, Q::NST>(v, t, g_tw);
        put8<Q::LO>(x, v, t);
    }
    __syncthreads();
    fwd_rest<LOGM, 1>(x, t, true, g_tw);
    using QL = PassOf<LOGM, NP - 1>;
    double2* o = outp + (long long)blockIdx.x * M;
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k * TPA + t] = x[swz(pidx<QL::LO>(t, k))];
}

// LWE key switch: out[b] = (0, in[b].body) - sum_{j,l} d_{b,j,l} KSK[j][l], digits of
// in[b].mask[j] (base 2^kb, kt levels).  CTA: KS_LWES LWEs x KS_COLS output columns;
// every key row is read once per CTA and reused for its KS_LWES LWEs.
constexpr int KS_LWES = 32;
constexpr int KS_COLS = 128;
constexpr int KS_J = 16;  // mask coefficients decomposed per round

__global__ void __launch_bounds__(KS_COLS) k_cggi_keyswitch(uint32_t* __restrict__ out, const uint32_t* __restrict__ in,
                                                            long long B, const uint32_t* __restrict__ ksk, int Nin,
                                                            int n, int base_log, int levels) {
    __shared__ int8_t dig[KS_J][kMaxLevels * 4][KS_LWES];  // levels <= 16
    const long long b0 = (long long)blockIdx.y * KS_LWES;
    const int col = blockIdx.x * KS_COLS + threadIdx.x;
    uint32_t accv[KS_LWES];
#pragma unroll
    for (int t = 0; t < KS_LWES; ++t) accv[t] = 0;
    for (int j0 = 0; j0 < Nin; j0 += KS_J) {
        // decompose KS_J x KS_LWES mask values
        for (int e = threadIdx.x; e < KS_J * KS_LWES; e += KS_COLS) {
            const int jj = e / KS_LWES, t = e - jj * KS_LWES;
            const long long b = b0 + t;
            uint32_t v = 0;
            if (b < B && j0 + jj < Nin) v = in[b * (Nin + 1) + j0 + jj];
            const int total = base_log * levels;
            uint64_t r = ((uint64_t)v + (1ULL << (31 - total))) >> (32 - total);
            r &= total >= 32 ? 0xFFFFFFFFULL : ((1ULL << total) - 1);
            const int half = 1 << (base_log - 1), full = 1 << base_log;
            for (int l = levels - 1; l >= 0; --l) {
                int x = (int)(r & (uint64_t)(full - 1));
                r >>= base_log;
                if (x >= half) {
                    x -= full;
                    r += 1;
                }
                dig[jj][l][t] = (int8_t)x;
            }
        }
        __syncthreads();
        if (col <= n) {
            for (int jj = 0; jj < KS_J && j0 + jj < Nin; ++jj)
                for (int l = 0; l < levels; ++l) {
                    const uint32_t kv = __ldg(ksk + ((long long)(j0 + jj) * levels + l) * (n + 1) + col);
#pragma unroll
                    for (int t = 0; t < KS_LWES; ++t) accv[t] -= (uint32_t)(int)dig[jj][l][t] * kv;
                }
        }
        __syncthreads();
    }
    if (col <= n) {
#pragma unroll
        for (int t = 0; t < KS_LWES; ++t) {
            const long long b = b0 + t;
            if (b >= B) break;
            uint32_t v = accv[t];
            if (col == n) v += in[b * (Nin + 1) + Nin];
            out[b * (n + 1) + col] = v;
        }
    }
}

bool check_shape(int N, int levels, int base_log, const char* where) {
    if (N != 512 && N != 1024 && N != 2048) {
        set_error(where, "N must be 512, 1024 or 2048");
        return false;
    }
    if (levels < 1 || levels > kMaxLevels || base_log < 1 || base_log * levels > 32) {
        set_error(where, "gadget needs 1..4 levels and base_log * levels <= 32");
        return false;
    }
    return true;
}

template <int LOGM, int LEVELS>
int launch_bootstrap_t(uint32_t* out, const uint32_t* in, long long B, const double2* bsk_f, const uint32_t* tv,
                       int n, int base_log, uint32_t offset, const FourierTables* ft, cudaStream_t st) {
    constexpr int THREADS = 2 * LEVELS * (1 << LOGM) / 8;
    const size_t smem = Smem<(2 << LOGM)>::bytes(LEVELS);
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_bootstrap<LOGM, LEVELS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem);
    if (e) return e;
    int per_sm = 0;
    e = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cggi_fft_bootstrap<LOGM, LEVELS>, THREADS, smem);
    if (e) return e;
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sm_count();
    if (grid > B) grid = B;
    k_cggi_fft_bootstrap<LOGM, LEVELS><<<(unsigned)grid, THREADS, smem, st>>>(out, in, B, bsk_f, tv, n, base_log, offset,
                                                                            ft->d_tw, ft->d_twist);
    note_launch();
    return (int)cudaGetLastError();
}

template <int LOGM, int LEVELS>
int launch_extprod_t(uint32_t* out, const uint32_t* c, long long B, const double2* ggsw_f, int base_log,
                     const FourierTables* ft, double* frac, cudaStream_t st) {
    constexpr int THREADS = 2 * LEVELS * (1 << LOGM) / 8;
    const size_t smem = Smem<(2 << LOGM)>::bytes(LEVELS);
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_extprod<LOGM, LEVELS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem);
    if (e) return e;
    k_cggi_fft_extprod<LOGM, LEVELS><<<(unsigned)B, THREADS, smem, st>>>(out, c, ggsw_f, base_log, ft->d_tw,
                                                                       ft->d_twist, frac);
    note_launch();
    return (int)cudaGetLastError();
}

// (N, levels) -> template instance
template <template <int, int> class F, typename... A>
int dispatch_nl(int N, int levels, A... args) {
    const int logm = N == 512 ? 8 : N == 1024 ? 9 : 10;
    switch (logm * 8 + levels) {
        case 8 * 8 + 1: return F<8, 1>::run(args...);
        case 8 * 8 + 2: return F<8, 2>::run(args...);
        case 8 * 8 + 3: return F<8, 3>::run(args...);
        case 8 * 8 + 4: return F<8, 4>::run(args...);
        case 9 * 8 + 1: return F<9, 1>::run(args...);
        case 9 * 8 + 2: return F<9, 2>::run(args...);
        case 9 * 8 + 3: return F<9, 3>::run(args...);
        case 9 * 8 + 4: return F<9, 4>::run(args...);
        case 10 * 8 + 1: return F<10, 1>::run(args...);
        case 10 * 8 + 2: return F<10, 2>::run(args...);
        case 10 * 8 + 3: return F<10, 3>::run(args...);
        default: return F<10, 4>::run(args...);
    }
}

template <int LOGM, int LEVELS>
struct BootstrapF {
    template <typename... A>
    static int run(A... a) { return launch_bootstrap_t<LOGM, LEVELS>(a...); }
};
template <int LOGM, int LEVELS>
struct ExtprodF {
    template <typename... A>
    static int run(A... a) { return launch_extprod_t<LOGM, LEVELS>(a...); }
};

int launch_to_fourier(int N, double2* outp, const uint32_t* rows, long long count, const FourierTables* ft,
                      cudaStream_t st) {
    for (long long off = 0; off < count; off += 65535LL * 16) {
        const long long m = count - off < 65535LL * 16 ? count - off : 65535LL * 16;
        switch (N) {
            case 512: k_rows_to_fourier<8><<<(unsigned)m, 32, 0, st>>>(outp + off * 256, rows + off * 512, ft->d_tw, ft->d_twist); break;
            case 1024: k_rows_to_fourier<9><<<(unsigned)m, 64, 0, st>>>(outp + off * 512, rows + off * 1024, ft->d_tw, ft->d_twist); break;
            default: k_rows_to_fourier<10><<<(unsigned)m, 128, 0, st>>>(outp + off * 1024, rows + off * 2048, ft->d_tw, ft->d_twist); break;
        }
        note_launch();
        const int e = (int)cudaGetLastError();
        if (e) return e;
    }
    return 0;
}

}  // namespace

}  // namespace vc

using namespace vc;

extern "C" {

int vfhe_cuda_cggi_fft_to_fourier(double* d_out, const uint32_t* d_rows, uint64_t count, uint32_t N, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_cggi_fft_to_fourier";
    if (!check_shape((int)N, 1, 1, where)) return 1;
    const FourierTables* ft = fourier_tables((int)N);
    if (!ft) return check_cuda(cudaErrorMemoryAllocation, where) ? 0 : 1;
    const int e = launch_to_fourier((int)N, (double2*)d_out, d_rows, (long long)count, ft, (cudaStream_t)stream);
    return check_cuda(e, where) ? 0 : 1;
}

int vfhe_cuda_cggi_fft_bootstrap_batch(uint32_t* d_out, const uint32_t* d_in, uint64_t batch, const double* d_bsk_f,
                                       const uint32_t* d_tv, uint32_t n, uint32_t N, uint32_t base_log, uint32_t levels,
                                       uint32_t torus_base, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_cggi_fft_bootstrap_batch";
    if (!check_shape((int)N, (int)levels, (int)base_log, where)) return 1;
    if (n == 0 || torus_base == 0 || batch == 0) {
        set_error(where, "need n > 0, torus_base > 0 and a nonempty batch");
        return 1;
    }
    const FourierTables* ft = fourier_tables((int)N);
    if (!ft) return check_cuda(cudaErrorMemoryAllocation, where) ? 0 : 1;
    const uint32_t offset = (uint32_t)((1ULL << 32) / (4ULL * torus_base));
    const int e = dispatch_nl<BootstrapF>((int)N, (int)levels, d_out, d_in, (long long)batch, (const double2*)d_bsk_f,
                                          d_tv, (int)n, (int)base_log, offset, ft, (cudaStream_t)stream);
    return check_cuda(e, where) ? 0 : 1;
}

int vfhe_cuda_cggi_fft_keyswitch_batch(uint32_t* d_out, const uint32_t* d_in, uint64_t batch, const uint32_t* d_ksk,
                                       uint32_t N, uint32_t n, uint32_t base_log, uint32_t levels, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_cggi_fft_keyswitch_batch";
    if (base_log < 1 || levels < 1 || levels > 16 || base_log * levels > 32 || n == 0 || N == 0 || batch == 0) {
        set_error(where, "need 1..16 levels, base_log * levels <= 32, n, N > 0");
        return 1;
    }
    const dim3 grid((n + 1 + KS_COLS - 1) / KS_COLS, (unsigned)((batch + KS_LWES - 1) / KS_LWES));
    if (grid.y > 65535) {
        set_error(where, "batch too large (at most 65535 x 32)");
        return 1;
    }
    k_cggi_keyswitch<<<grid, KS_COLS, 0, (cudaStream_t)stream>>>(d_out, d_in, (long long)batch, d_ksk, (int)N, (int)n,
                                                                 (int)base_log, (int)levels);
    note_launch();
    return check_cuda(cudaGetLastError(), where) ? 0 : 1;
}

int vfhe_cuda_cggi_fft_external_product(uint32_t* d_out, const uint32_t* d_c, uint64_t batch, const double* d_ggsw_f,
                                        uint32_t N, uint32_t base_log, uint32_t levels, double* d_frac,
                                        void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_cggi_fft_external_product";
    if (!check_shape((int)N, (int)levels, (int)base_log, where)) return 1;
    if (batch == 0 || batch > 65535) {
        set_error(where, "batch must be in [1, 65535]");
        return 1;
    }
    const FourierTables* ft = fourier_tables((int)N);
    if (!ft) return check_cuda(cudaErrorMemoryAllocation, where) ? 0 : 1;
    const int e = dispatch_nl<ExtprodF>((int)N, (int)levels, d_out, d_c, (long long)batch, (const double2*)d_ggsw_f,
                                        (int)base_log, ft, d_frac, (cudaStream_t)stream);
    return check_cuda(e, where) ? 0 : 1;
}

}  // extern "C"
