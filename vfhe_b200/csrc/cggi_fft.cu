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

// In-place forward DIF FFT (kernel e^{+2 pi i/M}) of `count` arrays of M points at
// x + a * stride; THREADS threads, one butterfly per thread per array per stage.
template <int M, int THREADS>
__device__ __forceinline__ void fft_fwd(double2* x, int count, int stride, const double2* tw) {
    for (int h = M / 2; h >= 1; h >>= 1) {
        for (int bf = threadIdx.x; bf < M / 2 * count; bf += THREADS) {
            const int a = bf / (M / 2), r = bf - a * (M / 2);
            const int grp = r / h, j = r - grp * h;
            const int i0 = grp * 2 * h + j;
            double2* y = x + a * stride;
            const double2 u = y[i0], v = y[i0 + h];
            y[i0] = make_double2(u.x + v.x, u.y + v.y);
            y[i0 + h] = cmul(make_double2(u.x - v.x, u.y - v.y), tw[j * (M / (2 * h))]);
        }
        __syncthreads();
    }
}

// In-place inverse DIT FFT (kernel e^{-2 pi i/M}, no 1/M) of `count` arrays.
template <int M, int THREADS>
__device__ __forceinline__ void fft_inv(double2* x, int count, int stride, const double2* tw) {
    for (int h = 1; h <= M / 2; h <<= 1) {
        for (int bf = threadIdx.x; bf < M / 2 * count; bf += THREADS) {
            const int a = bf / (M / 2), r = bf - a * (M / 2);
            const int grp = r / h, j = r - grp * h;
            const int i0 = grp * 2 * h + j;
            double2* y = x + a * stride;
            const double2 u = y[i0], v = cmulc(y[i0 + h], tw[j * (M / (2 * h))]);
            y[i0] = make_double2(u.x + v.x, u.y + v.y);
            y[i0 + h] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

// signed digits of v rounded to its top base_log * levels bits (digit 0 most significant)
__device__ __forceinline__ void decompose(int (&d)[kMaxLevels], uint32_t v, int base_log, int levels) {
    const int total = base_log * levels;
    uint64_t r = ((uint64_t)v + (1ULL << (31 - total))) >> (32 - total);
    r &= total >= 32 ? 0xFFFFFFFFULL : ((1ULL << total) - 1);
    const int half = 1 << (base_log - 1), full = 1 << base_log;
#pragma unroll
    for (int l = kMaxLevels - 1; l >= 0; --l) {
        if (l >= levels) continue;
        int x = (int)(r & (uint64_t)(full - 1));
        r >>= base_log;
        if (x >= half) {
            x -= full;
            r += 1;
        }
        d[l] = x;
    }
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

template <int N>
struct Smem {
    static constexpr int M = N / 2;
    // acc[2][N] uint32 | spec[2 L][M] double2 | outs[2][M] double2 | tw[M/2] | twist[M]
    static constexpr size_t bytes(int levels) {
        return sizeof(uint32_t) * 2 * N + sizeof(double2) * (2 * levels * M + 2 * M + M / 2 + M);
    }
};

// Blind rotation + sample extraction of B LWEs (in: [B][n+1], mask then body) into
// out [B][N+1] (extracted mask, body).  bsk_f: [n][2 levels][2][M] spectra.
template <int N, int THREADS>
__global__ void __launch_bounds__(THREADS) k_cggi_fft_bootstrap(uint32_t* __restrict__ out,
                                                                const uint32_t* __restrict__ in, long long B,
                                                                const double2* __restrict__ bsk_f,
                                                                const uint32_t* __restrict__ tv, int n, int base_log,
                                                                int levels, uint32_t offset,
                                                                const double2* __restrict__ g_tw,
                                                                const double2* __restrict__ g_twist) {
    constexpr int M = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    double2* spec = reinterpret_cast<double2*>(acc + 2 * N);
    double2* outs = spec + 2 * levels * M;
    double2* tw = outs + 2 * M;
    double2* twist = tw + M / 2;
    for (int k = threadIdx.x; k < M / 2; k += THREADS) tw[k] = g_tw[k];
    for (int k = threadIdx.x; k < M; k += THREADS) twist[k] = g_twist[k];
    int logN2 = 0;
    while ((1 << logN2) < 2 * N) ++logN2;
    const double inv_m = 1.0 / (double)M;
    const int R = 2 * levels;
    __syncthreads();

    for (long long lwe = blockIdx.x; lwe < B; lwe += gridDim.x) {
        const uint32_t* a = in + lwe * (long long)(n + 1);
        const int rb = modswitch(a[n] + offset, logN2);
        const int e0 = (2 * N - rb) & (2 * N - 1);
        for (int k = threadIdx.x; k < N; k += THREADS) {
            acc[k] = 0;
            acc[N + k] = rot_at<N>(tv, k, e0);
        }
        __syncthreads();
        for (int i = 0; i < n; ++i) {
            const int ai = modswitch(__ldg(a + i), logN2);
            // digits of (acc X^ai - acc), folded and twisted, into spec[c * levels + l]
            for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
                const int c = jj / M, j = jj - c * M;
                const uint32_t* p = acc + c * N;
                const uint32_t lo = rot_at<N>(p, j, ai) - p[j];
                const uint32_t hi = rot_at<N>(p, j + M, ai) - p[j + M];
                int dl[kMaxLevels], dh[kMaxLevels];
                decompose(dl, lo, base_log, levels);
                decompose(dh, hi, base_log, levels);
                const double2 w = twist[j];
                for (int l = 0; l < levels; ++l)
                    spec[(c * levels + l) * M + j] = cmul(make_double2((double)dl[l], (double)dh[l]), w);
            }
            __syncthreads();
            fft_fwd<M, THREADS>(spec, R, M, tw);
            // multiply-accumulate against step i's key spectra
            const double2* key = bsk_f + (long long)i * R * 2 * M;
            for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
                const int oc = jj / M, f = jj - oc * M;
                double2 s = make_double2(0.0, 0.0);
                for (int r = 0; r < R; ++r) {
                    const double2 kv = __ldg(key + ((long long)r * 2 + oc) * M + f);
                    const double2 dv = spec[r * M + f];
                    s.x = __fma_rn(dv.x, kv.x, __fma_rn(-dv.y, kv.y, s.x));
                    s.y = __fma_rn(dv.x, kv.y, __fma_rn(dv.y, kv.x, s.y));
                }
                outs[oc * M + f] = s;
            }
            __syncthreads();
            fft_inv<M, THREADS>(outs, 2, M, tw);
            // untwist, unfold, round and add
            for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
                const int oc = jj / M, j = jj - oc * M;
                const double2 z = cmulc(outs[oc * M + j], twist[j]);
                const long long lo = __double2ll_rn(z.x * inv_m);
                const long long hi = __double2ll_rn(z.y * inv_m);
                acc[oc * N + j] += (uint32_t)lo;
                acc[oc * N + j + M] += (uint32_t)hi;
            }
            __syncthreads();
        }
        uint32_t* o = out + lwe * (long long)(N + 1);
        for (int k = threadIdx.x; k < N; k += THREADS) o[k] = k == 0 ? acc[0] : (uint32_t)(0u - acc[N - k]);
        if (threadIdx.x == 0) o[N] = acc[N];
        __syncthreads();
    }
}

// Spectra of rows of N signed 32-bit coefficients (torus values read as int32):
// out[r][M] for r < rows.  One CTA per row.
template <int N, int THREADS>
__global__ void __launch_bounds__(THREADS) k_rows_to_fourier(double2* __restrict__ outp,
                                                             const uint32_t* __restrict__ rows,
                                                             const double2* __restrict__ g_tw,
                                                             const double2* __restrict__ g_twist) {
    constexpr int M = N / 2;
    __shared__ double2 x[M];
    __shared__ double2 tw[M / 2];
    for (int k = threadIdx.x; k < M / 2; k += THREADS) tw[k] = g_tw[k];
    const uint32_t* p = rows + (long long)blockIdx.x * N;
    for (int j = threadIdx.x; j < M; j += THREADS)
        x[j] = cmul(make_double2((double)(int32_t)p[j], (double)(int32_t)p[j + M]), g_twist[j]);
    __syncthreads();
    fft_fwd<M, THREADS>(x, 1, M, tw);
    for (int j = threadIdx.x; j < M; j += THREADS) outp[(long long)blockIdx.x * M + j] = x[j];
}

// out[B][2N] = ExtProd(ggsw_f, c[B][2N]) rounded, for measuring FFT error: same code
// path as one CMUX step with a fixed difference.
template <int N, int THREADS>
__global__ void __launch_bounds__(THREADS) k_cggi_fft_extprod(uint32_t* __restrict__ out,
                                                              const uint32_t* __restrict__ c,
                                                              const double2* __restrict__ ggsw_f, int base_log,
                                                              int levels, const double2* __restrict__ g_tw,
                                                              const double2* __restrict__ g_twist,
                                                              double* __restrict__ frac_err) {
    constexpr int M = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* spec = reinterpret_cast<double2*>(smem_raw);
    double2* outs = spec + 2 * levels * M;
    double2* tw = outs + 2 * M;
    double2* twist = tw + M / 2;
    const int R = 2 * levels;
    for (int k = threadIdx.x; k < M / 2; k += THREADS) tw[k] = g_tw[k];
    for (int k = threadIdx.x; k < M; k += THREADS) twist[k] = g_twist[k];
    __syncthreads();
    const uint32_t* cc = c + (long long)blockIdx.x * 2 * N;
    for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
        const int comp = jj / M, j = jj - comp * M;
        int dl[kMaxLevels], dh[kMaxLevels];
        decompose(dl, cc[comp * N + j], base_log, levels);
        decompose(dh, cc[comp * N + j + M], base_log, levels);
        for (int l = 0; l < levels; ++l)
            spec[(comp * levels + l) * M + j] = cmul(make_double2((double)dl[l], (double)dh[l]), twist[j]);
    }
    __syncthreads();
    fft_fwd<M, THREADS>(spec, R, M, tw);
    for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
        const int oc = jj / M, f = jj - oc * M;
        double2 s = make_double2(0.0, 0.0);
        for (int r = 0; r < R; ++r) {
            const double2 kv = ggsw_f[((long long)r * 2 + oc) * M + f];
            const double2 dv = spec[r * M + f];
            s.x = __fma_rn(dv.x, kv.x, __fma_rn(-dv.y, kv.y, s.x));
            s.y = __fma_rn(dv.x, kv.y, __fma_rn(dv.y, kv.x, s.y));
        }
        outs[oc * M + f] = s;
    }
    __syncthreads();
    fft_inv<M, THREADS>(outs, 2, M, tw);
    uint32_t* o = out + (long long)blockIdx.x * 2 * N;
    double worst = 0.0;
    for (int jj = threadIdx.x; jj < 2 * M; jj += THREADS) {
        const int oc = jj / M, j = jj - oc * M;
        const double2 z = cmulc(outs[oc * M + j], twist[j]);
        const double re = z.x / (double)M, im = z.y / (double)M;
        const double rr = rint(re), ri = rint(im);
        worst = fmax(worst, fmax(fabs(re - rr), fabs(im - ri)));
        o[oc * N + j] = (uint32_t)(long long)rr;
        o[oc * N + j + M] = (uint32_t)(long long)ri;
    }
    // per-row worst distance to the nearest integer (how close rounding came to failing)
    __shared__ double red[THREADS];
    red[threadIdx.x] = worst;
    __syncthreads();
    for (int s2 = THREADS / 2; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s2]);
        __syncthreads();
    }
    if (threadIdx.x == 0 && frac_err) frac_err[blockIdx.x] = red[0];
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

template <int N>
int launch_bootstrap(uint32_t* out, const uint32_t* in, long long B, const double2* bsk_f, const uint32_t* tv, int n,
                     int base_log, int levels, uint32_t offset, const FourierTables* ft, cudaStream_t st) {
    constexpr int THREADS = N / 4 < 128 ? 128 : N / 4;
    const size_t smem = Smem<N>::bytes(levels);
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_bootstrap<N, THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem);
    if (e) return e;
    int per_sm = 0;
    e = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cggi_fft_bootstrap<N, THREADS>, THREADS, smem);
    if (e) return e;
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sm_count();
    if (grid > B) grid = B;
    k_cggi_fft_bootstrap<N, THREADS><<<(unsigned)grid, THREADS, smem, st>>>(out, in, B, bsk_f, tv, n, base_log, levels,
                                                                          offset, ft->d_tw, ft->d_twist);
    note_launch();
    return (int)cudaGetLastError();
}

template <int N>
int launch_to_fourier(double2* outp, const uint32_t* rows, long long count, const FourierTables* ft, cudaStream_t st) {
    constexpr int THREADS = N / 4 < 128 ? 128 : N / 4;
    for (long long off = 0; off < count; off += 65535LL * 16) {
        const long long m = count - off < 65535LL * 16 ? count - off : 65535LL * 16;
        k_rows_to_fourier<N, THREADS><<<(unsigned)m, THREADS, 0, st>>>(outp + off * (N / 2), rows + off * N, ft->d_tw,
                                                                       ft->d_twist);
        note_launch();
        const int e = (int)cudaGetLastError();
        if (e) return e;
    }
    return 0;
}

template <int N>
int launch_extprod(uint32_t* out, const uint32_t* c, long long B, const double2* ggsw_f, int base_log, int levels,
                   const FourierTables* ft, double* frac, cudaStream_t st) {
    constexpr int THREADS = N / 4 < 128 ? 128 : N / 4;
    const size_t smem = sizeof(double2) * (2 * levels * (N / 2) + 2 * (N / 2) + N / 4 + N / 2);
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_extprod<N, THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem);
    if (e) return e;
    k_cggi_fft_extprod<N, THREADS><<<(unsigned)B, THREADS, smem, st>>>(out, c, ggsw_f, base_log, levels, ft->d_tw,
                                                                       ft->d_twist, frac);
    note_launch();
    return (int)cudaGetLastError();
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
    cudaStream_t st = (cudaStream_t)stream;
    int e;
    switch (N) {
        case 512: e = launch_to_fourier<512>((double2*)d_out, d_rows, (long long)count, ft, st); break;
        case 1024: e = launch_to_fourier<1024>((double2*)d_out, d_rows, (long long)count, ft, st); break;
        default: e = launch_to_fourier<2048>((double2*)d_out, d_rows, (long long)count, ft, st); break;
    }
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
    cudaStream_t st = (cudaStream_t)stream;
    int e;
    switch (N) {
        case 512:
            e = launch_bootstrap<512>(d_out, d_in, (long long)batch, (const double2*)d_bsk_f, d_tv, (int)n,
                                      (int)base_log, (int)levels, offset, ft, st);
            break;
        case 1024:
            e = launch_bootstrap<1024>(d_out, d_in, (long long)batch, (const double2*)d_bsk_f, d_tv, (int)n,
                                       (int)base_log, (int)levels, offset, ft, st);
            break;
        default:
            e = launch_bootstrap<2048>(d_out, d_in, (long long)batch, (const double2*)d_bsk_f, d_tv, (int)n,
                                       (int)base_log, (int)levels, offset, ft, st);
            break;
    }
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
    cudaStream_t st = (cudaStream_t)stream;
    int e;
    switch (N) {
        case 512:
            e = launch_extprod<512>(d_out, d_c, (long long)batch, (const double2*)d_ggsw_f, (int)base_log,
                                    (int)levels, ft, d_frac, st);
            break;
        case 1024:
            e = launch_extprod<1024>(d_out, d_c, (long long)batch, (const double2*)d_ggsw_f, (int)base_log,
                                     (int)levels, ft, d_frac, st);
            break;
        default:
            e = launch_extprod<2048>(d_out, d_c, (long long)batch, (const double2*)d_ggsw_f, (int)base_log,
                                     (int)levels, ft, d_frac, st);
            break;
    }
    return check_cuda(e, where) ? 0 : 1;
}

}  // extern "C"
