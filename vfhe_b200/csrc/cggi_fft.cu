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

// Twiddles per stage and the twist zeta^j (j < M), per N.  The stage whose butterflies
// span 2^(b+1) points uses e^{2 pi i j / 2^(b+1)}, j < 2^b, stored contiguously at
// offset 2^b - 1 (M - 1 entries in all), so that the threads of a warp, whose j are
// consecutive or broadcast, read consecutive entries.
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
    std::vector<double2> tw(M), twist(M);
    const long double pi = 3.141592653589793238462643383279502884L;
    tw[M - 1] = make_double2(0.0, 0.0);  // padding
    for (int b = 0; (1 << b) < M; ++b)
        for (int j = 0; j < (1 << b); ++j) {
            const long double ang = 2.0L * pi * (long double)j / (long double)(2 << b);
            tw[(1 << b) - 1 + j] = make_double2((double)cosl(ang), (double)sinl(ang));
        }
    for (int j = 0; j < M; ++j) {
        const long double ang = pi * (long double)j / (long double)N;
        twist[j] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    FourierTables t;
    t.N = N;
    if (cudaMalloc(&t.d_tw, sizeof(double2) * M) != cudaSuccess ||
        cudaMalloc(&t.d_twist, sizeof(double2) * M) != cudaSuccess ||
        cudaMemcpy(t.d_tw, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(t.d_twist, twist.data(), sizeof(double2) * M, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess)  // the uploads have landed before other streams read them
        return nullptr;
    g_ft.push_back(t);
    return &g_ft.back();
}

// Table loads issued where they stand: ordinary (coherent) loads that neither the
// compiler nor the assembler moves across the exchange barriers.  Through the read-only
// path they count as invariant, and every level's key and twiddle loads of a step would
// be hoisted to its top, keeping well over a hundred values live in registers.
__device__ __forceinline__ double2 ld_table(const double2* p) {
    double2 v;
    asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -a.y * b.y), __fma_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(__fma_rn(a.x, b.x, a.y * b.y), __fma_rn(a.y, b.x, -a.x * b.y));
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
__device__ __forceinline__ void dif(double2 (&v)[8], int t, const double2* tw) {
#pragma unroll
    for (int s = NST - 1; s >= 0; --s) {
        const int bit = 1 << s;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & bit) continue;
            const double2 u = v[k], x = v[k | bit];
            v[k] = make_double2(u.x + x.x, u.y + x.y);
            if (LO + s == 0) {  // twiddle index 0: the factor is exactly 1
                v[k | bit] = make_double2(u.x - x.x, u.y - x.y);
            } else {
                const int j = pidx<LO>(t, k) & ((1 << (LO + s)) - 1);
                v[k | bit] = cmul(make_double2(u.x - x.x, u.y - x.y), tw[(1 << (LO + s)) - 1 + j]);
            }
        }
    }
}

// decimation-in-time stages of one pass (kernel e^{-2 pi i / M})
template <int LOGM, int LO, int NST>
__device__ __forceinline__ void dit(double2 (&v)[8], int t, const double2* tw) {
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        const int bit = 1 << s;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & bit) continue;
            double2 x = v[k | bit];
            if (LO + s != 0) {  // (twiddle index 0 is exactly 1)
                const int j = pidx<LO>(t, k) & ((1 << (LO + s)) - 1);
                x = cmulc(x, tw[(1 << (LO + s)) - 1 + j]);
            }
            const double2 u = v[k];
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

// ---- group-split external product
//
// The GLWE of one LWE is handled by two groups of TPA = M/8 threads, group c owning
// component c: it forms the LEVELS digit polynomials of component c (one after another,
// each transformed in registers with exchanges through the group's own two shared
// buffers under a named barrier of TPA threads), and multiplies each spectrum with the
// GGSW rows (c, level) of both outputs, keeping the two partial sums in registers.  The
// groups then swap the partial sums of each other's output through shared memory (the
// only point where they meet) and each runs the inverse transform of output c, adding
// the rounded result into its own accumulator component.  Every thread works in every
// phase, and a group never waits for the other group except at the swap.

__device__ __forceinline__ void group_bar(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Signed gadget digits without a per-digit carry loop: adding B/2 to every base-B
// digit of the rounded value r (mod B^levels) makes digit l of the sum, minus B/2, the
// balanced digit in [-B/2, B/2) (the representation is unique, so it equals the
// carry-propagating decomposition).  Digit 0 is the most significant.
struct Gadget {
    int total;       // base_log * levels
    int base_log;
    uint32_t mask;   // 2^total - 1
    uint32_t half;   // sum over digits of B/2 at each digit position
};

__host__ __device__ inline Gadget make_gadget(int base_log, int levels) {
    Gadget g;
    g.total = base_log * levels;
    g.base_log = base_log;
    g.mask = g.total >= 32 ? 0xFFFFFFFFu : ((1u << g.total) - 1u);
    g.half = 0;
    for (int l = 0; l < levels; ++l) g.half += 1u << (base_log * l + base_log - 1);
    return g;
}

__device__ __forceinline__ uint32_t gadget_prepare(uint32_t v, const Gadget& g) {
    const uint32_t r = g.total >= 32 ? v : (uint32_t)(((uint64_t)v + (1ULL << (31 - g.total))) >> (32 - g.total));
    return (r + g.half) & g.mask;
}

template <int LEVELS>
__device__ __forceinline__ double gadget_digit(uint32_t prepared, const Gadget& g, int l) {
    const int sh = g.base_log * (LEVELS - 1 - l);
    const int d = (int)((prepared >> sh) & ((1u << g.base_log) - 1u)) - (1 << (g.base_log - 1));
    return (double)d;
}

// Exchange through buffer `b`: registers in the layout of pass PFROM, out in pass PTO's.
template <int LOGM, int PFROM, int PTO>
__device__ __forceinline__ void exchange(double2 (&v)[8], double2* b, int t, int bar) {
    put8<PassOf<LOGM, PFROM>::LO>(b, v, t);
    group_bar(bar, (1 << LOGM) / 8);
    get8<PassOf<LOGM, PTO>::LO>(v, b, t);
}

// forward passes P .. count-1, registers holding pass P-1's output; exchange e uses buffer e & 1
template <int LOGM, int P, int E>
__device__ __forceinline__ void group_fwd(double2 (&v)[8], double2* bufs, int t, int bar, const double2* tw) {
    if constexpr (P < Passes<LOGM>::count) {
        exchange<LOGM, P - 1, P>(v, bufs + (E & 1) * (1 << LOGM), t, bar);
        dif<LOGM, PassOf<LOGM, P>::LO, PassOf<LOGM, P>::NST>(v, t, tw);
        group_fwd<LOGM, P + 1, E + 1>(v, bufs, t, bar, tw);
    }
}

// inverse passes P down to 0, registers holding pass P+1's output
template <int LOGM, int P, int E>
__device__ __forceinline__ void group_inv(double2 (&v)[8], double2* bufs, int t, int bar, const double2* tw) {
    if constexpr (P >= 0) {
        exchange<LOGM, P + 1, P>(v, bufs + (E & 1) * (1 << LOGM), t, bar);
        dit<LOGM, PassOf<LOGM, P>::LO, PassOf<LOGM, P>::NST>(v, t, tw);
        group_inv<LOGM, P - 1, E + 1>(v, bufs, t, bar, tw);
    }
}

template <int LOGM, int LEVELS>
struct GroupSplit {
    static constexpr int M = 1 << LOGM, N = 2 * M, TPA = M / 8, THREADS = 2 * TPA;
    static constexpr int NP = Passes<LOGM>::count;
    static constexpr int FWD_EX = LEVELS * (NP - 1);  // exchanges of the forward transforms
    // acc[2][N] uint32 | bufs[2 groups][2][M] double2 | xbufs[2][M] double2 | twiddles[M]
    static constexpr size_t smem = sizeof(uint32_t) * 2 * N + sizeof(double2) * 7 * M;
    // resident blocks the register budget is sized for: about 168 registers a thread
    static constexpr int min_ctas = 65536 / (THREADS * 168) > 0 ? 65536 / (THREADS * 168) : 1;
};

// One external product on the block's GLWE, by group c (thread t of TPA).  Source
// (MODE 0): acc X^ai - acc from the block's accumulator; (MODE 1) the GLWE `src`.
// Result: MODE 0 adds the rounded output c into acc component c; MODE 1 writes it to
// dst and returns the largest distance of an unrounded coefficient to its integer.
// bufs: this group's two exchange buffers; xbufs: the two groups' receive buffers
// (xbufs + c M collects output c's share from the other group).  The caller has made
// the accumulator's last writes visible and the receive buffers free (__syncthreads).
template <int LOGM, int LEVELS, int MODE>
__device__ __forceinline__ double group_ext_product(uint32_t* acc, double2* bufs, double2* xbufs, int c, int t,
                                                    const double2* __restrict__ key, int ai, const Gadget& gd,
                                                    const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                    const double2* tw, const double2* __restrict__ twist) {
    using G = GroupSplit<LOGM, LEVELS>;
    constexpr int M = G::M, N = G::N, TPA = G::TPA, NP = G::NP;
    // Fresh copies of the thread coordinates: every shared-memory and table address of
    // the step derives from them, and without this the compiler hoists all of those
    // addresses out of the caller's step loop and keeps them live in registers.
    asm volatile("mov.b32 %0, %0;" : "+r"(t));
    asm volatile("mov.b32 %0, %0;" : "+r"(c));
    const int bar = 1 + c;
    // rounded, digit-prepared source coefficients j and j + M (j = k TPA + t: pass-0 layout)
    uint32_t plo[8], phi[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int j = k * TPA + t;
        uint32_t lo, hi;
        if (MODE == 0) {
            const uint32_t* pc = acc + c * N;
            lo = rot_at<N>(pc, j, ai) - pc[j];
            hi = rot_at<N>(pc, j + M, ai) - pc[j + M];
        } else {
            lo = src[c * N + j];
            hi = src[c * N + j + M];
        }
        plo[k] = gadget_prepare(lo, gd);
        phi[k] = gadget_prepare(hi, gd);
    }
    // output c's partial sum stays in registers; output 1 - c's goes straight into the
    // other group's receive buffer (same positions for every level, so no races)
    double2 pm[8];
    double2* give = xbufs + (1 - c) * M;
#pragma unroll
    for (int k = 0; k < 8; ++k) pm[k] = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < LEVELS; ++l) {
        double2 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            v[k] = cmul(make_double2(gadget_digit<LEVELS>(plo[k], gd, l), gadget_digit<LEVELS>(phi[k], gd, l)),
                        ld_table(&twist[k * TPA + t]));
        dif<LOGM, PassOf<LOGM, 0>::LO, PassOf<LOGM, 0>::NST>(v, t, tw);
        if (l == 0) group_fwd<LOGM, 1, 0>(v, bufs, t, bar, tw);
        else if (l == 1) group_fwd<LOGM, 1, (NP - 1)>(v, bufs, t, bar, tw);
        else if (l == 2) group_fwd<LOGM, 1, 2 * (NP - 1)>(v, bufs, t, bar, tw);
        else group_fwd<LOGM, 1, 3 * (NP - 1)>(v, bufs, t, bar, tw);
        // spectrum element 8 t + k meets key position k TPA + t (key order)
        const double2* km = key + (long long)((c * LEVELS + l) * 2 + c) * M;
        const double2* ko = key + (long long)((c * LEVELS + l) * 2 + (1 - c)) * M;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 ka = ld_table(&km[k * TPA + t]);
            pm[k].x = __fma_rn(v[k].x, ka.x, __fma_rn(-v[k].y, ka.y, pm[k].x));
            pm[k].y = __fma_rn(v[k].x, ka.y, __fma_rn(v[k].y, ka.x, pm[k].y));
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 kb = ld_table(&ko[k * TPA + t]);
            double2* g = give + swz(pidx<0>(t, k));
            const double2 o = l == 0 ? make_double2(0.0, 0.0) : *g;
            *g = make_double2(__fma_rn(v[k].x, kb.x, __fma_rn(-v[k].y, kb.y, o.x)),
                              __fma_rn(v[k].x, kb.y, __fma_rn(v[k].y, kb.x, o.y)));
        }
    }
    __syncthreads();  // both groups' contributions to each other's output are in place
    double2 v[8];
    {
        const double2* mine = xbufs + c * M;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 other = mine[swz(pidx<0>(t, k))];
            v[k] = make_double2(pm[k].x + other.x, pm[k].y + other.y);
        }
    }
    dit<LOGM, PassOf<LOGM, NP - 1>::LO, PassOf<LOGM, NP - 1>::NST>(v, t, tw);
    group_inv<LOGM, NP - 2, G::FWD_EX>(v, bufs, t, bar, tw);
    // untwist, unfold, round (element j = k TPA + t)
    const double inv_m = 1.0 / (double)M;
    double worst = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int j = k * TPA + t;
        const double2 z = cmulc(v[k], __ldg(&twist[j]));
        const double re = z.x * inv_m, im = z.y * inv_m;
        const long long lo = __double2ll_rn(re), hi = __double2ll_rn(im);
        if (MODE == 0) {
            acc[c * N + j] += (uint32_t)lo;
            acc[c * N + j + M] += (uint32_t)hi;
        } else {
            dst[c * N + j] = (uint32_t)lo;
            dst[c * N + j + M] = (uint32_t)hi;
            worst = fmax(worst, fmax(fabs(re - (double)lo), fabs(im - (double)hi)));
        }
    }
    return worst;
}

// Blind rotation + sample extraction of B LWEs (in: [B][n+1], mask then body) into
// out [B][N+1] (extracted mask, body).  bsk_f: [n][2 levels][2][M] spectra in key order.
// Block: two groups of M/8 threads (one per GLWE component); persistent over the LWEs.
template <int LOGM, int LEVELS>
__global__ void __launch_bounds__(GroupSplit<LOGM, LEVELS>::THREADS, GroupSplit<LOGM, LEVELS>::min_ctas)
    k_cggi_fft_bootstrap(uint32_t* __restrict__ out, const uint32_t* __restrict__ in, long long B,
                         const double2* __restrict__ bsk_f, const uint32_t* __restrict__ tv, int n, Gadget gd,
                         uint32_t offset, const double2* __restrict__ g_tw, const double2* __restrict__ g_twist) {
    using G = GroupSplit<LOGM, LEVELS>;
    constexpr int M = G::M, N = G::N, TPA = G::TPA, R = 2 * LEVELS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    double2* bufs_all = reinterpret_cast<double2*>(acc + 2 * N);
    const int c = threadIdx.x / TPA, t = threadIdx.x - c * TPA;
    double2* bufs = bufs_all + c * 2 * M;
    double2* xbufs = bufs_all + 4 * M;
    // the transforms' per-stage twiddles, read from shared memory (a warp's lookups are
    // consecutive or broadcast entries: one wavefront, against up to 16 L1 sectors)
    double2* stw = bufs_all + 6 * M;
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = g_tw[k];
    __syncthreads();
    constexpr int logN2 = LOGM + 2;
    for (long long lwe = blockIdx.x; lwe < B; lwe += gridDim.x) {
        const uint32_t* a = in + lwe * (long long)(n + 1);
        const int rb = modswitch(a[n] + offset, logN2);
        const int e0 = (2 * N - rb) & (2 * N - 1);
        for (int k = t; k < N; k += TPA) acc[c * N + k] = c == 0 ? 0u : rot_at<N>(tv, k, e0);
        for (int i = 0; i < n; ++i) {
            // accumulator writes visible; last step's receive-buffer reads done
            __syncthreads();
            const int ai = modswitch(__ldg(a + i), logN2);
            group_ext_product<LOGM, LEVELS, 0>(acc, bufs, xbufs, c, t, bsk_f + (long long)i * R * 2 * M, ai, gd,
                                               nullptr, nullptr, stw, g_twist);
        }
        group_bar(1 + c, TPA);
        uint32_t* o = out + lwe * (long long)(N + 1);
        if (c == 0) {
            for (int k = t; k < N; k += TPA) o[k] = k == 0 ? acc[0] : (uint32_t)(0u - acc[N - k]);
        } else if (t == 0) {
            o[N] = acc[N];
        }
        group_bar(1 + c, TPA);  // extraction reads done before the next LWE rewrites acc
    }
}

// out[B][2N] = ExtProd(ggsw_f, c[B][2N]) rounded; frac[b] = largest distance of an
// unrounded coefficient to its integer.  Same code path as a blind-rotation step.
template <int LOGM, int LEVELS>
__global__ void __launch_bounds__(GroupSplit<LOGM, LEVELS>::THREADS) k_cggi_fft_extprod(
    uint32_t* __restrict__ out, const uint32_t* __restrict__ c_in, const double2* __restrict__ ggsw_f, Gadget gd,
    const double2* __restrict__ g_tw, const double2* __restrict__ g_twist, double* __restrict__ frac) {
    using G = GroupSplit<LOGM, LEVELS>;
    constexpr int M = G::M, N = G::N, TPA = G::TPA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    double2* bufs_all = reinterpret_cast<double2*>(acc + 2 * N);
    const int c = threadIdx.x / TPA, t = threadIdx.x - c * TPA;
    double2* stw = bufs_all + 6 * M;
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = g_tw[k];
    __syncthreads();
    const double worst = group_ext_product<LOGM, LEVELS, 1>(
        acc, bufs_all + c * 2 * M, bufs_all + 4 * M, c, t, ggsw_f, 0, gd,
        c_in + (long long)blockIdx.x * 2 * N, out + (long long)blockIdx.x * 2 * N, stw, g_twist);
    // block maximum through the exchange buffers (no longer needed)
    double* red = reinterpret_cast<double*>(bufs_all);
    __syncthreads();
    red[threadIdx.x] = worst;
    __syncthreads();
    if (threadIdx.x == 0 && frac) {
        double m = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) m = fmax(m, red[i]);
        frac[blockIdx.x] = m;
    }
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
    using G = GroupSplit<LOGM, LEVELS>;
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_bootstrap<LOGM, LEVELS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)G::smem);
    if (e) return e;
    int per_sm = 0;
    e = (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cggi_fft_bootstrap<LOGM, LEVELS>, G::THREADS,
                                                           G::smem);
    if (e) return e;
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sm_count();
    if (grid > B) grid = B;
    k_cggi_fft_bootstrap<LOGM, LEVELS><<<(unsigned)grid, G::THREADS, G::smem, st>>>(
        out, in, B, bsk_f, tv, n, make_gadget(base_log, LEVELS), offset, ft->d_tw, ft->d_twist);
    note_launch();
    return (int)cudaGetLastError();
}

template <int LOGM, int LEVELS>
int launch_extprod_t(uint32_t* out, const uint32_t* c, long long B, const double2* ggsw_f, int base_log,
                     const FourierTables* ft, double* frac, cudaStream_t st) {
    using G = GroupSplit<LOGM, LEVELS>;
    int e = (int)cudaFuncSetAttribute(k_cggi_fft_extprod<LOGM, LEVELS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)G::smem);
    if (e) return e;
    k_cggi_fft_extprod<LOGM, LEVELS><<<(unsigned)B, G::THREADS, G::smem, st>>>(
        out, c, ggsw_f, make_gadget(base_log, LEVELS), ft->d_tw, ft->d_twist, frac);
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

namespace vc {
namespace {

// ---- torus key generation on the device (the big random material of the keys; the
// secret keys s and S are the caller's)
//
// Bootstrapping key: row (i, r), r = c levels + l, is a GLWE encryption of zero under
// S, (a, a S + e), with s_i 2^(32 - base_log (l + 1)) added to coefficient 0 of
// component c -- GGSW(s_i) in the layout vfhe_cuda_cggi_fft_bootstrap_batch reads.
// Key-switching key: row (j, l) is an LWE encryption under s of S_j 2^(32 - ks_base_log
// (l + 1)).  a is uniform over the torus, e a rounded Gaussian of width sigma 2^32.
// Randomness: the engine's ChaCha20 stream, uniform and Gaussian nonces, blocks counted
// from u0 / g0 per row.

__device__ __forceinline__ int32_t torus_gauss(const PrngKey& key, uint64_t counter, int k, double sigma32) {
    uint32_t blk[16];
    chacha20_block(key, counter, kStreamGaussian, blk);
    const double u1 = unit_open_low(block_u64(blk, 2 * (k & 3))), u2 = unit_closed_low(block_u64(blk, 2 * (k & 3) + 1));
    return (int32_t)(int64_t)llrint(sigma32 * sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
}

// one CTA of N threads per bootstrapping-key row; thread k computes coefficient k
__global__ void k_torus_bsk_rows(uint32_t* __restrict__ rows, const int32_t* __restrict__ s,
                                 const int32_t* __restrict__ S, int N, int levels, int base_log, double sigma32,
                                 const __grid_constant__ PrngKey key, uint64_t u0, uint64_t g0) {
    extern __shared__ uint32_t tsm[];  // a [N], S [N]
    uint32_t* a = tsm;
    uint32_t* Ssh = tsm + N;
    const long long row = blockIdx.x;  // i * 2 levels + r
    const int i = (int)(row / (2 * levels)), r = (int)(row - (long long)i * 2 * levels);
    const int k = threadIdx.x;
    const uint64_t per_row = (uint64_t)(N / 16);
    if ((k & 15) == 0) {
        uint32_t blk[16];
        chacha20_block(key, u0 + (uint64_t)row * per_row + (uint64_t)(k >> 4), kStreamUniform, blk);
#pragma unroll
        for (int w = 0; w < 16; ++w) a[k + w] = blk[w];
    }
    Ssh[k] = (uint32_t)S[k];
    __syncthreads();
    // (a S)_k = sum_j a_j S_(k-j) with the sign of the wrap (X^N = -1)
    uint32_t acc = 0;  // products mod 2^32: a small signed key entry multiplies as its residue
    for (int j = 0; j <= k; ++j) acc += a[j] * Ssh[k - j];
    for (int j = k + 1; j < N; ++j) acc -= a[j] * Ssh[k - j + N];
    const int32_t e = torus_gauss(key, g0 + (uint64_t)row * (uint64_t)(N / 4) + (uint64_t)(k >> 2), k, sigma32);
    uint32_t b = acc + (uint32_t)e;
    uint32_t av = a[k];
    const int c = r / levels, l = r - c * levels;
    if (k == 0) {
        const uint32_t m = (uint32_t)s[i] << (32 - base_log * (l + 1));
        if (c == 0) av += m;
        else b += m;
    }
    uint32_t* out = rows + (size_t)row * 2 * N;
    out[k] = av;
    out[N + k] = b;
}

// one thread per key-switching-key row (j, l): mask, then body
__global__ void k_torus_ksk_rows(uint32_t* __restrict__ ksk, const int32_t* __restrict__ s,
                                 const int32_t* __restrict__ S, int n, int N, int levels, int base_log, double sigma32,
                                 const __grid_constant__ PrngKey key, uint64_t u0, uint64_t g0) {
    const long long rows = (long long)N * levels;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < rows;
         row += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(row / levels), l = (int)(row - (long long)j * levels);
        uint32_t* out = ksk + (size_t)row * (n + 1);
        const uint64_t per_row = (uint64_t)((n + 15) / 16);
        uint32_t dot = 0;
        for (int c = 0; c < n; c += 16) {
            uint32_t blk[16];
            chacha20_block(key, u0 + (uint64_t)row * per_row + (uint64_t)(c >> 4), kStreamUniform, blk);
            for (int w = 0; w < 16 && c + w < n; ++w) {
                out[c + w] = blk[w];
                dot += blk[w] * (uint32_t)s[c + w];
            }
        }
        const int32_t e = torus_gauss(key, g0 + (uint64_t)row, 0, sigma32);
        out[n] = dot + (uint32_t)e + ((uint32_t)S[j] << (32 - base_log * (l + 1)));
    }
}

}  // namespace
}  // namespace vc

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

// Torus CGGI keys generated on the device from the caller's secret keys (binary or
// small signed int32): d_bsk_rows [n][2 bs_levels][2][N] uint32 (then to_fourier for the
// spectra the bootstrap reads) and d_ksk [N][ks_levels][n+1] uint32.
int vfhe_cuda_cggi_fft_gen_keys(uint32_t* d_bsk_rows, uint32_t* d_ksk, const int32_t* d_s, const int32_t* d_S,
                                uint32_t n, uint32_t N, uint32_t bs_base_log, uint32_t bs_levels, uint32_t ks_base_log,
                                uint32_t ks_levels, double lwe_sigma, double glwe_sigma, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_cggi_fft_gen_keys";
    if (!d_bsk_rows || !d_ksk || !d_s || !d_S || n == 0 || n > (1u << 16) || (N != 512 && N != 1024 && N != 2048) ||
        bs_levels == 0 || bs_levels * bs_base_log > 32 || ks_levels == 0 || ks_levels * ks_base_log > 32 ||
        !(lwe_sigma >= 0.0) || !(glwe_sigma >= 0.0)) {
        set_error(where, "bad buffers, n, N (512/1024/2048), gadget shapes or noise widths");
        return 1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t bsk_rows = (uint64_t)n * 2 * bs_levels;
    const uint64_t ksk_rows = (uint64_t)N * ks_levels;
    const uint64_t u0 = prng_advance(bsk_rows * (N / 16) + ksk_rows * ((n + 15) / 16));
    const uint64_t g0 = prng_advance(bsk_rows * (N / 4) + ksk_rows);
    const PrngKey key = prng_key();
    k_torus_bsk_rows<<<(unsigned)bsk_rows, N, 2 * N * sizeof(uint32_t), st>>>(
        d_bsk_rows, d_s, d_S, (int)N, (int)bs_levels, (int)bs_base_log, glwe_sigma * 4294967296.0, key, u0, g0);
    note_launch();
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    k_torus_ksk_rows<<<(unsigned)((ksk_rows + 255) / 256), 256, 0, st>>>(
        d_ksk, d_s, d_S, (int)n, (int)N, (int)ks_levels, (int)ks_base_log, lwe_sigma * 4294967296.0, key,
        u0 + bsk_rows * (N / 16), g0 + bsk_rows * (N / 4));
    note_launch();
    return check_cuda(cudaGetLastError(), where) ? 0 : 1;
}

}  // extern "C"
