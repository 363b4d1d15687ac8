// Element-wise limb kernels: canonical modular add/sub/mul/scale, the incomplete
// split-degree product, Galois permutation, X^a rotations, RNS round/floor division
// and the engine's sampling.  All are HBM-bound streaming kernels: one thread per
// residue (grid-stride), limbs and polynomials of a batch on gridDim.y.
#include <cuda_runtime.h>
#include <string.h>
#include <math.h>

#include "engine.cuh"

namespace vc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void limb_coords(const EwSet& set, int& k, long long& boff) {
    const int by = blockIdx.y;
    const int b = by / set.nlimbs;
    k = by - b * set.nlimbs;
    boff = (long long)b * set.batch_stride;
}

template <int OP>
__global__ void k_ew(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const PrimeInfo pi = primes[set.prime[k]];
    uint64_t* out = set.out[k] + boff;
    const uint64_t* a = set.a[k] ? set.a[k] + boff : nullptr;
    const uint64_t* b = set.b[k] ? set.b[k] + boff : nullptr;
    const uint64_t s = set.s[k], ssh = set.s_sh[k];
    const uint64_t q = pi.q;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < set.n;
         i += (long long)gridDim.x * blockDim.x) {
        uint64_t r;
        if (OP == EW_COPY) r = a[i];
        else if (OP == EW_ZERO) r = 0;
        else if (OP == EW_ADD) r = add_mod(a[i], b[i], q);
        else if (OP == EW_SUB) r = sub_mod(a[i], b[i], q);
        else if (OP == EW_NEG) r = neg_mod(a[i], q);
        else if (OP == EW_MUL) r = mul_mod(a[i], b[i], pi);
        else if (OP == EW_MUL_ADDTO) r = add_mod(out[i], mul_mod(a[i], b[i], pi), q);
        else if (OP == EW_MUL_SUBTO) r = sub_mod(out[i], mul_mod(a[i], b[i], pi), q);
        else if (OP == EW_SCALE) r = shoup(a[i], s, ssh, q);
        else if (OP == EW_SCALE_ADDTO) r = add_mod(out[i], shoup(a[i], s, ssh, q), q);
        else if (OP == EW_ADD_SCALAR) r = add_mod(a[i], s, q);
        else r = reduce64(a[i], pi);  // EW_REDUCE
        out[i] = r;
    }
}

dim3 ew_grid(const EwSet& set) {
    long long blocks = (set.n + kThreads - 1) / kThreads;
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    return dim3((unsigned)blocks, (unsigned)(set.nlimbs * set.batch), 1);
}

// Incomplete product over `split` blocks of P slots: for block indices j, k,
// out[j+k] += a_j b_k, and for j+k >= split, out[j+k-split] += a_j b_k w
// (rns_polynomial.c:311-356; w is the per-slot twist, rns_polynomial.c:19-27).
template <int MODE, int S>
__global__ void k_inc_product(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                              int logP) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const PrimeInfo pi = primes[set.prime[k]];
    const uint64_t q = pi.q;
    const long long P = 1LL << logP;
    uint64_t* out = set.out[k] + boff;
    const uint64_t* a = set.a[k] + boff;
    const uint64_t* b = set.b[k] + boff;
    const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.twist);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < P;
         x += (long long)gridDim.x * blockDim.x) {
        // every output block of slot x depends on every input block of slot x: read
        // them all before writing, so out may alias a or b
        uint64_t av[S], bv[S], res[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            av[j] = a[j * P + x];
            bv[j] = b[j * P + x];
        }
#pragma unroll
        for (int o = 0; o < S; ++o) {
            uint64_t acc = 0, wrap = 0;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                if (j <= o) acc = add_mod(acc, mul_mod(av[j], bv[o - j], pi), q);
                else wrap = add_mod(wrap, mul_mod(av[j], bv[o - j + S], pi), q);
            }
            if (S > 1) {
                const ulonglong2 w = tw[x];
                acc = add_mod(acc, shoup(wrap, w.x, w.y, q), q);
            }
            res[o] = acc;
        }
#pragma unroll
        for (int o = 0; o < S; ++o) {
            uint64_t r = res[o];
            if (MODE == 1) r = add_mod(out[o * P + x], r, q);
            else if (MODE == 2) r = sub_mod(out[o * P + x], r, q);
            out[o * P + x] = r;
        }
    }
}

// Galois map i -> i*gen mod 2N on the split-interleaved layout (rns_polynomial.c:996-1035):
// coefficient c = i + i2*split sits at row position i*P + i2.
__global__ void k_permute(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                          uint64_t N, int split, int log_split, uint64_t gen) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const PrimeInfo pi = primes[set.prime[k]];
    uint64_t* out = set.out[k] + boff;
    const uint64_t* in = set.a[k] + boff;
    const uint64_t P = N >> log_split;
    for (long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x; pos < (long long)N;
         pos += (long long)gridDim.x * blockDim.x) {
        const uint64_t i = (uint64_t)pos / P, i2 = (uint64_t)pos % P;
        const uint64_t idx = (i + (i2 << log_split)) * gen;
        const uint64_t dst = (idx & (uint64_t)(split - 1)) * P + ((idx & (N - 1)) >> log_split);
        const uint64_t v = in[pos];
        out[dst] = (idx & N) ? neg_mod(v, pi.q) : v;
    }
}

// out = in * X^a (or in * (X^a - 1)), negacyclic, split_degree 1 (rns_polynomial.c:1048-1180).
template <bool MINUS1>
__global__ void k_mul_xai(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                          uint64_t N, uint64_t a) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const uint64_t q = primes[set.prime[k]].q;
    uint64_t* out = set.out[k] + boff;
    const uint64_t* in = set.a[k] + boff;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < (long long)N;
         x += (long long)gridDim.x * blockDim.x) {
        // source index of X^a * in at position x: (x - a) mod 2N, negated past N
        const uint64_t src = ((uint64_t)x + 2 * N - a) & (2 * N - 1);
        const uint64_t v = src < N ? in[src] : neg_mod(in[src - N], q);
        out[x] = MINUS1 ? sub_mod(v, in[x], q) : v;
    }
}

// One prime dropped: t = (c_p + half) mod p; c_i <- (c_i + half - t) * p^-1 mod q_i; c_p <- 0.
__global__ void k_divide(const __grid_constant__ EwSet set, DivideArgs d, const PrimeInfo* __restrict__ primes,
                         long long n) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
         x += (long long)gridDim.x * blockDim.x) {
        const uint64_t cp = d.drop_row[x];
        const uint64_t t = add_mod(cp, d.half_drop, d.p);
        for (int k = 0; k < set.nlimbs; ++k) {
            const PrimeInfo& pi = primes[set.prime[k]];
            const uint64_t q = pi.q;
            uint64_t c = set.out[k][x];
            c = add_mod(c, reduce64(d.half_drop, pi), q);
            c = sub_mod(c, reduce64(t, pi), q);
            set.out[k][x] = shoup(c, set.s[k], set.s_sh[k], q);
        }
        d.drop_row[x] = 0;
    }
}

// Uniform residues, four per ChaCha20 block (128 bits each, so the residues are within
// q / 2^128 of uniform).  Row r (limb k of polynomial b) owns blocks
// counter + r ceil(n/4) ...; thread j fills elements 4j .. 4j+3 of its row.
__global__ void k_uniform(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                          const __grid_constant__ PrngKey key, uint64_t counter) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const uint64_t q = primes[set.prime[k]].q;
    uint64_t* out = set.out[k] + boff;
    const long long per_row = (set.n + 3) / 4;
    const uint64_t base = counter + (uint64_t)blockIdx.y * (uint64_t)per_row;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < per_row;
         j += (long long)gridDim.x * blockDim.x) {
        uint32_t blk[16];
        chacha20_block(key, base + j, kStreamUniform, blk);
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (4 * j + e < set.n) out[4 * j + e] = uniform_mod(block_u64(blk, 2 * e), block_u64(blk, 2 * e + 1), q);
    }
}

// Rounded Gaussian integers shared by every limb of a coefficient, reduced per limb
// (polynomial_gen_gaussian_RNSc_polynomial, rns_polynomial.c:255-271: Box-Muller with
// the cosine branch, then round).  Polynomial b owns blocks counter + b ceil(n/4) ...,
// four coefficients per block; every limb row of the polynomial recomputes the same
// blocks, so the integer is the same in each limb.
__global__ void k_gaussian(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                           double sigma, const __grid_constant__ PrngKey key, uint64_t counter) {
    int k;
    long long boff;
    limb_coords(set, k, boff);
    const PrimeInfo pi = primes[set.prime[k]];
    uint64_t* out = set.out[k] + boff;
    const long long per_poly = (set.n + 3) / 4;
    const uint64_t base = counter + (uint64_t)(blockIdx.y / set.nlimbs) * (uint64_t)per_poly;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < per_poly;
         j += (long long)gridDim.x * blockDim.x) {
        uint32_t blk[16];
        chacha20_block(key, base + j, kStreamGaussian, blk);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (4 * j + e >= set.n) break;
            const double z = sqrt(-2.0 * log(unit_open_low(block_u64(blk, 2 * e)))) *
                             cospi(2.0 * unit_closed_low(block_u64(blk, 2 * e + 1)));
            out[4 * j + e] = reduce_signed((int64_t)llrint(sigma * z), pi);
        }
    }
}

}  // namespace

int launch_ew(EwOp op, const EwSet& set, const PrimeInfo* d_primes, cudaStream_t st) {
    if (set.nlimbs <= 0 || set.n <= 0 || set.batch <= 0) return 0;
    dim3 g = ew_grid(set);
    switch (op) {
#define VC_EW(OPC) \
    case OPC:      \
        k_ew<OPC><<<g, kThreads, 0, st>>>(set, d_primes); break;
        VC_EW(EW_COPY)
        VC_EW(EW_ZERO)
        VC_EW(EW_ADD)
        VC_EW(EW_SUB)
        VC_EW(EW_NEG)
        VC_EW(EW_MUL)
        VC_EW(EW_MUL_ADDTO)
        VC_EW(EW_MUL_SUBTO)
        VC_EW(EW_SCALE)
        VC_EW(EW_SCALE_ADDTO)
        VC_EW(EW_ADD_SCALAR)
        VC_EW(EW_REDUCE)
#undef VC_EW
        default:
            return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

template <int MODE>
static int inc_product_mode(const EwSet& set, int split, int logP, const PrimeInfo* d_primes,
                            cudaStream_t st, dim3 g) {
    switch (split) {
        case 1: k_inc_product<MODE, 1><<<g, kThreads, 0, st>>>(set, d_primes, logP); break;
        case 2: k_inc_product<MODE, 2><<<g, kThreads, 0, st>>>(set, d_primes, logP); break;
        case 4: k_inc_product<MODE, 4><<<g, kThreads, 0, st>>>(set, d_primes, logP); break;
        case 8: k_inc_product<MODE, 8><<<g, kThreads, 0, st>>>(set, d_primes, logP); break;
        case 16: k_inc_product<MODE, 16><<<g, kThreads, 0, st>>>(set, d_primes, logP); break;
        default: return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

int launch_inc_product(int mode, const EwSet& set, int split, int logP, const PrimeInfo* d_primes,
                       cudaStream_t st) {
    if (set.nlimbs <= 0 || set.batch <= 0) return 0;
    EwSet s2 = set;
    s2.n = 1LL << logP;
    dim3 g = ew_grid(s2);
    if (mode == 0) return inc_product_mode<0>(set, split, logP, d_primes, st, g);
    if (mode == 1) return inc_product_mode<1>(set, split, logP, d_primes, st, g);
    return inc_product_mode<2>(set, split, logP, d_primes, st, g);
}

int launch_permute(const EwSet& set, uint64_t N, int split, uint64_t gen, const PrimeInfo* d_primes,
                   cudaStream_t st) {
    if (set.nlimbs <= 0 || set.batch <= 0) return 0;
    int ls = 0;
    while ((1 << ls) < split) ++ls;
    EwSet s2 = set;
    s2.n = (long long)N;
    k_permute<<<ew_grid(s2), kThreads, 0, st>>>(set, d_primes, N, split, ls, gen);
    return (int)cudaGetLastError();
}

int launch_mul_xai(const EwSet& set, uint64_t N, uint64_t a, bool minus1, const PrimeInfo* d_primes,
                   cudaStream_t st) {
    if (set.nlimbs <= 0 || set.batch <= 0) return 0;
    EwSet s2 = set;
    s2.n = (long long)N;
    if (minus1) k_mul_xai<true><<<ew_grid(s2), kThreads, 0, st>>>(set, d_primes, N, a);
    else k_mul_xai<false><<<ew_grid(s2), kThreads, 0, st>>>(set, d_primes, N, a);
    return (int)cudaGetLastError();
}

int launch_divide(const EwSet& set, const DivideArgs& d, const PrimeInfo* d_primes, cudaStream_t st) {
    long long blocks = (set.n + kThreads - 1) / kThreads;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    k_divide<<<(unsigned)blocks, kThreads, 0, st>>>(set, d, d_primes, set.n);
    return (int)cudaGetLastError();
}

int launch_sample_uniform(const EwSet& set, const PrngKey& key, uint64_t counter, const PrimeInfo* d_primes,
                          cudaStream_t st) {
    if (set.nlimbs <= 0) return 0;
    k_uniform<<<ew_grid(set), kThreads, 0, st>>>(set, d_primes, key, counter);
    return (int)cudaGetLastError();
}

int launch_sample_gaussian(const EwSet& set, double sigma, const PrngKey& key, uint64_t counter,
                           const PrimeInfo* d_primes, cudaStream_t st) {
    if (set.nlimbs <= 0) return 0;
    k_gaussian<<<ew_grid(set), kThreads, 0, st>>>(set, d_primes, sigma, key, counter);
    return (int)cudaGetLastError();
}

namespace {
struct SmallBlock {
    uint64_t v[256];
};
__global__ void k_upload_small(uint64_t* __restrict__ dst, const __grid_constant__ SmallBlock blk, int n) {
    if ((int)threadIdx.x < n) dst[threadIdx.x] = blk.v[threadIdx.x];
}
}  // namespace

int upload_small(uint64_t* d_dst, const uint64_t* h_src, uint64_t n, cudaStream_t st) {
    for (uint64_t off = 0; off < n; off += 256) {
        SmallBlock blk;
        const int m = (int)(n - off < 256 ? n - off : 256);
        memcpy(blk.v, h_src + off, (size_t)m * sizeof(uint64_t));
        k_upload_small<<<1, 256, 0, st>>>(d_dst + off, blk, m);
        note_launch();
        const int e = (int)cudaGetLastError();
        if (e) return e;
    }
    return 0;
}

}  // namespace vc
