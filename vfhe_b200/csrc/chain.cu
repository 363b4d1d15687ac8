// NTT -> product -> INTT chains in one kernel (vfhe_cuda_ntt_mul_intt_batch).
//
// The chain polynomial_RNSc_to_RNS(a), polynomial_RNSc_to_RNS(b),
// polynomial_mul_RNS_polynomial, polynomial_RNS_to_RNSc (rns_polynomial.c:311-356,
// 582-614) run as four launches moves every residue through HBM five times.  Here one
// CTA takes one (polynomial, limb) row of N = S P residues, S the ring's split degree
// and P = 2^K the per-block transform size: group g of its threads (2^(K-4) of them,
// 16 residues each) transforms block g of a, parks the spectrum in shared memory,
// transforms block g of b, and then every thread forms its output block's 16 slots of
// the incomplete product
//   out_o[x] = sum_{i <= o} a_i[x] b_{o-i}[x] + w[x] sum_{i > o} a_i[x] b_{o-i+S}[x]
// (w the pool's twist table) and runs the inverse transform of block o from registers.
// The row is read once per operand and written once.  Arithmetic is the exact FP64 form
// of fp64mod.cuh throughout: every product of two reduced operands (|.| <= q/2 + 1) is
// exact modulo q, so the canonical output equals the four-launch chain's bit for bit.
//
// Shapes: FP64 primes, N <= 2^13 (so S P <= 8192 residues of both operands fit in
// shared memory: 17 N bytes), P from 2^9 to 2^13 (a block's threads are whole warps,
// so each group meets at its own named barrier).
#include <cuda_runtime.h>

#include <mutex>

#include "engine.cuh"
#include "ntt_f64_dev.cuh"

namespace vc {

namespace {

struct ChainLimbs {
    uint32_t p[kMaxLimbs];  // pool index of each limb slot's prime
};

// Up to 128 registers for 256-thread CTAs (two per SM, 70 KB of shared memory each at
// N = 4096; a three-per-SM cap of 85 registers spilled 100-190 bytes per thread) and
// 512-thread CTAs (N = 8192, 139 KB, one per SM); smaller CTAs are left to the compiler.
template <int K, int S>
__global__ void __launch_bounds__(S << (K - 4), (S << (K - 4)) <= 256 ? 2 : 1) k_chain_f(uint64_t* __restrict__ out, const uint64_t* __restrict__ a,
                                                          const uint64_t* __restrict__ b,
                                                          const __grid_constant__ ChainLimbs cl,
                                                          const PrimeInfo* __restrict__ primes, int nl) {
    constexpr int TPT = 1 << (K - 4), P = 1 << K, PADDED = P + (P >> 4);
    constexpr bool GROUP = S > 1;
    extern __shared__ __align__(128) double csm[];
    double* spec = csm;            // [S][PADDED]: a's spectra, reduced, at pad(16 t + m)
    double* ex = csm + S * PADDED;  // [S][PADDED]: each block's exchanges, then b's spectra
    const int g = threadIdx.x / TPT;
    const int t = threadIdx.x - g * TPT;
    const long long row = blockIdx.x;  // polynomial * nl + limb slot
    const int slot = (int)(row % nl);
    const PrimeInfo& pi = primes[cl.p[slot]];
    const double q = pi.qd, qinv = pi.qinv;
    const long long off = row * (long long)(S * P) + (long long)g * P;
    double* exg = ex + g * PADDED;

    Tile tile;
    tile.hi = 0;
    tile.pi = &pi;
    tile.dst = nullptr;
    double x[16];
    // a's block g
    tile.src = a + off;
    tile_fwd_regs<K, false, false, GROUP>(tile, K, false, exg, t, x, g);
#pragma unroll
    for (int m = 0; m < 16; ++m) spec[g * PADDED + pad(16 * t + m)] = f_reduce(x[m], q, qinv);
    tile_sync<K, GROUP>(g);  // the block's last exchange reads are over before b's first write
    // b's block g.  Its twiddles are a's again; the prime's address goes through an
    // opaque move so that the compiler reloads them instead of keeping a's ~90 registers
    // of twiddles alive across both transforms.
    tile.src = b + off;
    const PrimeInfo* pib;
    asm volatile("mov.b64 %0, %1;" : "=l"(pib) : "l"(&pi));
    tile.pi = pib;
    tile_fwd_regs<K, false, false, GROUP>(tile, K, false, exg, t, x, g);
    if constexpr (S == 1) {
        // pointwise: this thread's own slots of a's spectrum (written by this thread)
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const double w = f_reduce(x[m], q, qinv);
            x[m] = f_mulmod(spec[pad(16 * t + m)], w, __dmul_rn(w, qinv), q);  // |x| <= 3q/4
        }
    } else {
        tile_sync<K, GROUP>(g);  // the block's exchanges are over: its buffer takes b's spectrum
#pragma unroll
        for (int m = 0; m < 16; ++m) exg[pad(16 * t + m)] = f_reduce(x[m], q, qinv);
        __syncthreads();  // every block's spectra of a and b are in shared memory
        const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.twist);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int xs = 16 * t + m, px = pad(xs);
            double acc = 0.0, wrap = 0.0;
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const double u = spec[i * PADDED + px];
                if (i <= g) {
                    const double v = ex[(g - i) * PADDED + px];
                    acc = __dadd_rn(acc, f_mulmod(u, v, __dmul_rn(v, qinv), q));
                } else {
                    const double v = ex[(g - i + S) * PADDED + px];
                    wrap = __dadd_rn(wrap, f_mulmod(u, v, __dmul_rn(v, qinv), q));
                }
            }
            // at most 8 terms of at most 3q/4 each: below 6q < 2^53
            acc = f_reduce(acc, q, qinv);
            wrap = f_reduce(wrap, q, qinv);
            const uint64_t wi = tw[xs].x;
            const double wd = wi > pi.q / 2 ? (double)wi - q : (double)wi;
            x[m] = f_reduce(__dadd_rn(acc, f_mulmod(wrap, wd, __dmul_rn(wd, qinv), q)), q, qinv);
        }
        __syncthreads();  // every block's b spectrum is read before the exchanges reuse it
    }
    tile_inv_regs<K, true, GROUP>(pi, K, 0, exg, t, x, g);
    uint64_t* o = out + off;
#pragma unroll
    for (int m = 0; m < 16; ++m) o[own<K - 4>(t, m)] = f_to_canonical(x[m], q, qinv, pi.q);
}

template <int K, int S>
constexpr size_t chain_smem() {
    return sizeof(double) * 2 * (size_t)S * ((1 << K) + (1 << (K - 4)));
}

template <int K, int S>
int chain_attr() {
    if (chain_smem<K, S>() <= 48 * 1024) return 0;
    return (int)cudaFuncSetAttribute(k_chain_f<K, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)chain_smem<K, S>());
}

template <int K, int S>
int chain_launch(uint64_t* out, const uint64_t* a, const uint64_t* b, long long rows, const ChainLimbs& cl,
                 const PrimeInfo* d, int nl, cudaStream_t st) {
    // the shared-memory limit is raised at the first launch (and by prepare_chain_kernels
    // before any stream capture)
    static std::once_flag once;
    static int attr_err = 0;
    std::call_once(once, [] { attr_err = chain_attr<K, S>(); });
    if (attr_err) return attr_err;
    k_chain_f<K, S><<<(unsigned)rows, S << (K - 4), chain_smem<K, S>(), st>>>(out, a, b, cl, d, nl);
    note_launch();
    return (int)cudaGetLastError();
}

}  // namespace

int prepare_chain_kernels() {
    int e = chain_attr<9, 1>();
    if (!e) e = chain_attr<9, 2>();
    if (!e) e = chain_attr<9, 4>();
    if (!e) e = chain_attr<9, 8>();
    if (!e) e = chain_attr<10, 1>();
    if (!e) e = chain_attr<10, 2>();
    if (!e) e = chain_attr<10, 4>();
    if (!e) e = chain_attr<10, 8>();
    if (!e) e = chain_attr<11, 1>();
    if (!e) e = chain_attr<11, 2>();
    if (!e) e = chain_attr<11, 4>();
    if (!e) e = chain_attr<12, 1>();
    if (!e) e = chain_attr<12, 2>();
    if (!e) e = chain_attr<13, 1>();
    return e;
}

int launch_chain(IncNtt* t, uint64_t* out, const uint64_t* a, const uint64_t* b, uint64_t batch,
                 const uint32_t* limbs, uint32_t nlimbs, cudaStream_t st) {
    const uint64_t N = t->pub.N, S = t->pub.split_degree;
    const int K = t->logP;
    if (N > 8192 || K < 9 || K > 13 || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs || batch == 0 ||
        batch * nlimbs > 0x7fffffffULL)
        return kChainUnavailable;
    if (((reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) != 0)
        return kChainUnavailable;
    ChainLimbs cl;
    for (uint32_t k = 0; k < nlimbs; ++k) {
        if (limbs[k] >= t->pub.l || !t->info[limbs[k]].fp64) return kChainUnavailable;
        cl.p[k] = limbs[k];
    }
    const long long rows = (long long)(batch * nlimbs);
    switch (K * 16 + (int)S) {
        case 9 * 16 + 1: return chain_launch<9, 1>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 9 * 16 + 2: return chain_launch<9, 2>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 9 * 16 + 4: return chain_launch<9, 4>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 9 * 16 + 8: return chain_launch<9, 8>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 10 * 16 + 1: return chain_launch<10, 1>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 10 * 16 + 2: return chain_launch<10, 2>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 10 * 16 + 4: return chain_launch<10, 4>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 10 * 16 + 8: return chain_launch<10, 8>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 11 * 16 + 1: return chain_launch<11, 1>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 11 * 16 + 2: return chain_launch<11, 2>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 11 * 16 + 4: return chain_launch<11, 4>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 12 * 16 + 1: return chain_launch<12, 1>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 12 * 16 + 2: return chain_launch<12, 2>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        case 13 * 16 + 1: return chain_launch<13, 1>(out, a, b, rows, cl, t->d_info, (int)nlimbs, st);
        default: return kChainUnavailable;
    }
}

}  // namespace vc
