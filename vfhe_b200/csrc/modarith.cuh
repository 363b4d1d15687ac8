// Modular arithmetic on 64-bit words for RNS primes q < 2^61 (the vfhe hot path
// uses q < 2^50: the reference routes every such prime to its 50-bit IFMA kernels,
// modules/arith/c/src/ntt.c:315-345, mod.c:69-276).
//
// Every helper returns the canonical residue in [0, q) unless its name says
// "lazy".  Canonical results are unique, so any sequence of these operations that
// is exact modular arithmetic reproduces the reference's outputs bit for bit
// (modules/arith/c/src/mod_portable.c:7-161 computes the same residues with
// unsigned __int128).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define VC_HD __host__ __device__ __forceinline__
#else
#define VC_HD inline
#endif

namespace vc {

// Per-prime constants, built on the host (see tables.cpp).
struct PrimeInfo {
    uint64_t q;
    uint64_t two_q;
    uint64_t bar_mu;     // floor(2^(b+62) / q), b = bit length of q (Barrett, see mul_mod)
    uint32_t bar_shift;  // b - 2
    uint32_t log_p;      // log2 of the per-block transform size P
    uint64_t p_inv;      // P^-1 mod q (the inverse transform's final scale)
    uint64_t p_inv_sh;   // Shoup companion of p_inv
    uint64_t inv_last;   // inverse twiddle of the last GS stage times P^-1
    uint64_t inv_last_sh;
    const uint64_t* fwd;     // P twiddles psi^brv(i), Shoup companions interleaved: [w, w']
    const uint64_t* inv;     // P twiddles psi^-brv(i), interleaved the same way
    const uint64_t* twist;   // P values psi^(2 brv(k) + 1), interleaved [w, w']
    // FP64 butterfly path (q < 2^50 only, fp64 != 0): twiddles centred to |w| <= q/2
    // and interleaved with fl(w/q); constants as (centred value, fl(value/q)).
    const double* fwd_d;
    const double* inv_d;
    double qd, qinv;
    double pinv_d, pinv_q;
    double ilast_d, ilast_q;
    int fp64;
    // The same FP64 twiddles of the four lowest stages (index bits 0..3) in lane-major
    // order: block g of 16 residues needs 15 of them (slot s = 2^(3-b) - 1 + h for bit b),
    // stored at ((g >> 5) * 15 + s) * 32 + (g & 31), so that a warp whose lanes hold 32
    // consecutive blocks reads 32 consecutive (w, fl(w/q)) pairs per slot.
    const double* fwd_lane;
    const double* inv_lane;
    // The stages at index bits 2..5 the same way, by group G of 64 residues (P >= 64,
    // else null): slot s = 2^(3-b') - 1 + h for bit b' + 2, at ((G >> 5) * 15 + s) * 32
    // + (G & 31); a radix-16 pass over bits 2..5 gives a warp 8 consecutive groups.
    const double* fwd_mid;
    const double* inv_mid;
};

VC_HD uint64_t umulhi(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

VC_HD uint64_t csub(uint64_t x, uint64_t q) { return x >= q ? x - q : x; }

VC_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }

VC_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

VC_HD uint64_t neg_mod(uint64_t a, uint64_t q) { return a == 0 ? 0 : q - a; }

// Shoup multiplication by a fixed operand w < q with companion ws = floor(w 2^64 / q).
// For any x < 2^64 the lazy result lies in [0, 2q).
VC_HD uint64_t shoup_lazy(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t qh = umulhi(x, ws);
    return x * w - qh * q;
}

VC_HD uint64_t shoup(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    return csub(shoup_lazy(x, w, ws, q), q);
}

// Barrett reduction of a 128-bit value x = hi:lo with x < 2^(2b), b = bit length of q.
// x1 = floor(x / 2^(b-2)) < 2^(b+2); qhat = floor(x1 * mu / 2^64) with
// mu = floor(2^(b+62)/q) satisfies floor(x/q) - 2 <= qhat <= floor(x/q), so the
// remainder before correction is below 3q.
VC_HD uint64_t barrett128(uint64_t hi, uint64_t lo, const PrimeInfo& p) {
    const uint32_t s = p.bar_shift;
    uint64_t x1 = (lo >> s) | (s ? (hi << (64 - s)) : 0);
    uint64_t qh = umulhi(x1, p.bar_mu);
    uint64_t r = lo - qh * p.q;
    r = csub(r, p.two_q);
    return csub(r, p.q);
}

// a * b mod q for a, b < q.
VC_HD uint64_t mul_mod(uint64_t a, uint64_t b, const PrimeInfo& p) {
    return barrett128(umulhi(a, b), a * b, p);
}

// x mod q for an arbitrary 64-bit x (x < 2^64 <= 2^(2b) whenever b >= 32;
// for smaller primes fall back to the hardware remainder).
VC_HD uint64_t reduce64(uint64_t x, const PrimeInfo& p) {
    if (p.bar_shift + 2 >= 32) return barrett128(0, x, p);
    return x % p.q;
}

// Signed 64-bit value to its residue (mod_eltwise_reduce_signed,
// modules/arith/c/src/mod_portable.c:120-137).
VC_HD uint64_t reduce_signed(int64_t v, const PrimeInfo& p) {
    uint64_t mag = v < 0 ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
    uint64_t r = reduce64(mag, p);
    return v < 0 ? neg_mod(r, p.q) : r;
}

}  // namespace vc
