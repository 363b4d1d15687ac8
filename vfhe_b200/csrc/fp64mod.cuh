// Exact modular arithmetic in FP64 for primes q < 2^50.
//
// Residues are carried as doubles holding exact integers (|x| < 2^52).  A product
// y * w is split error-free into h + l with h = fl(y w), l = fma(y, w, -h) (the
// classical FMA two-product).  The quotient estimate n = round(y * (w/q)) comes out of
// one FMA against M = 1.5 * 2^52: for |c| < 2^51, fl(c + M) - M is c rounded to the
// nearest integer.  Then r = fma(-n, q, h) is exact (its true value h - n q is an
// integer below 2^51) and t = r + l = y w - n q exactly.
//
// Bounds (q < 2^50, centred twiddles |w| <= q/2, wq = fl(w/q), |y| < 2^52):
//   |y wq| < 2^51, and |y w/q - n| <= 1/2 + |y| 2^-54, so |t| <= q/2 + q |y| 2^-54
//   <= 3q/4.  Reduction x -> x - round(x/q) q leaves |x| <= q/2 + q 2^-51.
// Every intermediate is an integer below 2^53 in magnitude, so each step is exact and
// the canonical residue produced at the end equals the integer algorithm's.
// All operations use the _rn intrinsics so the compiler cannot contract or reorder them.
#pragma once
#include <stdint.h>

namespace vc {

constexpr double kRoundMagic = 6755399441055744.0;  // 1.5 * 2^52

// y * w mod q, centred, |result| <= 3q/4 (needs |y| < 2^52, |w| <= q/2, wq = fl(w/q)).
// The same steps accept an uncentred 0 <= w < q when |y| < 2^50: then
// |y w/q - n| <= 1/2 + |y| 2^-53 and |result| <= q/2 + q/8.
__device__ __forceinline__ double f_mulmod(double y, double w, double wq, double q) {
    const double h = __dmul_rn(y, w);
    const double l = __fma_rn(y, w, -h);
    const double n = __dadd_rn(__fma_rn(y, wq, kRoundMagic), -kRoundMagic);
    const double r = __fma_rn(-n, q, h);
    return __dadd_rn(r, l);
}

// x mod q, centred, |result| <= q/2 + 1 (needs |x| < 2^52 and qinv = fl(1/q)).
__device__ __forceinline__ double f_reduce(double x, double q, double qinv) {
    const double n = __dadd_rn(__fma_rn(x, qinv, kRoundMagic), -kRoundMagic);
    return __fma_rn(-n, q, x);
}

// Canonical uint64 residue in [0, q) of a centred value.
__device__ __forceinline__ uint64_t f_to_canonical(double x, double q, double qinv, uint64_t qi) {
    const double c = f_reduce(x, q, qinv);
    // |c| < 2^51: c + M is exact, and its low 52 mantissa bits hold c + 2^51
    const long long bits = __double_as_longlong(__dadd_rn(c, kRoundMagic));
    long long v = (bits & 0xFFFFFFFFFFFFFLL) - (1LL << 51);
    v += (v >> 63) & (long long)qi;
    return (uint64_t)v;
}

// uint64 x < 2^52 to double, exactly.
__device__ __forceinline__ double f_from_u64(uint64_t x) {
    return __dadd_rn(__longlong_as_double((long long)(x | 0x4330000000000000ULL)), -4503599627370496.0);
}

}  // namespace vc
