// Shared pieces of the GHS key switch (mlwe.c:557-598): the constants of the
// special-prime round division and the optional CKKS rescale that follows it.
#pragma once
#include "engine.cuh"
#include "fp64mod.cuh"

namespace vc {

struct ModDownConsts {
    uint32_t prime[kMaxLimbs];      // pool index of output limb i (i < nl)
    uint64_t half_sp[kMaxLimbs];    // floor(p/2) mod q_i, p the special prime
    uint64_t inv_sp[kMaxLimbs];     // p^-1 mod q_i
    uint64_t inv_sp_sh[kMaxLimbs];
    uint64_t half_r[kMaxLimbs];     // floor(q_top/2) mod q_i
    uint64_t inv_r[kMaxLimbs];      // q_top^-1 mod q_i
    uint64_t inv_r_sh[kMaxLimbs];
    uint32_t special;               // pool index of the special prime
    uint64_t p, half_p;             // special prime and floor(p/2)
    uint64_t q_top, half_top;       // top prime dropped by the rescale
    // FP64 form (all primes below 2^50): multipliers centred in (-q/2, q/2] with
    // their quotients fl(w/q), halves as exact doubles
    int fp64;
    double half_sp_d[kMaxLimbs], inv_sp_d[kMaxLimbs], inv_sp_dq[kMaxLimbs];
    double half_r_d[kMaxLimbs], inv_r_d[kMaxLimbs], inv_r_dq[kMaxLimbs];
};

// Constants for dividing [nl + 1] limbs (limbs, then `special`) by the special prime,
// and for rescaling the result by limbs[nl - 1].
ModDownConsts moddown_consts(IncNtt* t, const uint32_t* limbs, int nl, uint32_t special);

// One output slot of -sum_j D_j (*) K_j for both key components, (*) the incomplete
// product over S blocks of P slots (polynomial_mul_subto_RNS_polynomial,
// rns_polynomial.c:398-435: block o collects D[i] K[o-i] and, through the twist w[x],
// D[i] K[o-i+S] for i > o; a pointwise product when S == 1).  Digit j of D is at
// d + j dstr, of key component a at ka + j kstr, of b at kb + j kstr; block i at + i P.
// Exact FP64 (fp64mod.cuh): every term is canonical x canonical, |term| <= 3q/4, and
// the four partial sums are reduced after every fourth term.  Needs q < 2^50.
__device__ __forceinline__ void mac_slot(uint64_t* oa, uint64_t* ob, const uint64_t* d, long long dstr,
                                         const uint64_t* ka, const uint64_t* kb, long long kstr, int nd, int S,
                                         long long P, long long x, int o, const PrimeInfo& pi) {
    const double q = pi.qd, qinv = pi.qinv;
    double sa = 0.0, sb = 0.0, wa = 0.0, wb = 0.0;
    int terms = 0;
    for (int j = 0; j < nd; ++j) {
        for (int i = 0; i < S; ++i) {
            const int k = o - i;
            const bool wrap = k < 0;
            const long long koff = (long long)(wrap ? k + S : k) * P + x;
            const double v = f_from_u64(d[j * dstr + (long long)i * P + x]);
            const double ya = f_from_u64(ka[j * kstr + koff]);
            const double yb = f_from_u64(kb[j * kstr + koff]);
            const double ta = f_mulmod(v, ya, __dmul_rn(ya, qinv), q);
            const double tb = f_mulmod(v, yb, __dmul_rn(yb, qinv), q);
            if (wrap) {
                wa = __dadd_rn(wa, ta);
                wb = __dadd_rn(wb, tb);
            } else {
                sa = __dadd_rn(sa, ta);
                sb = __dadd_rn(sb, tb);
            }
            if (++terms == 4) {
                terms = 0;
                sa = f_reduce(sa, q, qinv);
                sb = f_reduce(sb, q, qinv);
                wa = f_reduce(wa, q, qinv);
                wb = f_reduce(wb, q, qinv);
            }
        }
    }
    if (S > 1) {
        const double w = f_from_u64(reinterpret_cast<const ulonglong2*>(pi.twist)[x].x);
        const double wq = __dmul_rn(w, qinv);
        sa = __dadd_rn(f_reduce(sa, q, qinv), f_mulmod(f_reduce(wa, q, qinv), w, wq, q));
        sb = __dadd_rn(f_reduce(sb, q, qinv), f_mulmod(f_reduce(wb, q, qinv), w, wq, q));
    }
    oa[(long long)o * P + x] = f_to_canonical(-sa, q, qinv, pi.q);
    ob[(long long)o * P + x] = f_to_canonical(-sb, q, qinv, pi.q);
}

// mac_slot for all S output blocks of slot x at once (S = 2 or 4): every digit's S
// blocks of D and of both key components are loaded once (3 S loads per digit for S
// outputs, the traffic of a pointwise product).  Same exact FP64 arithmetic and result.
template <int S>
__device__ __forceinline__ void mac_slots(uint64_t* oa, uint64_t* ob, const uint64_t* d, long long dstr,
                                          const uint64_t* ka, const uint64_t* kb, long long kstr, int nd, long long P,
                                          long long x, const PrimeInfo& pi) {
    const double q = pi.qd, qinv = pi.qinv;
    double sa[S], sb[S], wa[S], wb[S];
#pragma unroll
    for (int o = 0; o < S; ++o) sa[o] = sb[o] = wa[o] = wb[o] = 0.0;
    int terms = 0;
    for (int j = 0; j < nd; ++j) {
        double v[S], ya[S], yqa[S], yb[S], yqb[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            v[i] = f_from_u64(d[j * dstr + (long long)i * P + x]);
            ya[i] = f_from_u64(ka[j * kstr + (long long)i * P + x]);
            yb[i] = f_from_u64(kb[j * kstr + (long long)i * P + x]);
            yqa[i] = __dmul_rn(ya[i], qinv);
            yqb[i] = __dmul_rn(yb[i], qinv);
        }
#pragma unroll
        for (int o = 0; o < S; ++o)
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const int k = o - i;
                const int kk = k < 0 ? k + S : k;
                const double ta = f_mulmod(v[i], ya[kk], yqa[kk], q);
                const double tb = f_mulmod(v[i], yb[kk], yqb[kk], q);
                if (k < 0) {
                    wa[o] = __dadd_rn(wa[o], ta);
                    wb[o] = __dadd_rn(wb[o], tb);
                } else {
                    sa[o] = __dadd_rn(sa[o], ta);
                    sb[o] = __dadd_rn(sb[o], tb);
                }
            }
        // each accumulator gains at most S terms of <= 9q/16 per digit; with q < 2^50
        // six terms on top of a reduced value stay below 2^52 (S <= 4 here)
        terms += S;
        if (terms + S > 6 || j == nd - 1) {
#pragma unroll
            for (int o = 0; o < S; ++o) {
                sa[o] = f_reduce(sa[o], q, qinv);
                sb[o] = f_reduce(sb[o], q, qinv);
                wa[o] = f_reduce(wa[o], q, qinv);
                wb[o] = f_reduce(wb[o], q, qinv);
            }
            terms = 0;
        }
    }
    const double w = f_from_u64(reinterpret_cast<const ulonglong2*>(pi.twist)[x].x);
    const double wq = __dmul_rn(w, qinv);
#pragma unroll
    for (int o = 0; o < S; ++o) {
        const double ra = __dadd_rn(sa[o], f_mulmod(wa[o], w, wq, q));
        const double rb = __dadd_rn(sb[o], f_mulmod(wb[o], w, wq, q));
        oa[(long long)o * P + x] = f_to_canonical(-ra, q, qinv, pi.q);
        ob[(long long)o * P + x] = f_to_canonical(-rb, q, qinv, pi.q);
    }
}

// mac_slot for primes of any size (64-bit Barrett products, canonical sums).
__device__ __forceinline__ void mac_slot_int(uint64_t* oa, uint64_t* ob, const uint64_t* d, long long dstr,
                                             const uint64_t* ka, const uint64_t* kb, long long kstr, int nd, int S,
                                             long long P, long long x, int o, const PrimeInfo& pi) {
    const uint64_t q = pi.q;
    uint64_t sa = 0, sb = 0, wa = 0, wb = 0;
    for (int j = 0; j < nd; ++j) {
        for (int i = 0; i < S; ++i) {
            const int k = o - i;
            const bool wrap = k < 0;
            const long long koff = (long long)(wrap ? k + S : k) * P + x;
            const uint64_t v = d[j * dstr + (long long)i * P + x];
            const uint64_t ta = mul_mod(v, ka[j * kstr + koff], pi);
            const uint64_t tb = mul_mod(v, kb[j * kstr + koff], pi);
            if (wrap) {
                wa = add_mod(wa, ta, q);
                wb = add_mod(wb, tb, q);
            } else {
                sa = add_mod(sa, ta, q);
                sb = add_mod(sb, tb, q);
            }
        }
    }
    if (S > 1) {
        const ulonglong2 w = reinterpret_cast<const ulonglong2*>(pi.twist)[x];
        sa = add_mod(sa, shoup(wa, w.x, w.y, q), q);
        sb = add_mod(sb, shoup(wb, w.x, w.y, q), q);
    }
    oa[(long long)o * P + x] = neg_mod(sa, q);
    ob[(long long)o * P + x] = neg_mod(sb, q);
}

}  // namespace vc
