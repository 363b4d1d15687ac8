// Batched CKKS evaluation over device-resident ciphertexts: multiply + relinearise +
// rescale, and rotate (Galois automorphism + key switch).
//
// The steps are the reference's (mlwe_multiply, mlwe.c:711-760; GHS key switch,
// mlwe.c:557-598; gadget product, gadget.c:5-36; round division,
// rns_polynomial.c:939-976; permutation, rns_polynomial.c:996-1035), batched over
// ciphertexts and fused where the data allows:
//   * the tensor product writes all three components in one pass;
//   * the digit broadcast (limb j reduced modulo every extended prime) happens in
//     the load of the forward transform, so the broadcast rows are never stored;
//   * the special-prime round division, the pass-through additions and the CKKS
//     rescale (division by the top prime) are one kernel per coefficient, which also
//     runs the accumulators' inverse column pass (k_coldown) where the transform's
//     schedule allows, so the coefficient-domain accumulators never reach HBM;
//   * the forward transform at the end of the reference's mlwe_multiply and the
//     inverse transform at the start of its rescale are both skipped: they are
//     inverse bijections on canonical residues, so skipping them changes no bit.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "abi_common.cuh"
#include "bulk.cuh"
#include "fp64mod.cuh"
#include "keyswitch.cuh"
#include "ntt_f64_dev.cuh"

namespace vc {

namespace {

struct LimbPrimes {
    uint32_t p[kMaxLimbs];
};

// Pass-through components folded into a key-switch accumulator before its inverse
// transform: acc_i += (P mod q_i) * pass_i for the first nl extended limbs (the special
// limbs get nothing, P mod P = 0).  Round division by P then yields acc / P + pass
// exactly -- the reference adds pass after the division (mlwe.c:737-756) -- because
// (acc_i + P pass_i + P/2 - t) P^-1 = (acc_i + P/2 - t) P^-1 + pass_i mod q_i, with t the
// special limb's residue (unchanged by the fold).  pass rows are NTT domain.
struct FoldConsts {
    const uint64_t* pass;  // ciphertext b's component c: pass + b * stride + c * comp_stride (null: no fold)
    long long stride, comp_stride;
    int nl;
    double pf[kMaxLimbs], pfq[kMaxLimbs];  // P mod q_i, centred, and fl(./q_i)
};

// Block o, slot x of the incomplete product u (*) v over S blocks of P slots
// (polynomial_mul_RNS_polynomial, rns_polynomial.c:311-356).
__device__ __forceinline__ uint64_t inc_prod_slot(const uint64_t* u, const uint64_t* v, int S, long long P,
                                                  long long x, int o, const PrimeInfo& pi) {
    if (S == 1) return mul_mod(u[x], v[x], pi);
    uint64_t acc = 0, wrap = 0;
    for (int i = 0; i < S; ++i) {
        const int k = o - i;
        if (k >= 0) acc = add_mod(acc, mul_mod(u[(long long)i * P + x], v[(long long)k * P + x], pi), pi.q);
        else wrap = add_mod(wrap, mul_mod(u[(long long)i * P + x], v[(long long)(k + S) * P + x], pi), pi.q);
    }
    const ulonglong2 w = reinterpret_cast<const ulonglong2*>(pi.twist)[x];
    return add_mod(acc, shoup(wrap, w.x, w.y, pi.q), pi.q);
}

// d0 = a1 a2, d1 = a1 b2 + b1 a2, d2 = b1 b2 in the NTT domain (mlwe.c:665-709 at rank 1).
// dd (may be null, split 1 only): also write d0's limb k to dd + b dd_stride + k dd_step
// -- the spectrum of key-switch digit k modulo its own prime, NTT(INTT(d0_k)) = d0_k.
template <int S>
__global__ void k_tensor(uint64_t* __restrict__ T, const uint64_t* __restrict__ c1,
                         const uint64_t* __restrict__ c2, const __grid_constant__ LimbPrimes lp,
                         const PrimeInfo* __restrict__ primes, int L, long long N, uint64_t* __restrict__ dd,
                         long long dd_stride, long long dd_step) {
    const int by = blockIdx.y;
    const int b = by / L, k = by - b * L;
    const PrimeInfo pi = primes[lp.p[k]];
    const long long cs = (long long)2 * L * N, ts = (long long)3 * L * N, LN = (long long)L * N;
    const uint64_t* a1 = c1 + b * cs + k * N;
    const uint64_t* b1 = a1 + LN;
    const uint64_t* a2 = c2 + b * cs + k * N;
    const uint64_t* b2 = a2 + LN;
    uint64_t* t0 = T + b * ts + k * N;
    uint64_t* d0k = dd ? dd + b * dd_stride + k * dd_step : nullptr;
    if (S == 1 && pi.fp64 && (N & 1) == 0 &&
        ((reinterpret_cast<uintptr_t>(a1) | reinterpret_cast<uintptr_t>(a2) | reinterpret_cast<uintptr_t>(t0)) & 15) ==
            0) {
        // exact FP64 products (canonical operands below 2^50, uncentred multipliers),
        // two coefficients per thread, inputs read once
        const double q = pi.qd, qinv = pi.qinv;
        for (long long x = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x); x < N;
             x += 2 * (long long)gridDim.x * blockDim.x) {
            const ulonglong2 ua1 = __ldcs(reinterpret_cast<const ulonglong2*>(a1 + x));
            const ulonglong2 ub1 = __ldcs(reinterpret_cast<const ulonglong2*>(b1 + x));
            const ulonglong2 ua2 = __ldcs(reinterpret_cast<const ulonglong2*>(a2 + x));
            const ulonglong2 ub2 = __ldcs(reinterpret_cast<const ulonglong2*>(b2 + x));
            ulonglong2 r0, r1, r2;
            auto one = [&](uint64_t xa1, uint64_t xb1, uint64_t xa2, uint64_t xb2, unsigned long long& d0,
                           unsigned long long& d1, unsigned long long& d2) {
                const double fa1 = f_from_u64(xa1), fb1 = f_from_u64(xb1);
                const double fa2 = f_from_u64(xa2), fb2 = f_from_u64(xb2);
                const double qa1 = __dmul_rn(fa1, qinv), qb1 = __dmul_rn(fb1, qinv);
                d0 = f_to_canonical(f_mulmod(fa2, fa1, qa1, q), q, qinv, pi.q);
                d1 = f_to_canonical(__dadd_rn(f_mulmod(fb2, fa1, qa1, q), f_mulmod(fa2, fb1, qb1, q)), q, qinv, pi.q);
                d2 = f_to_canonical(f_mulmod(fb2, fb1, qb1, q), q, qinv, pi.q);
            };
            one(ua1.x, ub1.x, ua2.x, ub2.x, r0.x, r1.x, r2.x);
            one(ua1.y, ub1.y, ua2.y, ub2.y, r0.y, r1.y, r2.y);
            *reinterpret_cast<ulonglong2*>(t0 + x) = r0;
            if (d0k) *reinterpret_cast<ulonglong2*>(d0k + x) = r0;
            *reinterpret_cast<ulonglong2*>(t0 + x + LN) = r1;
            *reinterpret_cast<ulonglong2*>(t0 + x + 2 * LN) = r2;
        }
        return;
    }
    if (S == 1) {
        for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
             x += (long long)gridDim.x * blockDim.x) {
            const uint64_t va1 = a1[x], vb1 = b1[x], va2 = a2[x], vb2 = b2[x];
            t0[x] = mul_mod(va1, va2, pi);
            if (d0k) d0k[x] = t0[x];
            t0[x + LN] = add_mod(mul_mod(va1, vb2, pi), mul_mod(vb1, va2, pi), pi.q);
            t0[x + 2 * LN] = mul_mod(vb1, vb2, pi);
        }
        return;
    }
    const long long P = N / S;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x) {
        const int o = (int)(idx / P);
        const long long x = idx - o * P;
        t0[idx] = inc_prod_slot(a1, a2, S, P, x, o, pi);
        t0[idx + LN] = add_mod(inc_prod_slot(a1, b2, S, P, x, o, pi), inc_prod_slot(b1, a2, S, P, x, o, pi), pi.q);
        t0[idx + 2 * LN] = inc_prod_slot(b1, b2, S, P, x, o, pi);
    }
}

// acc[b][c][i] = -sum_j D[b][j][i] (*) K_b[j][c][i]   (gadget_mul_subto_polynomial, gadget.c:22-36;
// (*) the ring's incomplete product, pointwise at split 1)
// D: [B][nd][ne][N]; K_b: [digits][2][ne][N] (only the first nd digits are used);
// acc: [B][2][ne][N].  Thread index over N = (block o, slot x).
// order (may be null): ciphertext processed by the by-th group of rows, so that the
// ciphertexts sharing a key run back to back and the key stays in L2 between them.
template <int S>
__global__ void k_mac(uint64_t* __restrict__ acc, const uint64_t* __restrict__ D,
                      const uint64_t* const* __restrict__ keys, const uint64_t* __restrict__ order,
                      const __grid_constant__ LimbPrimes lp, const PrimeInfo* __restrict__ primes, int nd, int ne,
                      long long N) {
    const int by = blockIdx.y;
    const int bo = by / ne, i = by - bo * ne;
    const int b = order ? (int)order[bo] : bo;
    const PrimeInfo pi = primes[lp.p[i]];
    const uint64_t* key = keys[b];
    const long long dstride = (long long)ne * N;       // between digits of D
    const long long kstride = (long long)2 * ne * N;   // between digits of K
    const uint64_t* d = D + (long long)b * nd * dstride + (long long)i * N;
    const uint64_t* ka = key + (long long)i * N;
    const uint64_t* kb = ka + dstride;
    uint64_t* oa = acc + (long long)b * 2 * dstride + (long long)i * N;
    uint64_t* ob = oa + dstride;
    if (S == 1 && pi.fp64) {
        // pointwise products: the streaming loop, partial sums reduced every four digits
        const double q = pi.qd, qinv = pi.qinv;
        for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
             x += (long long)gridDim.x * blockDim.x) {
            double sa = 0.0, sb = 0.0;
            for (int j = 0; j < nd; ++j) {
                const double v = f_from_u64(d[j * dstride + x]);
                const double wa = f_from_u64(ka[j * kstride + x]);
                const double wb = f_from_u64(kb[j * kstride + x]);
                sa = __dadd_rn(sa, f_mulmod(v, wa, __dmul_rn(wa, qinv), q));
                sb = __dadd_rn(sb, f_mulmod(v, wb, __dmul_rn(wb, qinv), q));
                if ((j & 3) == 3) {
                    sa = f_reduce(sa, q, qinv);
                    sb = f_reduce(sb, q, qinv);
                }
            }
            oa[x] = f_to_canonical(-sa, q, qinv, pi.q);
            ob[x] = f_to_canonical(-sb, q, qinv, pi.q);
        }
        return;
    }
    if constexpr (S == 1) {
        // pointwise, primes of any size: 64-bit Barrett products
        for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
             x += (long long)gridDim.x * blockDim.x) {
            uint64_t sa = 0, sb = 0;
            for (int j = 0; j < nd; ++j) {
                const uint64_t v = d[j * dstride + x];
                sa = add_mod(sa, mul_mod(v, ka[j * kstride + x], pi), pi.q);
                sb = add_mod(sb, mul_mod(v, kb[j * kstride + x], pi), pi.q);
            }
            oa[x] = neg_mod(sa, pi.q);
            ob[x] = neg_mod(sb, pi.q);
        }
        return;
    }
    const long long P = N / S;
    if constexpr (S == 2 || S == 4) {
        if (pi.fp64) {
            for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < P;
                 x += (long long)gridDim.x * blockDim.x)
                mac_slots<S>(oa, ob, d, dstride, ka, kb, kstride, nd, P, x, pi);
            return;
        }
    }
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x) {
        const int o = (int)(idx / P);
        const long long x = idx - o * P;
        if (pi.fp64) mac_slot(oa, ob, d, dstride, ka, kb, kstride, nd, S, P, x, o, pi);
        else mac_slot_int(oa, ob, d, dstride, ka, kb, kstride, nd, S, P, x, o, pi);
    }
}

// Per coefficient: divide the key-switch accumulator by the special prime with
// rounding, add the pass-through component, and optionally rescale by the top prime.
// acc: [B][2][nl+1][N] coefficient domain; pass_c: [B][..][nl][N] rows at pass_off[c]
// (null = nothing to add); out: [B][2][nl or nl-1][N].
__global__ void k_moddown(uint64_t* __restrict__ out, const uint64_t* __restrict__ acc,
                          const uint64_t* __restrict__ pass, long long pass_stride, long long pass_off_a,
                          long long pass_off_b, int use_pass_a, int use_pass_b, const __grid_constant__ ModDownConsts mc,
                          const PrimeInfo* __restrict__ primes, int nl, int rescale, long long N) {
    const int by = blockIdx.y;
    const int b = by >> 1, c = by & 1;
    const int ne = nl + 1;
    const int nout = rescale ? nl - 1 : nl;
    const uint64_t* a = acc + ((long long)b * 2 + c) * ne * N;
    uint64_t* o = out + ((long long)b * 2 + c) * nout * N;
    const int use_pass = c == 0 ? use_pass_a : use_pass_b;
    const uint64_t* ps = use_pass ? pass + (long long)b * pass_stride + (c == 0 ? pass_off_a : pass_off_b) : nullptr;
    const PrimeInfo psp = primes[mc.special];
    const bool aligned = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(o) |
                           reinterpret_cast<uintptr_t>(ps ? ps : a)) & 15) == 0;
    if (mc.fp64 && aligned) {
        // exact FP64 form of the branch below: every intermediate is an integer below
        // 2^52, so no residue differs; two coefficients per thread, streaming loads
        for (long long x = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x); x < N;
             x += 2 * (long long)gridDim.x * blockDim.x) {
            const ulonglong2 sp = __ldcs(reinterpret_cast<const ulonglong2*>(a + (long long)nl * N + x));
            uint64_t t0 = sp.x + mc.half_p, t1 = sp.y + mc.half_p;
            t0 -= t0 >= mc.p ? mc.p : 0;
            t1 -= t1 >= mc.p ? mc.p : 0;
            const double td0 = f_from_u64(t0), td1 = f_from_u64(t1);
            // limb i after the special-prime division and the pass-through add, |v| < 7q/4
            auto limb2 = [&](int i, double& v0, double& v1) {
                const PrimeInfo& pi = primes[mc.prime[i]];
                const ulonglong2 av = __ldcs(reinterpret_cast<const ulonglong2*>(a + (long long)i * N + x));
                const double y0 = __dadd_rn(__dadd_rn(f_from_u64(av.x), mc.half_sp_d[i]), -td0);
                const double y1 = __dadd_rn(__dadd_rn(f_from_u64(av.y), mc.half_sp_d[i]), -td1);
                v0 = f_mulmod(y0, mc.inv_sp_d[i], mc.inv_sp_dq[i], pi.qd);
                v1 = f_mulmod(y1, mc.inv_sp_d[i], mc.inv_sp_dq[i], pi.qd);
                if (ps) {
                    const ulonglong2 pv = __ldcs(reinterpret_cast<const ulonglong2*>(ps + (long long)i * N + x));
                    v0 = __dadd_rn(v0, f_from_u64(pv.x));
                    v1 = __dadd_rn(v1, f_from_u64(pv.y));
                }
            };
            if (!rescale) {
#pragma unroll 2
                for (int i = 0; i < nl; ++i) {
                    const PrimeInfo& pi = primes[mc.prime[i]];
                    double v0, v1;
                    limb2(i, v0, v1);
                    ulonglong2 r;
                    r.x = f_to_canonical(v0, pi.qd, pi.qinv, pi.q);
                    r.y = f_to_canonical(v1, pi.qd, pi.qinv, pi.q);
                    *reinterpret_cast<ulonglong2*>(o + (long long)i * N + x) = r;
                }
            } else {
                const PrimeInfo& pt = primes[mc.prime[nl - 1]];
                double u0, u1;
                limb2(nl - 1, u0, u1);
                uint64_t s0 = f_to_canonical(u0, pt.qd, pt.qinv, pt.q) + mc.half_top;
                uint64_t s1 = f_to_canonical(u1, pt.qd, pt.qinv, pt.q) + mc.half_top;
                s0 -= s0 >= mc.q_top ? mc.q_top : 0;
                s1 -= s1 >= mc.q_top ? mc.q_top : 0;
                const double sd0 = f_from_u64(s0), sd1 = f_from_u64(s1);
#pragma unroll 2
                for (int i = 0; i < nl - 1; ++i) {
                    const PrimeInfo& pi = primes[mc.prime[i]];
                    double v0, v1;
                    limb2(i, v0, v1);
                    const double y0 = __dadd_rn(__dadd_rn(v0, mc.half_r_d[i]), -sd0);
                    const double y1 = __dadd_rn(__dadd_rn(v1, mc.half_r_d[i]), -sd1);
                    ulonglong2 r;
                    r.x = f_to_canonical(f_mulmod(y0, mc.inv_r_d[i], mc.inv_r_dq[i], pi.qd), pi.qd, pi.qinv, pi.q);
                    r.y = f_to_canonical(f_mulmod(y1, mc.inv_r_d[i], mc.inv_r_dq[i], pi.qd), pi.qd, pi.qinv, pi.q);
                    *reinterpret_cast<ulonglong2*>(o + (long long)i * N + x) = r;
                }
            }
        }
        return;
    }
    if (aligned) {
        // two coefficients per thread with 16-byte accesses; acc and the pass-through
        // rows are read once (streaming loads)
        for (long long x = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x); x < N;
             x += 2 * (long long)gridDim.x * blockDim.x) {
            const ulonglong2 sp = __ldcs(reinterpret_cast<const ulonglong2*>(a + (long long)nl * N + x));
            const uint64_t t0 = add_mod(sp.x, mc.half_p, mc.p), t1 = add_mod(sp.y, mc.half_p, mc.p);
            auto limb2 = [&](int i, unsigned long long& v0, unsigned long long& v1) {
                const PrimeInfo& pi = primes[mc.prime[i]];
                const ulonglong2 av = __ldcs(reinterpret_cast<const ulonglong2*>(a + (long long)i * N + x));
                v0 = shoup(sub_mod(add_mod(av.x, mc.half_sp[i], pi.q), reduce64(t0, pi), pi.q), mc.inv_sp[i],
                           mc.inv_sp_sh[i], pi.q);
                v1 = shoup(sub_mod(add_mod(av.y, mc.half_sp[i], pi.q), reduce64(t1, pi), pi.q), mc.inv_sp[i],
                           mc.inv_sp_sh[i], pi.q);
                if (ps) {
                    const ulonglong2 pv = __ldcs(reinterpret_cast<const ulonglong2*>(ps + (long long)i * N + x));
                    v0 = add_mod(v0, pv.x, pi.q);
                    v1 = add_mod(v1, pv.y, pi.q);
                }
            };
            if (!rescale) {
#pragma unroll 2
                for (int i = 0; i < nl; ++i) {
                    ulonglong2 r;
                    limb2(i, r.x, r.y);
                    *reinterpret_cast<ulonglong2*>(o + (long long)i * N + x) = r;
                }
            } else {
                unsigned long long u0, u1;
                limb2(nl - 1, u0, u1);
                const uint64_t s0 = add_mod(u0, mc.half_top, mc.q_top), s1 = add_mod(u1, mc.half_top, mc.q_top);
#pragma unroll 2
                for (int i = 0; i < nl - 1; ++i) {
                    const PrimeInfo& pi = primes[mc.prime[i]];
                    unsigned long long v0, v1;
                    limb2(i, v0, v1);
                    ulonglong2 r;
                    r.x = shoup(sub_mod(add_mod(v0, mc.half_r[i], pi.q), reduce64(s0, pi), pi.q), mc.inv_r[i],
                                mc.inv_r_sh[i], pi.q);
                    r.y = shoup(sub_mod(add_mod(v1, mc.half_r[i], pi.q), reduce64(s1, pi), pi.q), mc.inv_r[i],
                                mc.inv_r_sh[i], pi.q);
                    *reinterpret_cast<ulonglong2*>(o + (long long)i * N + x) = r;
                }
            }
        }
        return;
    }
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
         x += (long long)gridDim.x * blockDim.x) {
        const uint64_t t = add_mod(a[(long long)nl * N + x], mc.half_p, mc.p);
        // value of limb i after the special-prime division and the pass-through add
        auto limb = [&](int i) -> uint64_t {
            const PrimeInfo& pi = primes[mc.prime[i]];
            uint64_t v = add_mod(a[(long long)i * N + x], mc.half_sp[i], pi.q);
            v = sub_mod(v, reduce64(t, pi), pi.q);
            v = shoup(v, mc.inv_sp[i], mc.inv_sp_sh[i], pi.q);
            if (ps) v = add_mod(v, ps[(long long)i * N + x], pi.q);
            return v;
        };
        // unrolled so that several limbs' loads are in flight at once
        if (!rescale) {
#pragma unroll 4
            for (int i = 0; i < nl; ++i) o[(long long)i * N + x] = limb(i);
        } else {
            const uint64_t t2 = add_mod(limb(nl - 1), mc.half_top, mc.q_top);
#pragma unroll 4
            for (int i = 0; i < nl - 1; ++i) {
                const PrimeInfo& pi = primes[mc.prime[i]];
                uint64_t v = add_mod(limb(i), mc.half_r[i], pi.q);
                v = sub_mod(v, reduce64(t2, pi), pi.q);
                o[(long long)i * N + x] = shoup(v, mc.inv_r[i], mc.inv_r_sh[i], pi.q);
            }
        }
    }
    (void)psp;
}

constexpr int kColdownThreads = 128;

// The inverse transform's column pass (its last 2^K1-point stages, index bits KT..logP-1
// of each 2^logP-point block) of the key-switch accumulators, fused with k_moddown's
// FP64 form (k_moddown works coefficient by coefficient, so the split layout does not
// matter to it): thread (block column cx,
// ciphertext b, component c) finishes coefficients cx + m 2^KT of the special limb first
// and keeps (t + p/2) mod p of them, then (rescaling) finishes and divides the top limb
// and keeps its rounded value, then finishes, divides (and rescales) every output limb.
// The accumulator rows hold the tile pass's centred doubles; they are read once and the
// coefficient-domain accumulator never reaches HBM.  Per coefficient the operations are
// k_moddown's, in the same order, so the residues are the same.
template <int K1>
__global__ void __launch_bounds__(kColdownThreads, 6) k_coldown(uint64_t* __restrict__ out, const uint64_t* __restrict__ acc,
                                                 const uint64_t* __restrict__ pass, long long pass_stride,
                                                 long long pass_off_a, long long pass_off_b, int use_pass_a,
                                                 int use_pass_b, const __grid_constant__ ModDownConsts mc,
                                                 const PrimeInfo* __restrict__ primes, int nl, int rescale, long long N,
                                                 int logP, int KT) {
    constexpr int R = 1 << K1;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // block g >> KT, column g mod 2^KT
    if (g >= (N >> K1)) return;  // no barriers in this kernel
    const long long cx = ((g >> KT) << logP) + (g & ((1LL << KT) - 1));
    const int b = (int)(blockIdx.y >> 1), c = (int)(blockIdx.y & 1);
    const int ne = nl + 1;
    const int nout = rescale ? nl - 1 : nl;
    const uint64_t* a = acc + ((long long)b * 2 + c) * ne * N + cx;
    uint64_t* o = out + ((long long)b * 2 + c) * nout * N + cx;
    const int use_pass = c == 0 ? use_pass_a : use_pass_b;
    const uint64_t* ps = use_pass ? pass + (long long)b * pass_stride + (c == 0 ? pass_off_a : pass_off_b) + cx : nullptr;

    // limb `row` of the accumulator in the coefficient domain: canonical residues as doubles
    auto finish = [&](int row, const PrimeInfo& pi, double (&v)[R]) {
#pragma unroll
        for (int m = 0; m < R; ++m)
            v[m] = __longlong_as_double((long long)__ldcs(a + (long long)row * N + ((long long)m << KT)));
        col_inv_regs<K1>(v, pi, logP, KT);
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = f_from_u64(f_to_canonical(v[m], pi.qd, pi.qinv, pi.q));
    };
    // The special limb's (t + p/2) mod p and the rescale's rounded top limb stay in
    // shared memory, entry m of this thread at [m][threadIdx.x] (conflict-free), so the
    // registers hold one limb's column at a time.
    __shared__ double td[R][kColdownThreads], sd[R][kColdownThreads];
    const int tx = threadIdx.x;
    // limb i after the special-prime division and the pass-through add, |v| < 7q/4
    auto divide = [&](int i, double (&v)[R]) {
        const PrimeInfo& pi = primes[mc.prime[i]];
        finish(i, pi, v);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const double y = __dadd_rn(__dadd_rn(v[m], mc.half_sp_d[i]), -td[m][tx]);
            v[m] = f_mulmod(y, mc.inv_sp_d[i], mc.inv_sp_dq[i], pi.qd);
            if (ps) v[m] = __dadd_rn(v[m], f_from_u64(__ldcs(ps + (long long)i * N + ((long long)m << KT))));
        }
    };

    double v[R];
    {
        const PrimeInfo& psp = primes[mc.special];
        finish(nl, psp, v);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            uint64_t t = (uint64_t)v[m] + mc.half_p;
            t -= t >= mc.p ? mc.p : 0;
            td[m][tx] = f_from_u64(t);
        }
    }
    if (!rescale) {
        for (int i = 0; i < nl; ++i) {
            const PrimeInfo& pi = primes[mc.prime[i]];
            divide(i, v);
#pragma unroll
            for (int m = 0; m < R; ++m) o[(long long)i * N + ((long long)m << KT)] = f_to_canonical(v[m], pi.qd, pi.qinv, pi.q);
        }
        return;
    }
    {
        const PrimeInfo& pt = primes[mc.prime[nl - 1]];
        divide(nl - 1, v);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            uint64_t s = f_to_canonical(v[m], pt.qd, pt.qinv, pt.q) + mc.half_top;
            s -= s >= mc.q_top ? mc.q_top : 0;
            sd[m][tx] = f_from_u64(s);
        }
    }
    for (int i = 0; i < nl - 1; ++i) {
        const PrimeInfo& pi = primes[mc.prime[i]];
        divide(i, v);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const double y = __dadd_rn(__dadd_rn(v[m], mc.half_r_d[i]), -sd[m][tx]);
            o[(long long)i * N + ((long long)m << KT)] =
                f_to_canonical(f_mulmod(y, mc.inv_r_d[i], mc.inv_r_dq[i], pi.qd), pi.qd, pi.qinv, pi.q);
        }
    }
}

// Galois permutation of both components, per-ciphertext generator (rns_polynomial.c:996-1035:
// coefficient c moves to c gen mod 2N, negated when that is >= N; position k of block i
// holds coefficient i + k S at split degree S).  Written as a gather: output coefficient
// c' takes source coefficient p = c' gen^-1 mod 2N when p < N, and minus coefficient
// p - N otherwise (gen odd, so N gen = N mod 2N).  Stores are coalesced 16-byte pairs;
// the scattered 8-byte reads hit the source row in L2.  Index arithmetic is 32-bit
// (2N <= 2^31, so products wrap correctly modulo 2N).
__global__ void k_permute_batch(uint64_t* __restrict__ out, const uint64_t* __restrict__ in,
                                const uint64_t* __restrict__ ginvs, const __grid_constant__ LimbPrimes lp,
                                const PrimeInfo* __restrict__ primes, int L, long long N, int log_split) {
    const int by = blockIdx.y;  // (b, c, k)
    const int k = by % L;
    const int bc = by / L;
    const int b = bc >> 1;
    const uint64_t q = primes[lp.p[k]].q;
    const uint32_t ginv = (uint32_t)ginvs[b];
    const uint64_t* src = in + ((long long)bc * L + k) * N;
    uint64_t* dst = out + ((long long)bc * L + k) * N;
    const uint32_t n = (uint32_t)N, mask2n = 2 * n - 1;
    const uint32_t split = 1u << log_split;
    const int log_p = 31 - __clz((int)(n >> log_split));
    const uint32_t pmask = (n >> log_split) - 1;
    auto gather = [&](uint32_t d) -> uint64_t {
        const uint32_t cd = (d >> log_p) + ((d & pmask) << log_split);  // output coefficient
        const uint32_t p = (cd * ginv) & mask2n;
        const uint32_t c = p & (n - 1);
        const uint64_t v = src[((c & (split - 1)) << log_p) + (c >> log_split)];
        return p >= n ? neg_mod(v, q) : v;
    };
    for (uint32_t d = 2 * (blockIdx.x * blockDim.x + threadIdx.x); d < n; d += 2 * gridDim.x * blockDim.x) {
        ulonglong2 r;
        r.x = gather(d);
        r.y = gather(d + 1);
        *reinterpret_cast<ulonglong2*>(dst + d) = r;
    }
}

// k_mac at split 1 for FP64 primes, its operands staged through shared memory by bulk
// copies: block (chunk, pair, limb) walks the digits of kMacChunk residues of one
// extended limb for two ciphertexts that use the same key, and thread 0 keeps
// kMacStages digits (both ciphertexts' digit chunks and one copy of the two key chunks)
// in flight ahead of the one being multiplied; the digits stream from HBM, the keys
// mostly from L2, each key chunk once per pair.  Same result as k_mac<1>, which takes
// the shapes this kernel does not: N a multiple of kMacChunk and every row 16-byte
// aligned (checked by the launcher).  Against one ciphertext per block, the pairs cut
// the kernel's time by 12% (the key chunks' L2 traffic halves).
constexpr int kMacChunk = 512;   // residues per block: two per thread
constexpr int kMacStages = 4;    // digits in flight per block
constexpr int kMacStageWords = 4 * kMacChunk;  // two digit chunks, two key chunks
constexpr size_t kMacSmem = (size_t)kMacStages * kMacStageWords * 8;

__device__ int vc_mac_fault;  // nonzero: a staged MAC copy wait gave up

// Thread 0: request digit j's chunks of both ciphertexts (d1 null: one ciphertext) and
// both key chunks into stage j mod kMacStages.
__device__ __forceinline__ void mac2_issue(uint64_t* msm, uint64_t* bars, const uint64_t* d0, const uint64_t* d1,
                                           const uint64_t* ka, int j, long long dstride, long long kstride) {
    uint64_t* st = msm + (j % kMacStages) * kMacStageWords;
    uint64_t* bar = &bars[j % kMacStages];
    mbar_expect_tx(bar, (d1 ? 4 : 3) * kMacChunk * 8);
    bulk_load(st, d0 + j * dstride, kMacChunk * 8, bar);
    if (d1) bulk_load(st + kMacChunk, d1 + j * dstride, kMacChunk * 8, bar);
    bulk_load(st + 2 * kMacChunk, ka + j * kstride, kMacChunk * 8, bar);
    bulk_load(st + 3 * kMacChunk, ka + j * kstride + dstride, kMacChunk * 8, bar);
}

// acc_k = -sum_j D_j (*) key_j (+ fold) for one ciphertext's two residues at r.
__device__ __forceinline__ void mac2_store(uint64_t* acc, long long b, long long dstride, long long off, int i,
                                           double sa0, double sa1, double sb0, double sb1,
                                           const FoldConsts& fold, double q, double qinv, uint64_t qi) {
    sa0 = -sa0;
    sa1 = -sa1;
    sb0 = -sb0;
    sb1 = -sb1;
    if (fold.pass && i < fold.nl) {
        // + (P mod q_i) pass_i (|sum| <= 3.5q + 3q/4 < 2^52)
        const uint64_t* pa = fold.pass + b * fold.stride + off;
        const ulonglong2 da = *reinterpret_cast<const ulonglong2*>(pa);
        const ulonglong2 db = *reinterpret_cast<const ulonglong2*>(pa + fold.comp_stride);
        const double w = fold.pf[i], wq = fold.pfq[i];
        sa0 = __dadd_rn(sa0, f_mulmod(f_from_u64(da.x), w, wq, q));
        sa1 = __dadd_rn(sa1, f_mulmod(f_from_u64(da.y), w, wq, q));
        sb0 = __dadd_rn(sb0, f_mulmod(f_from_u64(db.x), w, wq, q));
        sb1 = __dadd_rn(sb1, f_mulmod(f_from_u64(db.y), w, wq, q));
    }
    ulonglong2 ra, rb;
    ra.x = f_to_canonical(sa0, q, qinv, qi);
    ra.y = f_to_canonical(sa1, q, qinv, qi);
    rb.x = f_to_canonical(sb0, q, qinv, qi);
    rb.y = f_to_canonical(sb1, q, qinv, qi);
    uint64_t* oa = acc + b * 2 * dstride + off;
    *reinterpret_cast<ulonglong2*>(oa) = ra;
    *reinterpret_cast<ulonglong2*>(oa + dstride) = rb;
}

// pairs[k] = b0 | (b1 + 1) << 32 (b1 = -1: b0 alone).
__global__ void __launch_bounds__(256) k_mac_paired(uint64_t* __restrict__ acc, const uint64_t* __restrict__ D,
                                                    const uint64_t* const* __restrict__ keys,
                                                    const uint64_t* __restrict__ pairs,
                                                    const __grid_constant__ LimbPrimes lp,
                                                    const PrimeInfo* __restrict__ primes, int nd, int ne,
                                                    long long N, const __grid_constant__ FoldConsts fold) {
    extern __shared__ __align__(128) uint64_t msm[];
    __shared__ uint64_t bars[kMacStages];
    const int by = blockIdx.y;
    const int bp = by / ne, i = by - bp * ne;
    const uint64_t pr = pairs[bp];
    const long long b0 = (long long)(pr & 0xffffffffULL);
    const long long b1 = (long long)(pr >> 32) - 1;
    const bool two = b1 >= 0;
    const long long x0 = (long long)blockIdx.x * kMacChunk;
    const long long dstride = (long long)ne * N;
    const long long kstride = (long long)2 * ne * N;
    const uint64_t* d0 = D + b0 * nd * dstride + (long long)i * N + x0;
    const uint64_t* d1 = two ? D + b1 * nd * dstride + (long long)i * N + x0 : nullptr;
    const uint64_t* ka = keys[b0] + (long long)i * N + x0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kMacStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        for (int j = 0; j < nd && j < kMacStages; ++j) mac2_issue(msm, bars, d0, d1, ka, j, dstride, kstride);
    }
    __syncthreads();
    const PrimeInfo& pi = primes[lp.p[i]];
    const double q = pi.qd, qinv = pi.qinv;
    const int r = 2 * threadIdx.x;
    double sa0 = 0.0, sb0 = 0.0, sa1 = 0.0, sb1 = 0.0;  // ciphertext b0
    double ta0 = 0.0, tb0 = 0.0, ta1 = 0.0, tb1 = 0.0;  // ciphertext b1
    for (int j = 0; j < nd; ++j) {
        const int s = j % kMacStages;
        mbar_wait_bounded(&bars[s], (uint32_t)((j / kMacStages) & 1), &vc_mac_fault);
        const uint64_t* st = msm + s * kMacStageWords;
        const ulonglong2 dv = *reinterpret_cast<const ulonglong2*>(st + r);
        const ulonglong2 ev = two ? *reinterpret_cast<const ulonglong2*>(st + kMacChunk + r) : make_ulonglong2(0, 0);
        const ulonglong2 av = *reinterpret_cast<const ulonglong2*>(st + 2 * kMacChunk + r);
        const ulonglong2 bv = *reinterpret_cast<const ulonglong2*>(st + 3 * kMacChunk + r);
        // each digit multiplies both key products (one quotient for two products;
        // uncentred operands below 2^50, each term |t| <= 3q/4)
        const double v0 = f_from_u64(dv.x), v1 = f_from_u64(dv.y);
        const double u0 = f_from_u64(ev.x), u1 = f_from_u64(ev.y);
        const double wa0 = f_from_u64(av.x), wa1 = f_from_u64(av.y);
        const double wb0 = f_from_u64(bv.x), wb1 = f_from_u64(bv.y);
        __syncthreads();  // every thread has read stage s: it may be refilled
        if (threadIdx.x == 0 && j + kMacStages < nd) {
            fence_proxy_async_smem();
            mac2_issue(msm, bars, d0, d1, ka, j + kMacStages, dstride, kstride);
        }
        const double vq0 = __dmul_rn(v0, qinv), vq1 = __dmul_rn(v1, qinv);
        sa0 = __dadd_rn(sa0, f_mulmod(wa0, v0, vq0, q));
        sa1 = __dadd_rn(sa1, f_mulmod(wa1, v1, vq1, q));
        sb0 = __dadd_rn(sb0, f_mulmod(wb0, v0, vq0, q));
        sb1 = __dadd_rn(sb1, f_mulmod(wb1, v1, vq1, q));
        if (two) {
            const double uq0 = __dmul_rn(u0, qinv), uq1 = __dmul_rn(u1, qinv);
            ta0 = __dadd_rn(ta0, f_mulmod(wa0, u0, uq0, q));
            ta1 = __dadd_rn(ta1, f_mulmod(wa1, u1, uq1, q));
            tb0 = __dadd_rn(tb0, f_mulmod(wb0, u0, uq0, q));
            tb1 = __dadd_rn(tb1, f_mulmod(wb1, u1, uq1, q));
        }
        if ((j & 3) == 3) {
            sa0 = f_reduce(sa0, q, qinv);
            sa1 = f_reduce(sa1, q, qinv);
            sb0 = f_reduce(sb0, q, qinv);
            sb1 = f_reduce(sb1, q, qinv);
            ta0 = f_reduce(ta0, q, qinv);
            ta1 = f_reduce(ta1, q, qinv);
            tb0 = f_reduce(tb0, q, qinv);
            tb1 = f_reduce(tb1, q, qinv);
        }
    }
    const long long off = (long long)i * N + x0 + r;
    mac2_store(acc, b0, dstride, off, i, sa0, sa1, sb0, sb1, fold, q, qinv, pi.q);
    if (two) mac2_store(acc, b1, dstride, off, i, ta0, ta1, tb0, tb1, fold, q, qinv, pi.q);
}

// One k_mac launch for the ring's split degree (each split degree is its own kernel,
// so the pointwise one keeps its small register footprint).
// keys_aligned: every key polynomial starts on a 16-byte boundary.
// pairs (device, npairs entries, see k_mac_paired): the staged kernel runs when they are
// given and its shape conditions hold (mac_staged_ok); k_mac otherwise.
void launch_mac(IncNtt* t, uint64_t* acc, const uint64_t* D, const uint64_t* const* keys, const uint64_t* order,
                const LimbPrimes& lpe, int nd, int ne, long long N, uint64_t B, cudaStream_t st, bool keys_aligned,
                const FoldConsts* fold = nullptr, const uint64_t* pairs = nullptr, uint64_t npairs = 0);

// Pairs of consecutive ciphertexts (in `order`, or 0..B-1) whose key pointers are
// equal, singles elsewhere, in k_mac_paired's encoding; returns the count.
uint64_t key_pairs(const uint64_t* const* keys, const uint64_t* order, uint64_t B, uint64_t* out) {
    uint64_t n = 0;
    for (uint64_t p = 0; p < B;) {
        const uint64_t b0 = order ? order[p] : p;
        if (p + 1 < B) {
            const uint64_t b1 = order ? order[p + 1] : p + 1;
            if (keys[b0] == keys[b1]) {
                out[n++] = b0 | ((b1 + 1) << 32);
                p += 2;
                continue;
            }
        }
        out[n++] = b0;
        p += 1;
    }
    return n;
}

// Whether launch_mac, given key pairs, takes the staged pointwise kernel (the only one
// that folds pass-through components): split 1, FP64 primes, aligned rows, N a multiple
// of the chunk.
bool mac_staged_ok(IncNtt* t, const uint64_t* acc, const uint64_t* D, const LimbPrimes& lpe, int ne, long long N,
                   bool keys_aligned);

// Grid for one launch of a per-coefficient kernel; every call site launches exactly
// one kernel with it, so it also counts the launch.
dim3 grid_xy(long long n, long long y) {
    note_launch();
    long long blocks = (n + 255) / 256;
    if (blocks > 64) blocks = 64;
    if (blocks < 1) blocks = 1;
    return dim3((unsigned)blocks, (unsigned)y, 1);
}

bool mac_staged_ok(IncNtt* t, const uint64_t* acc, const uint64_t* D, const LimbPrimes& lpe, int ne, long long N,
                   bool keys_aligned) {
    bool pointwise = t->pub.split_degree == 1 && keys_aligned && (N & 1) == 0 &&
                     ((reinterpret_cast<uintptr_t>(acc) | reinterpret_cast<uintptr_t>(D)) & 15) == 0;
    for (int i = 0; i < ne && pointwise; ++i) pointwise = t->info[lpe.p[i]].fp64 != 0;
    return pointwise && N % kMacChunk == 0 && prepare_ckks_kernels() == 0;
}

void launch_mac(IncNtt* t, uint64_t* acc, const uint64_t* D, const uint64_t* const* keys, const uint64_t* order,
                const LimbPrimes& lpe, int nd, int ne, long long N, uint64_t B, cudaStream_t st, bool keys_aligned,
                const FoldConsts* fold, const uint64_t* pairs, uint64_t npairs) {
    // (the callers that fold pass-through components check mac_staged_ok and pass pairs)
    if (pairs && npairs && mac_staged_ok(t, acc, D, lpe, ne, N, keys_aligned)) {
        note_launch();
        FoldConsts none;
        memset(&none, 0, sizeof none);
        const dim3 g((unsigned)(N / kMacChunk), (unsigned)(npairs * ne), 1);
        k_mac_paired<<<g, kMacChunk / 2, kMacSmem, st>>>(acc, D, keys, pairs, lpe, t->d_info, nd, ne, N,
                                                          fold ? *fold : none);
        return;
    }
    const dim3 g = grid_xy(N, (long long)B * ne);
    switch (t->pub.split_degree) {
        case 1: k_mac<1><<<g, 256, 0, st>>>(acc, D, keys, order, lpe, t->d_info, nd, ne, N); break;
        case 2: k_mac<2><<<g, 256, 0, st>>>(acc, D, keys, order, lpe, t->d_info, nd, ne, N); break;
        case 4: k_mac<4><<<g, 256, 0, st>>>(acc, D, keys, order, lpe, t->d_info, nd, ne, N); break;
        case 8: k_mac<8><<<g, 256, 0, st>>>(acc, D, keys, order, lpe, t->d_info, nd, ne, N); break;
        default: k_mac<16><<<g, 256, 0, st>>>(acc, D, keys, order, lpe, t->d_info, nd, ne, N); break;
    }
}

bool check_shape(IncNtt* t, const uint32_t* limbs, uint32_t L, uint32_t special, const char* where) {
    if (!t || !limbs || L == 0 || L + 1 > (uint32_t)kMaxLimbs) {
        set_error(where, "bad pool or limb list (1 <= nlimbs <= 63)");
        return false;
    }
    for (uint32_t k = 0; k < L; ++k)
        if (limbs[k] >= t->pub.l) {
            set_error(where, "limb index outside the pool");
            return false;
        }
    if (special >= t->pub.l) {
        set_error(where, "special prime outside the pool");
        return false;
    }
    return true;
}

// Forward transforms of every digit: D[b][j][i] = NTT(d_j mod q_i), reading digit
// rows from src (limb j at src + j N, polynomials src_stride apart).
// skip_diag: the rows i == j are already in D (k_tensor's dd) and are not transformed.
int digits_forward(IncNtt* t, uint64_t* D, const uint64_t* src, long long src_stride, uint64_t B,
                   const uint32_t* ext, int nd, int ne, cudaStream_t st, bool skip_diag = false) {
    const long long N = (long long)t->pub.N;
    for (int j = 0; j < nd; ++j) {
        RowSet rs;
        memset(&rs, 0, sizeof rs);
        int k = 0;
        for (int i = 0; i < ne; ++i) {
            if (skip_diag && i == j) continue;
            rs.in[k] = src + (long long)j * N;
            rs.out[k] = D + ((long long)j * ne + i) * N;
            rs.prime[k] = ext[i];
            ++k;
        }
        rs.nlimbs = k;
        rs.split = (int)t->pub.split_degree;
        rs.logP = t->logP;
        rs.batch = (int)B;
        rs.batch_stride = (long long)nd * ne * N;
        rs.in_batch_stride = src_stride;
        rs.reduce_input = 1;
        mark_fp64(rs, t);
        const int e = launch_ntt(rs, t->d_info, false, st);
        if (e) return e;
    }
    return 0;
}

// In-place transform of `count` consecutive [nl][N] blocks with the given limb primes.
int blocks_transform(IncNtt* t, uint64_t* data, uint64_t count, const uint32_t* lim, int nl, bool inverse,
                     cudaStream_t st) {
    const long long N = (long long)t->pub.N;
    RowSet rs;
    memset(&rs, 0, sizeof rs);
    for (int i = 0; i < nl; ++i) {
        rs.in[i] = data + (long long)i * N;
        rs.out[i] = data + (long long)i * N;
        rs.prime[i] = lim[i];
    }
    rs.nlimbs = nl;
    rs.split = (int)t->pub.split_degree;
    rs.logP = t->logP;
    rs.batch = (int)count;
    rs.batch_stride = (long long)nl * N;
    rs.in_batch_stride = rs.batch_stride;
    mark_fp64(rs, t);
    return launch_ntt(rs, t->d_info, inverse, st);
}

// In-place transform of the first [nl][N] block of `count` polynomials `stride` apart.
int strided_transform(IncNtt* t, uint64_t* data, uint64_t count, long long stride, const uint32_t* lim, int nl,
                      bool inverse, cudaStream_t st) {
    const long long N = (long long)t->pub.N;
    RowSet rs;
    memset(&rs, 0, sizeof rs);
    for (int i = 0; i < nl; ++i) {
        rs.in[i] = data + (long long)i * N;
        rs.out[i] = data + (long long)i * N;
        rs.prime[i] = lim[i];
    }
    rs.nlimbs = nl;
    rs.split = (int)t->pub.split_degree;
    rs.logP = t->logP;
    rs.batch = (int)count;
    rs.batch_stride = stride;
    rs.in_batch_stride = stride;
    mark_fp64(rs, t);
    return launch_ntt(rs, t->d_info, inverse, st);
}

// ---- batched RLWE encryption (mlwe_RNSc_sample, modules/mlwe/c/src/mlwe.c:190-241)
//
// Four rounded Gaussians of width sigma from ChaCha20 block `ctr` of the Gaussian stream
// (Box-Muller on two 53-bit uniforms each, rounded: generate_normal_random and
// polynomial_gen_gaussian_RNSc_polynomial, misc_tp.c:26-33, rns_polynomial.c:255-271).
__device__ __forceinline__ void gaussian4(const PrngKey& key, uint64_t ctr, double sigma, int64_t ev[4]) {
    uint32_t blk[16];
    chacha20_block(key, ctr, kStreamGaussian, blk);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        ev[k] = (int64_t)llrint(sigma * sqrt(-2.0 * log(unit_open_low(block_u64(blk, 2 * k)))) *
                                cospi(2.0 * unit_closed_low(block_u64(blk, 2 * k + 1))));
}

// out [B][2][L][N]: the a rows are drawn uniform (polynomial_gen_random_RNSc_polynomial,
// rns_polynomial.c:242-253) and, with E, the b rows receive the rounded Gaussian integer
// of each coefficient reduced into every limb (polynomial_gen_gaussian_RNSc_polynomial,
// rns_polynomial.c:255-271).  Uniform residues are uniform in either domain (the
// transform is a bijection), so the same draw serves as a's coefficients or as its
// transform.  The reference reduces one 64-bit word per residue with a small bias;
// here the reduction is exact (uniform_mod64 with redraws).
//
// Replacement for a rejected uniform_mod64 draw: the first accepted of the eight 64-bit
// words of redraw-stream block `ctr`.  If all eight are rejected (probability below
// 2^-112 for the primes here) the first draw's hi(r q), `first`, which is in [0, q), is
// kept.  Out of line, so that the common path keeps its draws in registers.
__device__ __noinline__ uint64_t uniform_redraw(const PrngKey& key, uint64_t ctr, uint64_t q, uint64_t thresh,
                                                uint64_t first) {
    uint32_t blk[16];
    chacha20_block(key, ctr, kStreamUniformRedraw, blk);
    for (int w = 0; w < 8; ++w) {
        uint64_t r;
        if (uniform_mod64(block_u64(blk, w), q, thresh, r)) return r;
    }
    return first;
}

// ChaCha20 blocks: Gaussian g0 + b ceil(N/4) + c for coefficients 4c..4c+3 (the layout
// k_encrypt_noise_msg reads), uniform u0 + (b L + i) ceil(N/8) + j for coefficients
// 8j..8j+7 of limb i (one 64-bit word each), and the redraw of coefficient 8j + k at
// counter u0 + 8 ((b L + i) ceil(N/8) + j) + k of the redraw stream.
template <bool E>
__global__ void k_encrypt_sample(uint64_t* __restrict__ out, const __grid_constant__ LimbPrimes lp,
                                 const PrimeInfo* __restrict__ primes, int L, long long N, double sigma,
                                 const __grid_constant__ PrngKey key, uint64_t g0, uint64_t u0) {
    const long long b = blockIdx.y;
    const long long per4 = (N + 3) / 4, per8 = (N + 7) / 8;
    uint64_t* a = out + b * 2 * L * N;
    uint64_t* e = a + (long long)L * N;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < per8;
         j += (long long)gridDim.x * blockDim.x) {
        int64_t ev[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (E) {
            gaussian4(key, g0 + (uint64_t)(b * per4 + 2 * j), sigma, ev);
            if (2 * j + 1 < per4) gaussian4(key, g0 + (uint64_t)(b * per4 + 2 * j + 1), sigma, ev + 4);
        }
        for (int i = 0; i < L; ++i) {
            const PrimeInfo& pi = primes[lp.p[i]];
            const uint64_t thresh = reduce64((uint64_t)0 - pi.q, pi);  // 2^64 mod q
            const uint64_t idx = (uint64_t)((b * L + i) * per8 + j);
            uint32_t blk[16];
            chacha20_block(key, u0 + idx, kStreamUniform, blk);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const long long x = 8 * j + k;
                if (x >= N) break;
                uint64_t v;
                if (!uniform_mod64(block_u64(blk, k), pi.q, thresh, v))
                    v = uniform_redraw(key, u0 + 8 * idx + (uint64_t)k, pi.q, thresh, v);
                a[(long long)i * N + x] = v;
                if (E) e[(long long)i * N + x] = reduce_signed(ev[k], pi);
            }
        }
    }
}

// b = e + s a in the NTT domain: the ring's incomplete product over S blocks of P
// slots (rns_polynomial.c:358-396), with the key broadcast to every ciphertext.
// NOISE: b <- b + a s, with a in the a rows and b holding the transformed noise.
// Otherwise b <- b s in place, with b holding a's transform: each thread reads the S
// residues of its position x in every block before it writes them.
template <int S, bool NOISE>
__global__ void k_encrypt_combine(uint64_t* __restrict__ out, const uint64_t* __restrict__ sk,
                                  const __grid_constant__ LimbPrimes lp, const PrimeInfo* __restrict__ primes, int L,
                                  long long N) {
    const long long b = blockIdx.y / L;
    const int i = blockIdx.y - (int)(b * L);
    const PrimeInfo pi = primes[lp.p[i]];
    const uint64_t q = pi.q;
    const long long P = N / S;
    uint64_t* eb = out + (b * 2 * L + L + i) * N;
    const uint64_t* a = NOISE ? out + (b * 2 * L + i) * N : eb;
    const uint64_t* s = sk + (long long)i * N;
    if (S == 1 && pi.fp64 && (N & 1) == 0 &&
        ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(eb) | reinterpret_cast<uintptr_t>(s)) & 15) ==
            0) {
        // exact FP64 products (canonical operands below 2^50, uncentred multiplier s with
        // fl(s qinv) as its quotient estimate: |a s - n q| < q), two residues per thread
        const double qd = pi.qd, qinv = pi.qinv;
        for (long long x = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x); x < N;
             x += 2 * (long long)gridDim.x * blockDim.x) {
            const ulonglong2 ua = *reinterpret_cast<const ulonglong2*>(a + x);
            const ulonglong2 us = __ldg(reinterpret_cast<const ulonglong2*>(s + x));
            const double s0 = f_from_u64(us.x), s1 = f_from_u64(us.y);
            double t0 = f_mulmod(f_from_u64(ua.x), s0, __dmul_rn(s0, qinv), qd);
            double t1 = f_mulmod(f_from_u64(ua.y), s1, __dmul_rn(s1, qinv), qd);
            if (NOISE) {
                const ulonglong2 ue = *reinterpret_cast<const ulonglong2*>(eb + x);
                t0 = __dadd_rn(t0, f_from_u64(ue.x));
                t1 = __dadd_rn(t1, f_from_u64(ue.y));
            }
            ulonglong2 r;
            r.x = f_to_canonical(t0, qd, qinv, pi.q);
            r.y = f_to_canonical(t1, qd, qinv, pi.q);
            *reinterpret_cast<ulonglong2*>(eb + x) = r;
        }
        return;
    }
    const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(pi.twist);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < P;
         x += (long long)gridDim.x * blockDim.x) {
        uint64_t av[S], sv[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            av[j] = a[j * P + x];
            sv[j] = s[j * P + x];
        }
#pragma unroll
        for (int o = 0; o < S; ++o) {
            uint64_t acc = 0, wrap = 0;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                if (j <= o) acc = add_mod(acc, mul_mod(sv[j], av[o - j], pi), q);
                else wrap = add_mod(wrap, mul_mod(sv[j], av[o - j + S], pi), q);
            }
            if (S > 1) {
                const ulonglong2 w = tw[x];
                acc = add_mod(acc, shoup(wrap, w.x, w.y, q), q);
            }
            eb[o * P + x] = NOISE ? add_mod(eb[o * P + x], acc, q) : acc;
        }
    }
}

// b <- b + e + m in the coefficient domain: the four rounded Gaussians of block j
// (the same stream positions k_encrypt_sample<true> uses) reduced into every limb, and
// the message rows when given.
__global__ void k_encrypt_noise_msg(uint64_t* __restrict__ out, const uint64_t* __restrict__ msg,
                                    const __grid_constant__ LimbPrimes lp, const PrimeInfo* __restrict__ primes, int L,
                                    long long N, double sigma, const __grid_constant__ PrngKey key, uint64_t g0) {
    const long long b = blockIdx.y;
    const long long per = (N + 3) / 4;
    uint64_t* eb = out + (b * 2 * L + L) * N;
    const uint64_t* m = msg ? msg + b * L * N : nullptr;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < per;
         j += (long long)gridDim.x * blockDim.x) {
        int64_t ev[4];
        gaussian4(key, g0 + (uint64_t)(b * per + j), sigma, ev);
        for (int i = 0; i < L; ++i) {
            const PrimeInfo& pi = primes[lp.p[i]];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const long long x = 4 * j + k;
                if (x >= N) break;
                uint64_t v = add_mod(eb[(long long)i * N + x], reduce_signed(ev[k], pi), pi.q);
                if (m) v = add_mod(v, m[(long long)i * N + x], pi.q);
                eb[(long long)i * N + x] = v;
            }
        }
    }
}

// Gadget messages of a key-switching key, added in the NTT domain: digit d = j L + i of
// source polynomial j gets factor_i * src_j (limb i only) in its b row
// (_gen_ksk_components, modules/mlwe/python/src/vfhe/mlwe/mlwe.py:145-177: the message
// poly_j * (P mod q_i) e_i, whose transform is factor_i times the limb-i transform).
struct GadgetFactors {
    uint64_t f[kMaxLimbs];
};

__global__ void k_gadget_add(uint64_t* __restrict__ out, const uint64_t* __restrict__ src,
                             const __grid_constant__ GadgetFactors gf, const __grid_constant__ LimbPrimes lp,
                             const PrimeInfo* __restrict__ primes, int L, long long N) {
    const long long d = blockIdx.y;
    const long long j = d / L;
    const int i = (int)(d - j * L);
    const PrimeInfo pi = primes[lp.p[i]];
    uint64_t* b = out + (d * 2 + 1) * L * N + (long long)i * N;
    const uint64_t* sr = src + (j * L + i) * N;
    const uint64_t f = gf.f[i] % pi.q;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
         x += (long long)gridDim.x * blockDim.x)
        b[x] = add_mod(b[x], mul_mod(sr[x], f, pi), pi.q);
}

__global__ void k_prng_blocks(uint32_t* __restrict__ out, uint64_t nblocks, const __grid_constant__ PrngKey key,
                              uint64_t counter0, uint64_t nonce) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nblocks;
         j += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t blk[16];
        chacha20_block(key, counter0 + j, nonce, blk);
#pragma unroll
        for (int k = 0; k < 16; ++k) out[j * 16 + k] = blk[k];
    }
}


}  // namespace

int prepare_ckks_kernels() {
    static std::once_flag once;
    static int err = 0;
    std::call_once(once, [] {
        err = (int)cudaFuncSetAttribute(k_mac_paired, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMacSmem);
    });
    return err;
}

int read_mac_fault(int* out) {
    return (int)cudaMemcpyFromSymbol(out, vc_mac_fault, sizeof(int));
}

int clear_mac_fault() {
    const int zero = 0;
    return (int)cudaMemcpyToSymbol(vc_mac_fault, &zero, sizeof(int));
}

namespace {
// Self-check of the bounded wait: one thread arms an mbarrier for 16 bytes that no copy
// will ever deliver and waits on it with the same bounded retry loop the staged kernels
// use, so the wait must give up, set vc_mac_fault and return.  No copy is issued, so
// nothing can land in shared memory after the block exits.
__global__ void k_bounded_wait_selfcheck(int tries, int* gave_up) {
    __shared__ uint64_t bar;
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_expect_tx(&bar, 16);
    int i = 0;
    while (i < tries && !mbar_try_wait(&bar, 0)) ++i;
    if (i == tries) {
        atomicExch(&vc_mac_fault, 1);
        *gave_up = 1;
    }
}
}  // namespace

int bounded_wait_selfcheck(int tries, int* gave_up_host) {
    int* d = nullptr;
    int e = (int)cudaMalloc(&d, sizeof(int));
    if (e) return e;
    e = (int)cudaMemset(d, 0, sizeof(int));
    if (!e) {
        k_bounded_wait_selfcheck<<<1, 1>>>(tries, d);
        e = (int)cudaGetLastError();
    }
    if (!e) e = (int)cudaMemcpy(gave_up_host, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e;
}

ModDownConsts moddown_consts(IncNtt* t, const uint32_t* limbs, int nl, uint32_t special) {
    ModDownConsts mc;
    memset(&mc, 0, sizeof mc);
    const uint64_t p = t->info[special].q;
    mc.special = special;
    mc.p = p;
    mc.half_p = p / 2;
    const uint64_t qt = t->info[limbs[nl - 1]].q;
    mc.q_top = qt;
    mc.half_top = qt / 2;
    for (int i = 0; i < nl; ++i) {
        const uint64_t q = t->info[limbs[i]].q;
        mc.prime[i] = limbs[i];
        mc.half_sp[i] = (p / 2) % q;
        mc.inv_sp[i] = host_inv_mod(p % q, q);
        mc.inv_sp_sh[i] = host_shoup(mc.inv_sp[i], q);
        mc.half_r[i] = (qt / 2) % q;
        mc.inv_r[i] = host_inv_mod(qt % q, q);
        mc.inv_r_sh[i] = host_shoup(mc.inv_r[i], q);
    }
    mc.fp64 = p < (1ULL << 50);
    for (int i = 0; i < nl; ++i) {
        const uint64_t q = t->info[limbs[i]].q;
        mc.fp64 = mc.fp64 && q < (1ULL << 50);
        auto centred = [q](uint64_t w) { return w > q / 2 ? (double)w - (double)q : (double)w; };
        mc.half_sp_d[i] = (double)mc.half_sp[i];
        mc.inv_sp_d[i] = centred(mc.inv_sp[i]);
        mc.inv_sp_dq[i] = mc.inv_sp_d[i] / (double)q;
        mc.half_r_d[i] = (double)mc.half_r[i];
        mc.inv_r_d[i] = centred(mc.inv_r[i]);
        mc.inv_r_dq[i] = mc.inv_r_d[i] / (double)q;
    }
    return mc;
}

uint64_t ckks_mul_ws_elems(uint64_t N, uint64_t B, uint64_t L) {
    const uint64_t ne = L + 1;
    return B * N * (3 * L + L * ne + 2 * ne) + 2 * B + 64;
}

uint64_t ckks_rot_ws_elems(uint64_t N, uint64_t B, uint64_t L) {
    const uint64_t ne = L + 1;
    return B * N * (2 * L + L * ne + 2 * ne) + 4 * B + 64;
}

namespace {
// VFHE_CUDA_CKKS_UNFUSED=1: the whole inverse transform, then k_moddown (the fused and
// unfused forms give the same residues; tests compare them)
bool coldown_disabled() {
    const char* s = getenv("VFHE_CUDA_CKKS_UNFUSED");
    return s && atoi(s) != 0;
}

// Inverse transform of the key-switch accumulators [B][2][ne][N] (in place; limbs
// ext[0..ne-1], the special prime last) and the special-prime division (+ pass-through,
// + rescale by ext[ne-2]) into out.  Where every prime takes the FP64 form and the
// transform's schedule is a tile pass plus a column pass of at most 16 points, the
// column pass runs inside the division (k_coldown); otherwise the whole transform runs
// and then k_moddown.
int acc_inverse_moddown(IncNtt* t, uint64_t* out, uint64_t* acc, uint64_t B, const uint32_t* ext, int ne,
                        const ModDownConsts& mc, const uint64_t* pass, long long pass_stride, long long off_a,
                        long long off_b, int use_a, int use_b, int rescale, cudaStream_t st) {
    const long long N = (long long)t->pub.N;
    const int nl = ne - 1;
    if (mc.fp64 && !coldown_disabled()) {
        RowSet rs;
        memset(&rs, 0, sizeof rs);
        for (int i = 0; i < ne; ++i) {
            rs.in[i] = acc + (long long)i * N;
            rs.out[i] = acc + (long long)i * N;
            rs.prime[i] = ext[i];
        }
        rs.nlimbs = ne;
        rs.split = (int)t->pub.split_degree;
        rs.logP = t->logP;
        rs.batch = (int)(2 * B);
        rs.batch_stride = (long long)ne * N;
        rs.in_batch_stride = rs.batch_stride;
        mark_fp64(rs, t);
        int K1 = 0, KT = 0;
        const int e = launch_ntt_f64_inverse_tiles(rs, t->d_info, 4, &K1, &KT, st);
        if (e != kTilePassUnavailable) {
            if (e) return e;
            const dim3 g((unsigned)(((N >> K1) + kColdownThreads - 1) / kColdownThreads), (unsigned)(2 * B), 1);
            note_launch();
#define VC_COLDOWN(K1V)                                                                                          \
    k_coldown<K1V><<<g, kColdownThreads, 0, st>>>(out, acc, pass, pass_stride, off_a, off_b, use_a, use_b, mc, t->d_info, nl, \
                                      rescale, N, t->logP, KT)
            switch (K1) {
                case 1: VC_COLDOWN(1); break;
                case 2: VC_COLDOWN(2); break;
                case 3: VC_COLDOWN(3); break;
                default: VC_COLDOWN(4); break;
            }
#undef VC_COLDOWN
            return (int)cudaGetLastError();
        }
    }
    const int e = blocks_transform(t, acc, 2 * B, ext, ne, true, st);
    if (e) return e;
    k_moddown<<<grid_xy((N + 1) / 2, (long long)B * 2), 256, 0, st>>>(out, acc, pass, pass_stride, off_a, off_b, use_a,
                                                                    use_b, mc, t->d_info, nl, rescale, N);
    return (int)cudaGetLastError();
}
}  // namespace

int mac_one_sample(IncNtt* t, uint64_t* acc, const uint64_t* D, const uint64_t* keys, uint64_t* keyptr,
                   const uint32_t* ext, int nd, int ne, cudaStream_t st) {
    LimbPrimes lpe;
    memset(&lpe, 0, sizeof lpe);
    for (int i = 0; i < ne; ++i) lpe.p[i] = ext[i];
    const uint64_t kp = (uint64_t)(uintptr_t)keys;
    const int e = upload_small(keyptr, &kp, 1, st);
    if (e) return e;
    const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
    launch_mac(t, acc, D, (const uint64_t* const*)keyptr, nullptr, lpe, nd, ne, (long long)t->pub.N, 1, st, aligned,
               nullptr, nullptr, 0);
    return (int)cudaGetLastError();
}

int ckks_mul_relin_rescale(IncNtt* t, uint64_t* out, const uint64_t* ct1, const uint64_t* ct2, uint64_t B,
                           const uint32_t* limbs, uint32_t L, uint32_t special, const uint64_t* rlk,
                           uint64_t* ws, cudaStream_t st) {
    const char* where = "vfhe_cuda_ckks_mul_relin_rescale_batch";
    if (!check_shape(t, limbs, L, special, where)) return 1;
    if (L < 2) {
        set_error(where, "rescaling needs at least two limbs");
        return 1;
    }
    const long long N = (long long)t->pub.N;
    const int nl = (int)L, ne = nl + 1;
    uint32_t ext[kMaxLimbs];
    for (int i = 0; i < nl; ++i) ext[i] = limbs[i];
    ext[nl] = special;
    LimbPrimes lp, lpe;
    memset(&lp, 0, sizeof lp);
    memset(&lpe, 0, sizeof lpe);
    for (int i = 0; i < nl; ++i) lp.p[i] = limbs[i];
    for (int i = 0; i < ne; ++i) lpe.p[i] = ext[i];

    uint64_t* T = ws;                                   // [B][3][L][N]
    uint64_t* D = T + B * 3 * nl * N;                   // [B][L][ne][N]
    uint64_t* acc = D + B * (uint64_t)nl * ne * N;      // [B][2][ne][N]
    uint64_t* keyptrs = acc + B * 2 * ne * N;           // [B]

    uint64_t* d_pairs = keyptrs + B;                    // [B]
    std::vector<const uint64_t*> kp(B, rlk);
    if (!check_cuda(upload_small(keyptrs, (const uint64_t*)kp.data(), B, st), where)) return 1;
    const bool rlk_aligned = (reinterpret_cast<uintptr_t>(rlk) & 15) == 0;
    // When the staged MAC runs: d1 and d2 pass through the key switch and stay in the
    // NTT domain, folded into the accumulator (FoldConsts), so only d0 -- whose limbs are
    // the digits -- goes back to the coefficient domain; and the spectrum of digit j
    // modulo its own prime is d0's limb j itself, which the tensor kernel writes into the
    // digit buffer, so those nl digit rows are not transformed.
    const bool fold = mac_staged_ok(t, acc, D, lpe, ne, N, rlk_aligned) &&
                      (reinterpret_cast<uintptr_t>(T) & 15) == 0 && (N & 1) == 0;
    const bool diag = fold;
    switch (t->pub.split_degree) {
        case 1:  // the FP64 path takes two coefficients per thread
            k_tensor<1><<<grid_xy((N + 1) / 2, (long long)B * nl), 256, 0, st>>>(T, ct1, ct2, lp, t->d_info, nl, N,
                                                                              diag ? D : nullptr, (long long)nl * ne * N,
                                                                              (long long)(ne + 1) * N);
            break;
        case 2: k_tensor<2><<<grid_xy(N, (long long)B * nl), 256, 0, st>>>(T, ct1, ct2, lp, t->d_info, nl, N, nullptr, 0, 0); break;
        case 4: k_tensor<4><<<grid_xy(N, (long long)B * nl), 256, 0, st>>>(T, ct1, ct2, lp, t->d_info, nl, N, nullptr, 0, 0); break;
        case 8: k_tensor<8><<<grid_xy(N, (long long)B * nl), 256, 0, st>>>(T, ct1, ct2, lp, t->d_info, nl, N, nullptr, 0, 0); break;
        default: k_tensor<16><<<grid_xy(N, (long long)B * nl), 256, 0, st>>>(T, ct1, ct2, lp, t->d_info, nl, N, nullptr, 0, 0); break;
    }
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    if (fold) {
        if (!check_cuda(strided_transform(t, T, B, 3LL * nl * N, limbs, nl, true, st), where)) return 1;
    } else {
        if (!check_cuda(blocks_transform(t, T, 3 * B, limbs, nl, true, st), where)) return 1;
    }
    if (!check_cuda(digits_forward(t, D, T, 3LL * nl * N, B, ext, nl, ne, st, diag), where)) return 1;
    FoldConsts fc;
    memset(&fc, 0, sizeof fc);
    if (fold) {
        fc.pass = T + (long long)nl * N;
        fc.stride = 3LL * nl * N;
        fc.comp_stride = (long long)nl * N;
        fc.nl = nl;
        const uint64_t P = t->info[special].q;
        for (int i = 0; i < nl; ++i) {
            const uint64_t q = t->info[limbs[i]].q;
            const uint64_t r = P % q;
            fc.pf[i] = r > q / 2 ? (double)r - (double)q : (double)r;
            fc.pfq[i] = fc.pf[i] / (double)q;
        }
    }
    // every ciphertext uses the relinearisation key: pairs (0, 1), (2, 3), ...
    std::vector<uint64_t> pairs(B);
    const uint64_t npairs = key_pairs(kp.data(), nullptr, B, pairs.data());
    if (!check_cuda(upload_small(d_pairs, pairs.data(), npairs, st), where)) return 1;
    launch_mac(t, acc, D, (const uint64_t* const*)keyptrs, nullptr, lpe, nl, ne, N, B, st, rlk_aligned,
               fold ? &fc : nullptr, d_pairs, npairs);
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    const ModDownConsts mc = moddown_consts(t, limbs, nl, special);
    const int use_pass = fold ? 0 : 1;
    return check_cuda(acc_inverse_moddown(t, out, acc, B, ext, ne, mc, T, 3LL * nl * N, (long long)nl * N,
                                          2LL * nl * N, use_pass, use_pass, 1, st),
                      where)
               ? 0
               : 1;
}

// gens == nullptr: a plain key switch of every ciphertext (no automorphism); the
// digits and the pass-through b are read from ct itself.
int ckks_rotate(IncNtt* t, uint64_t* out, const uint64_t* ct, uint64_t B, const uint32_t* limbs, uint32_t L,
                uint32_t special, const uint64_t* gens, const uint64_t* const* gks, uint64_t* ws, cudaStream_t st) {
    const char* where = gens ? "vfhe_cuda_ckks_rotate_batch" : "vfhe_cuda_keyswitch_batch";
    if (!check_shape(t, limbs, L, special, where)) return 1;
    const long long N = (long long)t->pub.N;
    if (gens && N > (1LL << 30)) {
        set_error(where, "rotation needs N <= 2^30");
        return 1;
    }
    if (gens)
        for (uint64_t b = 0; b < B; ++b)
            if ((gens[b] & 1) == 0 || gens[b] >= 2 * (uint64_t)N) {
                set_error(where, "Galois elements must be odd and below 2N");
                return 1;
            }
    const int nl = (int)L, ne = nl + 1;
    uint32_t ext[kMaxLimbs];
    for (int i = 0; i < nl; ++i) ext[i] = limbs[i];
    ext[nl] = special;
    LimbPrimes lp, lpe;
    memset(&lp, 0, sizeof lp);
    memset(&lpe, 0, sizeof lpe);
    for (int i = 0; i < nl; ++i) lp.p[i] = limbs[i];
    for (int i = 0; i < ne; ++i) lpe.p[i] = ext[i];
    int ls = 0;
    while ((1ULL << ls) < t->pub.split_degree) ++ls;

    uint64_t* Pm = ws;                                  // [B][2][L][N]
    uint64_t* D = Pm + B * 2 * nl * N;                  // [B][L][ne][N]
    uint64_t* acc = D + B * (uint64_t)nl * ne * N;      // [B][2][ne][N]
    uint64_t* keyptrs = acc + B * 2 * ne * N;           // [B]
    uint64_t* d_gens = keyptrs + B;                     // [B]
    uint64_t* d_order = d_gens + B;                     // [B]
    uint64_t* d_pairs = d_order + B;                    // [B]
    if (!check_cuda(upload_small(keyptrs, (const uint64_t*)gks, B, st), where)) return 1;
    // ciphertexts grouped by key (stable), so each key is read from HBM about once
    std::vector<uint64_t> order(B);
    for (uint64_t b = 0; b < B; ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [gks](uint64_t x, uint64_t y) {
        return reinterpret_cast<uintptr_t>(gks[x]) < reinterpret_cast<uintptr_t>(gks[y]);
    });
    bool identity = true;
    for (uint64_t b = 0; b < B && identity; ++b) identity = order[b] == b;
    if (!identity && !check_cuda(upload_small(d_order, order.data(), B, st), where)) return 1;
    const uint64_t* src = ct;
    if (gens) {
        // the gather needs gen^-1 mod 2N (Newton's iteration doubles the correct low bits)
        std::vector<uint64_t> ginv(B);
        for (uint64_t b = 0; b < B; ++b) {
            uint64_t x = gens[b];
            for (int it = 0; it < 6; ++it) x *= 2 - gens[b] * x;
            ginv[b] = x & (2 * (uint64_t)N - 1);
        }
        if (!check_cuda(upload_small(d_gens, ginv.data(), B, st), where)) return 1;
        k_permute_batch<<<grid_xy((N + 1) / 2, (long long)B * 2 * nl), 256, 0, st>>>(Pm, ct, d_gens, lp, t->d_info, nl,
                                                                                N, ls);
        if (!check_cuda(cudaGetLastError(), where)) return 1;
        src = Pm;
    }
    if (!check_cuda(digits_forward(t, D, src, 2LL * nl * N, B, ext, nl, ne, st), where)) return 1;
    bool keys_aligned = true;
    for (uint64_t b = 0; b < B; ++b) keys_aligned = keys_aligned && (reinterpret_cast<uintptr_t>(gks[b]) & 15) == 0;
    // ciphertexts that share a Galois key (adjacent in the key-grouped order) in pairs
    std::vector<uint64_t> pairs(B);
    const uint64_t npairs = key_pairs(gks, order.data(), B, pairs.data());
    if (!check_cuda(upload_small(d_pairs, pairs.data(), npairs, st), where)) return 1;
    launch_mac(t, acc, D, (const uint64_t* const*)keyptrs, identity ? nullptr : d_order, lpe, nl, ne, N, B, st,
               keys_aligned, nullptr, d_pairs, npairs);
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    const ModDownConsts mc = moddown_consts(t, limbs, nl, special);
    return check_cuda(acc_inverse_moddown(t, out, acc, B, ext, ne, mc, src, 2LL * nl * N, 0, (long long)nl * N, 0, 1, 0, st),
                      where)
               ? 0
               : 1;
}

namespace {
// ntt_out: leave both components in the NTT domain (msg must then be null).
template <bool NOISE>
int launch_encrypt_combine(const IncNtt* t, dim3 g, uint64_t* out, const uint64_t* sk, const LimbPrimes& lp, int nl,
                           long long N, cudaStream_t st) {
    switch (t->pub.split_degree) {
        case 1: k_encrypt_combine<1, NOISE><<<g, 256, 0, st>>>(out, sk, lp, t->d_info, nl, N); break;
        case 2: k_encrypt_combine<2, NOISE><<<g, 256, 0, st>>>(out, sk, lp, t->d_info, nl, N); break;
        case 4: k_encrypt_combine<4, NOISE><<<g, 256, 0, st>>>(out, sk, lp, t->d_info, nl, N); break;
        case 8: k_encrypt_combine<8, NOISE><<<g, 256, 0, st>>>(out, sk, lp, t->d_info, nl, N); break;
        default: k_encrypt_combine<16, NOISE><<<g, 256, 0, st>>>(out, sk, lp, t->d_info, nl, N); break;
    }
    return (int)cudaGetLastError();
}

int rlwe_encrypt_impl(IncNtt* t, uint64_t* out, const uint64_t* msg, uint64_t B, const uint32_t* limbs, uint32_t L,
                      const uint64_t* sk, double sigma, bool ntt_out, const char* where, cudaStream_t st) {
    if (!t || !limbs || L == 0 || L > (uint32_t)kMaxLimbs || !out || !sk || B == 0 || B > 65535 / L ||
        !(sigma >= 0.0)) {
        set_error(where, "bad pool, limb list, buffers, batch (1 <= batch * nlimbs <= 65535) or sigma");
        return 1;
    }
    for (uint32_t k = 0; k < L; ++k)
        if (limbs[k] >= t->pub.l) {
            set_error(where, "limb index outside the pool");
            return 1;
        }
    const long long N = (long long)t->pub.N;
    const int nl = (int)L;
    LimbPrimes lp;
    memset(&lp, 0, sizeof lp);
    for (int i = 0; i < nl; ++i) lp.p[i] = limbs[i];
    const uint64_t per4 = (uint64_t)((N + 3) / 4), per8 = (uint64_t)((N + 7) / 8);
    // counters: the Gaussian blocks, then the uniform blocks and their redraws (two streams
    // over the same range)
    const uint64_t g0 = prng_advance(B * per4 + B * L * per8 * 8);
    const uint64_t u0 = g0 + B * per4;
    const dim3 gs = grid_xy((long long)per8, (long long)B);   // k_encrypt_sample: 8 coefficients a thread
    const dim3 gn = grid_xy((long long)per4, (long long)B);   // k_encrypt_noise_msg: 4 a thread
    // rows: a component (limb i) at b 2L N + i N, b component at b 2L N + (L + i) N
    RowSet rs;
    memset(&rs, 0, sizeof rs);
    for (int i = 0; i < nl; ++i) {
        rs.in[i] = out + ((long long)(ntt_out ? nl : 0) + i) * N;
        rs.out[i] = out + ((long long)nl + i) * N;
        rs.prime[i] = limbs[i];
    }
    rs.nlimbs = nl;
    rs.split = (int)t->pub.split_degree;
    rs.logP = t->logP;
    rs.batch = (int)B;
    rs.batch_stride = 2LL * nl * N;
    rs.in_batch_stride = rs.batch_stride;
    mark_fp64(rs, t);
    const dim3 g = grid_xy(N / (long long)t->pub.split_degree, (long long)B * nl);
    if (ntt_out) {
        // keys stay in the NTT domain: a drawn there, the noise transformed, b = e + a s
        k_encrypt_sample<true><<<gs, 256, 0, st>>>(out, lp, t->d_info, nl, N, sigma, prng_key(), g0, u0);
        if (!check_cuda(cudaGetLastError(), where)) return 1;
        if (!check_cuda(launch_ntt(rs, t->d_info, false, st), where)) return 1;
        if (!check_cuda(launch_encrypt_combine<true>(t, g, out, sk, lp, nl, N, st), where)) return 1;
        return 0;
    }
    // ciphertexts in the coefficient domain: a drawn as coefficients, then
    // b = INTT(NTT(a) s) + e + m, two transforms of B L rows where the reference's
    // order (transform e and a, multiply, inverse-transform a and b) takes four
    k_encrypt_sample<false><<<gs, 256, 0, st>>>(out, lp, t->d_info, nl, N, sigma, prng_key(), g0, u0);
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    if (!check_cuda(launch_ntt(rs, t->d_info, false, st), where)) return 1;  // b rows <- NTT(a)
    if (!check_cuda(launch_encrypt_combine<false>(t, g, out, sk, lp, nl, N, st), where)) return 1;
    for (int i = 0; i < nl; ++i) rs.in[i] = rs.out[i];
    if (!check_cuda(launch_ntt(rs, t->d_info, true, st), where)) return 1;
    k_encrypt_noise_msg<<<gn, 256, 0, st>>>(out, msg, lp, t->d_info, nl, N, sigma, prng_key(), g0);
    if (!check_cuda(cudaGetLastError(), where)) return 1;
    return 0;
}

}  // namespace

int rlwe_encrypt(IncNtt* t, uint64_t* out, const uint64_t* msg, uint64_t B, const uint32_t* limbs, uint32_t L,
                 const uint64_t* sk, double sigma, cudaStream_t st) {
    return rlwe_encrypt_impl(t, out, msg, B, limbs, L, sk, sigma, false, "vfhe_cuda_rlwe_encrypt_batch", st);
}

int rlwe_gen_ksk(IncNtt* t, uint64_t* out, const uint64_t* src, uint64_t nsrc, const uint32_t* limbs, uint32_t L,
                 const uint64_t* factors, const uint64_t* sk, double sigma, cudaStream_t st) {
    const char* where = "vfhe_cuda_gen_ksk_batch";
    if (!src || !factors || nsrc == 0 || L == 0 || nsrc * L > 65535 / (L ? L : 1)) {
        set_error(where, "need source polynomials, gadget factors and 1 <= nsrc * nlimbs^2 <= 65535");
        return 1;
    }
    if (rlwe_encrypt_impl(t, out, nullptr, nsrc * L, limbs, L, sk, sigma, true, where, st)) return 1;
    LimbPrimes lp;
    memset(&lp, 0, sizeof lp);
    GadgetFactors gf;
    memset(&gf, 0, sizeof gf);
    for (uint32_t i = 0; i < L; ++i) {
        lp.p[i] = limbs[i];
        gf.f[i] = factors[i];
    }
    const long long N = (long long)t->pub.N;
    k_gadget_add<<<grid_xy(N, (long long)(nsrc * L)), 256, 0, st>>>(out, src, gf, lp, t->d_info, (int)L, N);
    return check_cuda(cudaGetLastError(), where) ? 0 : 1;
}

int prng_blocks(uint32_t* out, uint64_t nblocks, const uint32_t* key8, uint64_t counter0, uint64_t nonce,
                cudaStream_t st) {
    PrngKey k;
    memcpy(k.w, key8, sizeof k.w);
    long long blocks = (long long)((nblocks + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    k_prng_blocks<<<(unsigned)blocks, 256, 0, st>>>(out, nblocks, k, counter0, nonce);
    note_launch();
    return check_cuda(cudaGetLastError(), "vfhe_cuda_prng_blocks") ? 0 : 1;
}

}  // namespace vc
