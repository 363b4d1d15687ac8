// arith.cdef surface of the cuda engine (modules/arith/python/cdef/arith.cdef).
// Each entry point validates its handles, enqueues kernels on the engine stream
// over the active limbs (rns_mask) and synchronises before returning, because the
// caller reads coefficient rows from the host as soon as the call returns.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "abi_common.cuh"

using namespace vc;

namespace {

// Scatter natural-order coefficients into the split-interleaved row layout
// (coefficient j -> row position (j mod s) * P + j / s, rns_polynomial.c:199-238),
// optionally reducing signed 64-bit inputs.
template <bool REDUCE>
__global__ void k_scatter(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                          int split, int log_split, long long P) {
    const int k = blockIdx.y;
    const PrimeInfo pi = primes[set.prime[k]];
    const uint64_t* src = set.a[k];
    uint64_t* dst = set.out[k];
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < set.n;
         j += (long long)gridDim.x * blockDim.x) {
        const uint64_t v = src[j];
        dst[(j & (split - 1)) * P + (j >> log_split)] = REDUCE ? reduce_signed((int64_t)v, pi) : v;
    }
}

// Slot operations on NTT-domain rows (rns_polynomial.c:1212-1280).
// mode 0 broadcast slot `a0`; mode 1 rotate by `a0`; mode 2 copy slot a1 -> a0.
__global__ void k_slots(const __grid_constant__ EwSet set, int mode, int split, long long P, long long a0,
                        long long a1) {
    const int k = blockIdx.y;
    const uint64_t* in = set.a[k];
    uint64_t* out = set.out[k];
    const long long total = mode == 2 ? split : (long long)split * P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        if (mode == 2) {
            out[e * P + a0] = in[e * P + a1];
            continue;
        }
        const long long blk = e / P, x = e - blk * P;
        long long src;
        if (mode == 0) src = a0;
        else src = (x + a0) % P;
        out[e] = in[blk * P + src];
    }
}

// Slot-wise inverse by Fermat (a^(q-2)); any zero slot sets *flag.
__global__ void k_inverse(const __grid_constant__ EwSet set, const PrimeInfo* __restrict__ primes,
                          int* flag) {
    const int k = blockIdx.y;
    const PrimeInfo pi = primes[set.prime[k]];
    const uint64_t* in = set.a[k];
    uint64_t* out = set.out[k];
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < set.n;
         x += (long long)gridDim.x * blockDim.x) {
        const uint64_t a = in[x];
        if (a == 0) {
            atomicOr(flag, 1);
            out[x] = 0;
            continue;
        }
        uint64_t r = 1, b = a, e = pi.q - 2;
        while (e) {
            if (e & 1) r = mul_mod(r, b, pi);
            b = mul_mod(b, b, pi);
            e >>= 1;
        }
        out[x] = r;
    }
}

// polynomial_eq (rns_polynomial.c:91-124): rows active on both sides must match;
// rows active on one side only must be zero.  set.a/b hold the rows or null.
__global__ void k_eq(const __grid_constant__ EwSet set, int* flag) {
    const int k = blockIdx.y;
    const uint64_t* a = set.a[k];
    const uint64_t* b = set.b[k];
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < set.n;
         x += (long long)gridDim.x * blockDim.x) {
        const uint64_t va = a ? a[x] : 0, vb = b ? b[x] : 0;
        if (va != vb) atomicOr(flag, 1);
    }
}

dim3 grid_for(long long n, int limbs) {
    long long blocks = (n + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    return dim3((unsigned)blocks, (unsigned)limbs, 1);
}

bool valid_poly(void* p, const char* where) {
    if (!p) {
        set_error(where, "null polynomial handle");
        return false;
    }
    return true;
}

int* g_flag = nullptr;  // managed 1-int flag for reductions

int* flag() {
    if (!g_flag) g_flag = (int*)managed_alloc(sizeof(int));
    return g_flag;
}

void ew_mask(EwOp op, Poly* out, Poly* a, Poly* b, uint64_t mask, const char* where) {
    prefetch_poly(a);
    prefetch_poly(b);
    prefetch_poly(out);
    EwSet s = poly_set(out, a, b, mask);
    check_cuda(launch_ew(op, s, pool_of(out)->d_info, stream()), where);
}

}  // namespace

namespace vc {

// Signed 64-bit integers (device array of N) into every active limb of `out`, in the
// ring's coefficient layout, then the forward transform (int_array_to_RNS,
// rns_polynomial.c:199-238).  Enqueued on `st` (the engine stream).
int int_array_to_RNS_device(void* out, const int64_t* d_in, cudaStream_t st) {
    Poly* o = as_poly(out);
    IncNtt* t = pool_of(o);
    const uint64_t N = t->pub.N;
    prefetch_poly(o);
    EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask);
    for (int k = 0; k < s.nlimbs; ++k) s.a[k] = (const uint64_t*)d_in;
    int ls = 0;
    while ((1ULL << ls) < t->pub.split_degree) ++ls;
    if (s.nlimbs) {
        k_scatter<true><<<grid_for((long long)N, s.nlimbs), 256, 0, st>>>(s, t->d_info, (int)t->pub.split_degree, ls,
                                                                        (long long)t->P);
        const int e = (int)cudaGetLastError();
        if (e) return e;
    }
    return poly_ntt(o, o, o->pub.rns_mask, false);
}

}  // namespace vc

extern "C" {

void* safe_aligned_malloc(uint64_t size) {
    void* p = nullptr;
    if (posix_memalign(&p, 64, size ? size : 64) != 0) return nullptr;
    return p;
}

void* new_incomplete_ntt_list(uint64_t* primes, uint64_t split_degree, uint64_t N, uint64_t count) {
    if (!vc::ensure_ready()) return nullptr;
    std::lock_guard<std::recursive_mutex> lk(vc::ctx().mu);
    return ntt_create(primes, split_degree, N, count);
}

void incNTT_extend_with_primes(void* ntt, uint64_t* new_primes, uint64_t count) {
    VC_ENTER("incNTT_extend_with_primes");
    if (!ntt || count == 0) {
        if (!ntt) set_error(vc_where_, "null pool");
        return;
    }
    ntt_extend(as_ntt(ntt), new_primes, count);
}

uint64_t** incNTT_get_rou_matrix(void* ntt) { return ntt ? as_ntt(ntt)->pub.w : nullptr; }

void* polynomial_new_RNS_polynomial(uint64_t N, uint64_t rns_mask, void* ntt) {
    VC_ENTER_RET("polynomial_new_RNS_polynomial", nullptr);
    (void)vc_where_;
    return poly_create(N, rns_mask, as_ntt(ntt));
}

void free_RNS_polynomial(void* p) {
    if (!p) return;
    std::lock_guard<std::recursive_mutex> lk(vc::ctx().mu);
    // Every outermost entry point synchronises before returning and all engine work
    // is ordered on one stream, so a recycled block is never touched by a stale kernel.
    poly_destroy(as_poly(p));
}

void polynomial_copy_RNS_polynomial(void* out, void* in) {
    VC_ENTER("polynomial_copy_RNS_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    o->pub.rns_mask = i->pub.rns_mask;
    if (o != i) ew_mask(EW_COPY, o, i, nullptr, o->pub.rns_mask, vc_where_);
    VC_FINISH();
}

void int_array_to_RNS(void* out, uint64_t* in) {
    VC_ENTER("int_array_to_RNS");
    if (!valid_poly(out, vc_where_) || !in) return;
    const uint64_t N = pool_of(as_poly(out))->pub.N;
    uint64_t* d_in = (uint64_t*)device_alloc(N * 8);
    if (!d_in) return;
    VC_CHECK(cudaMemcpyAsync(d_in, in, N * 8, cudaMemcpyHostToDevice, stream()));
    VC_CHECK(vc::int_array_to_RNS_device(out, (const int64_t*)d_in, stream()));
    VC_FINISH();
    device_free(d_in);
}

void array_to_RNS(void* out, uint64_t** in) {
    VC_ENTER("array_to_RNS");
    if (!valid_poly(out, vc_where_) || !in) return;
    Poly* o = as_poly(out);
    IncNtt* t = pool_of(o);
    const uint64_t N = t->pub.N;
    EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask);
    uint64_t* d_in = (uint64_t*)device_alloc(N * 8 * (s.nlimbs ? s.nlimbs : 1));
    if (!d_in) return;
    for (int k = 0; k < s.nlimbs; ++k) {
        const uint64_t* row = in[s.prime[k]];
        if (!row) {
            set_error(vc_where_, "missing input row for an active limb");
            device_free(d_in);
            return;
        }
        VC_CHECK(cudaMemcpyAsync(d_in + k * N, row, N * 8, cudaMemcpyHostToDevice, stream()));
        s.a[k] = d_in + k * N;
    }
    prefetch_poly(o);
    int ls = 0;
    while ((1ULL << ls) < t->pub.split_degree) ++ls;
    if (s.nlimbs) {
        k_scatter<false><<<grid_for((long long)N, s.nlimbs), 256, 0, stream()>>>(
            s, t->d_info, (int)t->pub.split_degree, ls, (long long)t->P);
        VC_CHECK(cudaGetLastError());
    }
    VC_CHECK(poly_ntt(o, o, o->pub.rns_mask, false));
    VC_FINISH();
    device_free(d_in);
}

void polynomial_gen_random_RNSc_polynomial(void* out) {
    VC_ENTER("polynomial_gen_random_RNSc_polynomial");
    if (!valid_poly(out, vc_where_)) return;
    Poly* o = as_poly(out);
    prefetch_poly(o);
    EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask);
    const uint64_t ctr = prng_advance((uint64_t)((s.n + 3) / 4) * (uint64_t)(s.nlimbs ? s.nlimbs : 1));
    VC_CHECK(launch_sample_uniform(s, prng_key(), ctr, pool_of(o)->d_info, stream()));
    VC_FINISH();
}

void polynomial_gen_gaussian_RNSc_polynomial(void* out, double sigma) {
    VC_ENTER("polynomial_gen_gaussian_RNSc_polynomial");
    if (!valid_poly(out, vc_where_)) return;
    Poly* o = as_poly(out);
    prefetch_poly(o);
    EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask);
    const uint64_t ctr = prng_advance((uint64_t)((s.n + 3) / 4));
    VC_CHECK(launch_sample_gaussian(s, sigma, prng_key(), ctr, pool_of(o)->d_info, stream()));
    VC_FINISH();
}

static void product(void* out, void* in1, void* in2, int mode, bool set_mask_only_common,
                    const char* where) {
    Poly* o = as_poly(out);
    Poly* a = as_poly(in1);
    Poly* b = as_poly(in2);
    IncNtt* t = pool_of(o);
    const uint64_t mask = a->pub.rns_mask & b->pub.rns_mask;
    (void)set_mask_only_common;
    o->pub.rns_mask = mask;
    prefetch_poly(a);
    prefetch_poly(b);
    prefetch_poly(o);
    EwSet s = poly_set(o, a, b, mask);
    check_cuda(launch_inc_product(mode, s, (int)t->pub.split_degree, t->logP, t->d_info, stream()), where);
}

void polynomial_mul_RNS_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("polynomial_mul_RNS_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_) || !valid_poly(in2, vc_where_)) return;
    if (out == in1 || out == in2) {
        set_error(vc_where_, "out must differ from the inputs (rns_polynomial.c:313-314)");
        return;
    }
    product(out, in1, in2, 0, true, vc_where_);
    VC_FINISH();
}

void polynomial_multo_RNS_polynomial(void* out, void* in) {
    VC_ENTER("polynomial_multo_RNS_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    const uint64_t mask = o->pub.rns_mask & i->pub.rns_mask;
    o->pub.rns_mask = mask;
    IncNtt* t = pool_of(o);
    prefetch_poly(o);
    prefetch_poly(i);
    EwSet s = poly_set(o, i, o, mask);
    VC_CHECK(launch_inc_product(0, s, (int)t->pub.split_degree, t->logP, t->d_info, stream()));
    VC_FINISH();
}

void polynomial_sub_RNS_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("polynomial_sub_RNS_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_) || !valid_poly(in2, vc_where_)) return;
    const uint64_t mask = as_poly(in1)->pub.rns_mask & as_poly(in2)->pub.rns_mask;
    as_poly(out)->pub.rns_mask = mask;
    ew_mask(EW_SUB, as_poly(out), as_poly(in1), as_poly(in2), mask, vc_where_);
    VC_FINISH();
}

void polynomial_sub_RNSc_polynomial(void* out, void* in1, void* in2) {
    polynomial_sub_RNS_polynomial(out, in1, in2);
}

void polynomial_add_RNSc_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("polynomial_add_RNSc_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_) || !valid_poly(in2, vc_where_)) return;
    const uint64_t mask = as_poly(in1)->pub.rns_mask & as_poly(in2)->pub.rns_mask;
    as_poly(out)->pub.rns_mask = mask;
    ew_mask(EW_ADD, as_poly(out), as_poly(in1), as_poly(in2), mask, vc_where_);
    VC_FINISH();
}

void polynomial_add_RNS_polynomial(void* out, void* in1, void* in2) {
    polynomial_add_RNSc_polynomial(out, in1, in2);
}

static void scale_by(Poly* o, Poly* a, const uint64_t* per_limb, uint64_t uniform, bool addto,
                     const char* where) {
    IncNtt* t = pool_of(o);
    const uint64_t mask = a->pub.rns_mask;
    o->pub.rns_mask = mask;
    prefetch_poly(a);
    prefetch_poly(o);
    EwSet s = poly_set(o, a, nullptr, mask);
    for (int k = 0; k < s.nlimbs; ++k) {
        const uint64_t q = t->info[s.prime[k]].q;
        const uint64_t v = (per_limb ? per_limb[s.prime[k]] : uniform) % q;
        s.s[k] = v;
        s.s_sh[k] = host_shoup(v, q);
    }
    check_cuda(launch_ew(addto ? EW_SCALE_ADDTO : EW_SCALE, s, t->d_info, stream()), where);
}

void polynomial_scale_RNSc_polynomial(void* out, void* in1, uint64_t scale) {
    VC_ENTER("polynomial_scale_RNSc_polynomial");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_)) return;
    scale_by(as_poly(out), as_poly(in1), nullptr, scale, false, vc_where_);
    VC_FINISH();
}

void polynomial_scale_RNS_polynomial_RNS(void* out, void* in1, uint64_t* scale) {
    VC_ENTER("polynomial_scale_RNS_polynomial_RNS");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_) || !scale) return;
    scale_by(as_poly(out), as_poly(in1), scale, 0, false, vc_where_);
    VC_FINISH();
}

void polynomial_RNSc_negate(void* out, void* in) {
    VC_ENTER("polynomial_RNSc_negate");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    const uint64_t mask = as_poly(in)->pub.rns_mask;
    as_poly(out)->pub.rns_mask = mask;
    ew_mask(EW_NEG, as_poly(out), as_poly(in), nullptr, mask, vc_where_);
    VC_FINISH();
}

// Adds the integer in2 (two's complement) to the first `count` residues of every
// active row: count 1 in the coefficient domain (rns_polynomial.c:460-474), the whole
// first split block in the NTT domain (rns_polynomial.c:476-500).
static void add_integer(Poly* o, Poly* a, uint64_t in2, long long count, const char* where) {
    IncNtt* t = pool_of(o);
    const uint64_t mask = a->pub.rns_mask;
    o->pub.rns_mask = mask;
    if (o != a) ew_mask(EW_COPY, o, a, nullptr, mask, where);
    prefetch_poly(o);
    EwSet s = poly_set(o, o, nullptr, mask);
    s.n = count;
    for (int k = 0; k < s.nlimbs; ++k) s.s[k] = host_reduce_signed(in2, t->info[s.prime[k]].q);
    check_cuda(launch_ew(EW_ADD_SCALAR, s, t->d_info, stream()), where);
}

void polynomial_RNSc_add_integer(void* out, void* in1, uint64_t in2) {
    VC_ENTER("polynomial_RNSc_add_integer");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_)) return;
    add_integer(as_poly(out), as_poly(in1), in2, 1, vc_where_);
    VC_FINISH();
}

void polynomial_RNS_add_integer(void* out, void* in1, uint64_t in2) {
    VC_ENTER("polynomial_RNS_add_integer");
    if (!valid_poly(out, vc_where_) || !valid_poly(in1, vc_where_)) return;
    add_integer(as_poly(out), as_poly(in1), in2, (long long)pool_of(as_poly(out))->P, vc_where_);
    VC_FINISH();
}

void polynomial_RNSc_permute(void* out, void* in, uint64_t gen) {
    VC_ENTER("polynomial_RNSc_permute");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    if (out == in) {
        set_error(vc_where_, "out must differ from in (rns_polynomial.c:998)");
        return;
    }
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    IncNtt* t = pool_of(o);
    const uint64_t N = t->pub.N;
    if (gen == 0 || gen >= 2 * N) {
        set_error(vc_where_, "gen must lie in (0, 2N) (rns_polynomial.c:1007-1008)");
        return;
    }
    o->pub.rns_mask = i->pub.rns_mask;
    const uint64_t all = (o->pub.allocated_l >= 64) ? ~0ULL : ((1ULL << o->pub.allocated_l) - 1);
    ew_mask(EW_ZERO, o, nullptr, nullptr, all & ~i->pub.rns_mask, vc_where_);
    prefetch_poly(i);
    EwSet s = poly_set(o, i, nullptr, i->pub.rns_mask);
    VC_CHECK(launch_permute(s, N, (int)t->pub.split_degree, gen, t->d_info, stream()));
    VC_FINISH();
}

void polynomial_RNSc_to_RNS(void* out, void* in) {
    VC_ENTER("polynomial_RNSc_to_RNS");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    o->pub.rns_mask = i->pub.rns_mask;
    prefetch_poly(i);
    prefetch_poly(o);
    VC_CHECK(poly_ntt(o, i, o->pub.rns_mask, false));
    VC_FINISH();
}

void polynomial_RNS_to_RNSc(void* out, void* in) {
    VC_ENTER("polynomial_RNS_to_RNSc");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    o->pub.rns_mask = i->pub.rns_mask;
    prefetch_poly(i);
    prefetch_poly(o);
    VC_CHECK(poly_ntt(o, i, o->pub.rns_mask, true));
    VC_FINISH();
}

void polynomial_RNSc_mod_reduce(void* out, void* in) {
    VC_ENTER("polynomial_RNSc_mod_reduce");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    if (out != in) ew_mask(EW_COPY, o, as_poly(in), nullptr, o->pub.rns_mask, vc_where_);
    VC_FINISH();
}

void polynomial_RNSc_mod_reduce_lifted(void* out, void* in, uint64_t idx) {
    VC_ENTER("polynomial_RNSc_mod_reduce_lifted");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    if (idx >= i->pub.allocated_l) {
        set_error(vc_where_, "limb index outside the input's pool");
        return;
    }
    prefetch_poly(i);
    prefetch_poly(o);
    EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask);
    for (int k = 0; k < s.nlimbs; ++k) s.a[k] = i->pub.coeffs[idx];
    VC_CHECK(launch_ew(EW_REDUCE, s, pool_of(o)->d_info, stream()));
    VC_FINISH();
}

// Sequential division by every prime of `divide_mask` in increasing limb order
// (rns_polynomial.c:905-976): each step updates every other active limb, including
// limbs dropped later, then clears the dropped row and its mask bit.
static void divide(Poly* o, uint64_t divide_mask, bool round, const char* where) {
    IncNtt* t = pool_of(o);
    uint64_t mask = divide_mask & o->pub.rns_mask;
    if (!mask) return;
    prefetch_poly(o);
    for (uint64_t idx = 0; idx < o->pub.allocated_l; ++idx) {
        if (!(mask & (1ULL << idx))) continue;
        const uint64_t p = t->info[idx].q;
        DivideArgs d;
        d.drop_row = o->pub.coeffs[idx];
        d.half_drop = round ? p / 2 : 0;
        d.p = p;
        d.drop_prime = (uint32_t)idx;
        EwSet s = poly_set(o, nullptr, nullptr, o->pub.rns_mask & ~(1ULL << idx));
        for (int k = 0; k < s.nlimbs; ++k) {
            const uint64_t q = t->info[s.prime[k]].q;
            s.s[k] = host_inv_mod(p % q, q);
            s.s_sh[k] = host_shoup(s.s[k], q);
        }
        if (!check_cuda(launch_divide(s, d, t->d_info, stream()), where)) return;
        o->pub.rns_mask &= ~(1ULL << idx);
    }
}

void polynomial_round_division_RNSc_wo_free(void* out, uint64_t divide_mask) {
    VC_ENTER("polynomial_round_division_RNSc_wo_free");
    if (!valid_poly(out, vc_where_)) return;
    divide(as_poly(out), divide_mask, true, vc_where_);
    VC_FINISH();
}

void polynomial_floor_division_RNSc_wo_free(void* out, uint64_t divide_mask) {
    VC_ENTER("polynomial_floor_division_RNSc_wo_free");
    if (!valid_poly(out, vc_where_)) return;
    divide(as_poly(out), divide_mask, false, vc_where_);
    VC_FINISH();
}

void polynomial_RNSc_scaled_lift(void* out, void* in, uint64_t* delta) {
    VC_ENTER("polynomial_RNSc_scaled_lift");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    IncNtt* t = pool_of(o);
    uint64_t local[64];
    const uint64_t l = t->pub.l;
    if (!delta) {
        // rns_compute_scaling_factors (rns_polynomial.c:1463-1496): product of the primes
        // present in out but not in in, per limb of in
        const uint64_t diff = o->pub.rns_mask & ~i->pub.rns_mask;
        for (uint64_t k = 0; k < l && k < 64; ++k) {
            local[k] = 0;
            if ((o->pub.rns_mask & (1ULL << k)) && (i->pub.rns_mask & (1ULL << k))) {
                const uint64_t q = t->info[k].q;
                uint64_t d = 1 % q;
                for (uint64_t j = 0; j < l && j < 64; ++j)
                    if (diff & (1ULL << j)) d = host_mul_mod(d, t->info[j].q % q, q);
                local[k] = d;
            }
        }
        delta = local;
    }
    const uint64_t both = o->pub.rns_mask & i->pub.rns_mask;
    ew_mask(EW_ZERO, o, nullptr, nullptr, o->pub.rns_mask & ~i->pub.rns_mask, vc_where_);
    prefetch_poly(i);
    EwSet s = poly_set(o, i, nullptr, both);
    for (int k = 0; k < s.nlimbs; ++k) {
        const uint64_t q = t->info[s.prime[k]].q;
        s.s[k] = delta[s.prime[k]] % q;
        s.s_sh[k] = host_shoup(s.s[k], q);
    }
    VC_CHECK(launch_ew(EW_SCALE, s, t->d_info, stream()));
    VC_FINISH();
}

int polynomial_RNS_inverse(void* out, void* in) {
    VC_ENTER_RET("polynomial_RNS_inverse", -1);
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return -1;
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    IncNtt* t = pool_of(o);
    if (t->pub.split_degree != 1) {
        set_error(vc_where_, "slot inversion over field extensions (split_degree > 1) is not part of this engine");
        return -1;
    }
    o->pub.rns_mask = i->pub.rns_mask;
    int* f = flag();
    if (!f) return -1;
    *f = 0;
    prefetch_poly(i);
    prefetch_poly(o);
    EwSet s = poly_set(o, i, nullptr, i->pub.rns_mask);
    if (s.nlimbs) {
        k_inverse<<<grid_for(s.n, s.nlimbs), 256, 0, stream()>>>(s, t->d_info, f);
        VC_CHECK(cudaGetLastError());
    }
    if (!vc::sync(vc_where_)) return -1;
    return *f ? -2 : 0;
}

bool polynomial_eq(void* a, void* b) {
    VC_ENTER_RET("polynomial_eq", false);
    if (!valid_poly(a, vc_where_) || !valid_poly(b, vc_where_)) return false;
    Poly* pa = as_poly(a);
    Poly* pb = as_poly(b);
    const uint64_t la = pa->pub.ntt->l, lb = pb->pub.ntt->l;
    const uint64_t max_l = la > lb ? la : lb;
    int* f = flag();
    if (!f) return false;
    *f = 0;
    prefetch_poly(pa);
    prefetch_poly(pb);
    EwSet s = empty_set((long long)pa->pub.ntt->N);
    int n = 0;
    for (uint64_t i = 0; i < max_l && i < 64; ++i) {
        const bool aa = i < la && i < pa->pub.allocated_l && (pa->pub.rns_mask & (1ULL << i));
        const bool bb = i < lb && i < pb->pub.allocated_l && (pb->pub.rns_mask & (1ULL << i));
        if (!aa && !bb) continue;
        s.a[n] = aa ? pa->pub.coeffs[i] : nullptr;
        s.b[n] = bb ? pb->pub.coeffs[i] : nullptr;
        ++n;
    }
    s.nlimbs = n;
    if (n) {
        k_eq<<<grid_for(s.n, n), 256, 0, stream()>>>(s, f);
        VC_CHECK(cudaGetLastError());
    }
    if (!vc::sync(vc_where_)) return false;
    return *f == 0;
}

static void slots(void* out, void* in, int mode, long long a0, long long a1, const char* where) {
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    IncNtt* t = pool_of(o);
    if (a0 < 0 || a1 < 0 || (mode != 1 && a0 >= (long long)t->P) || a1 >= (long long)t->P) {
        set_error(where, "slot index outside [0, N/split_degree)");
        return;
    }
    if (mode == 1) a0 %= (long long)t->P;
    o->pub.rns_mask = i->pub.rns_mask;
    prefetch_poly(i);
    prefetch_poly(o);
    EwSet s = poly_set(o, i, nullptr, i->pub.rns_mask);
    if (!s.nlimbs) return;
    const long long total = mode == 2 ? (long long)t->pub.split_degree : (long long)t->pub.N;
    k_slots<<<grid_for(total, s.nlimbs), 256, 0, stream()>>>(s, mode, (int)t->pub.split_degree,
                                                             (long long)t->P, a0, a1);
    check_cuda(cudaGetLastError(), where);
}

void polynomial_RNS_broadcast_slot(void* out, void* in, uint64_t slot_idx) {
    VC_ENTER("polynomial_RNS_broadcast_slot");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    if (out == in) {
        // broadcasting in place reads the slot after it was overwritten in other blocks
        // only if a block's own slot changes first; stage through a copy to be safe
        Poly* tmp = poly_create(0, as_poly(in)->pub.rns_mask, pool_of(as_poly(in)));
        polynomial_copy_RNS_polynomial(tmp, in);
        slots(out, tmp, 0, (long long)slot_idx, 0, vc_where_);
        VC_FINISH();
        poly_destroy(tmp);
        return;
    }
    slots(out, in, 0, (long long)slot_idx, 0, vc_where_);
    VC_FINISH();
}

void polynomial_RNS_rotate_slot(void* out, void* in, uint64_t rot) {
    VC_ENTER("polynomial_RNS_rotate_slot");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    if (out == in) {
        set_error(vc_where_, "out must differ from in (rns_polynomial.c:1246)");
        return;
    }
    slots(out, in, 1, (long long)rot, 0, vc_where_);
    VC_FINISH();
}

void polynomial_RNS_copy_slot(void* out, uint64_t dst, void* in, uint64_t src) {
    VC_ENTER("polynomial_RNS_copy_slot");
    if (!valid_poly(out, vc_where_) || !valid_poly(in, vc_where_)) return;
    slots(out, in, 2, (long long)dst, (long long)src, vc_where_);
    VC_FINISH();
}

void polynomial_RNS_get_hash(uint64_t* out, void* p) {
    (void)p;
    if (out) memset(out, 0, 32);
    set_error("polynomial_RNS_get_hash", "BLAKE3 hashing is not part of the cuda engine");
}

uint64_t* polynomial_RNS_get_hash_p(void* p) {
    uint64_t* out = (uint64_t*)malloc(32);
    polynomial_RNS_get_hash(out, p);
    return out;
}

}  // extern "C"

namespace vc {

void op_product(Poly* out, Poly* a, Poly* b, int mode, const char* where) {
    product(out, a, b, mode, true, where);
}

void op_zero_rows(Poly* p, uint64_t rows, const char* where) {
    const uint64_t all = (p->pub.allocated_l >= 64) ? ~0ULL : ((1ULL << p->pub.allocated_l) - 1);
    ew_mask(EW_ZERO, p, nullptr, nullptr, rows & all, where);
}

void op_scale_addto(Poly* out, Poly* a, uint64_t s, const char* where) {
    scale_by(out, a, nullptr, s, true, where);
}

}  // namespace vc
