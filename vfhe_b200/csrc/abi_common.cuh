// Helpers shared by the ABI translation units: building limb sets from masks,
// prefetching managed rows, launching the transform over a polynomial.
#pragma once
#include <string.h>

#include "engine.cuh"

namespace vc {

inline int popcount64(uint64_t m) { return __builtin_popcountll(m); }

// Active limb indices of `mask` that exist in a pool of `l` primes.
inline int mask_indices(uint64_t mask, uint64_t l, uint32_t* idx) {
    int n = 0;
    for (uint64_t i = 0; i < l && i < 64; ++i)
        if (mask & (1ULL << i)) idx[n++] = (uint32_t)i;
    return n;
}

inline IncNtt* pool_of(Poly* p) { return reinterpret_cast<IncNtt*>(p->pub.ntt); }

inline int& call_depth();
inline void prefetch_poly(Poly* p) {
    if (call_depth() > 1) return;  // the outermost call already prefetched its operands
    if (p && p->base) prefetch_to_device(p->base, sizeof(uint64_t) * p->pub.allocated_l * p->pub.ntt->N);
}

inline EwSet empty_set(long long n) {
    EwSet s;
    memset(&s, 0, sizeof s);
    s.n = n;
    s.batch = 1;
    s.batch_stride = 0;
    return s;
}

// Set over the active limbs `mask` of out (and optional a, b operands, same rows).
inline EwSet poly_set(Poly* out, Poly* a, Poly* b, uint64_t mask) {
    IncNtt* t = pool_of(out);
    EwSet s = empty_set((long long)t->pub.N);
    uint32_t idx[64];
    const int n = mask_indices(mask, out->pub.allocated_l, idx);
    for (int k = 0; k < n; ++k) {
        const uint32_t i = idx[k];
        s.out[k] = out->pub.coeffs[i];
        s.a[k] = a ? a->pub.coeffs[i] : nullptr;
        s.b[k] = b ? b->pub.coeffs[i] : nullptr;
        s.prime[k] = i;
    }
    s.nlimbs = n;
    return s;
}

// Forward (inverse=false) or inverse transform of the active limbs of `in` into `out`.
inline int poly_ntt(Poly* out, Poly* in, uint64_t mask, bool inverse) {
    IncNtt* t = pool_of(out);
    RowSet rs;
    memset(&rs, 0, sizeof rs);
    uint32_t idx[64];
    const int n = mask_indices(mask, out->pub.allocated_l, idx);
    for (int k = 0; k < n; ++k) {
        rs.out[k] = out->pub.coeffs[idx[k]];
        rs.in[k] = in->pub.coeffs[idx[k]];
        rs.prime[k] = idx[k];
    }
    rs.nlimbs = n;
    rs.split = (int)t->pub.split_degree;
    rs.logP = t->logP;
    rs.batch = 1;
    rs.batch_stride = 0;
    mark_fp64(rs, t);
    return launch_ntt(rs, t->d_info, inverse, stream());
}

// Canonical residue of a signed 64-bit integer given as its two's complement bits.
inline uint64_t host_reduce_signed(uint64_t v, uint64_t q) {
    if (v & (1ULL << 63)) {
        uint64_t r = ((uint64_t)0 - v) % q;
        return r == 0 ? 0 : q - r;
    }
    return v % q;
}

// Enqueue-only building blocks shared with the mlwe surface (defined in abi_arith.cu).
// Incomplete product out (=, +=, -=) a*b for mode 0, 1, 2; out's mask becomes a & b.
void op_product(Poly* out, Poly* a, Poly* b, int mode, const char* where);
// Zero the rows selected by `rows` (limb bit mask) regardless of the active mask.
void op_zero_rows(Poly* p, uint64_t rows, const char* where);
// out += a * s (per-limb scalar s[limb index]); out's mask becomes a's mask.
void op_scale_addto(Poly* out, Poly* a, uint64_t s, const char* where);

}  // namespace vc

namespace vc {
// Nesting depth of ABI calls on this thread.  Composite entry points (key switch,
// CMUX, ...) call the elementary ones; only the outermost call synchronises.
inline int& call_depth() {
    static thread_local int d = 0;
    return d;
}
struct CallScope {
    CallScope() { ++call_depth(); }
    ~CallScope() { --call_depth(); }
};
}  // namespace vc

#define VC_ENTER(name)                                             \
    if (!vc::ensure_ready()) return;                               \
    std::lock_guard<std::recursive_mutex> vc_lock_(vc::ctx().mu);  \
    vc::CallScope vc_scope_;                                       \
    static const char* const vc_where_ = name
#define VC_ENTER_RET(name, ret)                                    \
    if (!vc::ensure_ready()) return ret;                           \
    std::lock_guard<std::recursive_mutex> vc_lock_(vc::ctx().mu);  \
    vc::CallScope vc_scope_;                                       \
    static const char* const vc_where_ = name
#define VC_CHECK(expr) vc::check_cuda((int)(expr), vc_where_)
#define VC_FINISH() (vc::call_depth() == 1 ? vc::sync(vc_where_) : true)
