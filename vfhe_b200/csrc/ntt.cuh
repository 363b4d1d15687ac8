// Negacyclic (incomplete) NTT kernels for sm_100a.
//
// Transform conventions follow the reference exactly (bit-exactness depends on it):
//   forward  = Cooley-Tukey, natural order in, bit-reversed order out
//              (ntt_CT_NR_portable, modules/arith/c/src/ntt_portable.c:76-100):
//              stage s (m = 2^s, t = P/2m) pairs (j, j+t) of group i = j/2t with
//              twiddle fwd[m+i], fwd[brv(i)] = psi^i;
//   inverse  = Gentleman-Sande, bit-reversed in, natural out, scaled by P^-1
//              (ntt_GS_RN_portable, ntt_portable.c:102-135): stage with h groups,
//              t = P/2h, twiddle inv[h+i], inv[brv(i)] = psi^-i.
// psi is the reference's deterministic root (ntt_new_proc, ntt_portable.c:137-179).
//
// Design: a transform of P = 2^logP residues is one or two "passes".  A pass owns a
// contiguous range [bit_lo, bit_lo+k) of index bits: one CTA loads a tile of 2^k
// sub-problem points x 2^logC adjacent columns into shared memory (coalesced along
// the columns), runs the k butterfly stages of those bits with Shoup twiddle
// products and lazy [0,4q) residues, and writes the tile back.  P <= 2^14 fits one
// CTA (one pass, one HBM round trip); larger P uses two passes.
#pragma once
#include "modarith.cuh"

namespace vc {

constexpr int kMaxLimbs = 64;

// A set of rows (one row = one P-point transform) described compactly.
// Row r of the launch maps to (poly b, limb slot k, block blk):
//   r = (b * nlimbs + k) * split + blk
//   in  = in_base[k]  + b * in_batch_stride + blk * P
//   out = out_base[k] + b * batch_stride    + blk * P
// With reduce_input set, a forward transform first reduces each loaded residue
// modulo its row's prime (the digit broadcast of a key switch: the input row holds
// residues of another prime, rns_polynomial.c:824-843).
struct RowSet {
    uint64_t* out[kMaxLimbs];
    const uint64_t* in[kMaxLimbs];
    uint32_t prime[kMaxLimbs];
    int nlimbs;
    int split;
    int logP;
    int batch;
    long long batch_stride;     // output stride between polynomials, in elements
    long long in_batch_stride;  // input stride between polynomials, in elements
    int reduce_input;
    // set by launch_ntt when every prime of the set is below 2^50 (FP64 butterflies)
    int fp64;
};

// Launch the forward (inverse=false) or inverse transform of every row in `rows`.
// Work is enqueued on `stream`; returns a cudaError_t code (0 on success).
int launch_ntt(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream);

// Count of kernels this engine has launched (vfhe_cuda_launch_count).
void note_launch(int n = 1);

}  // namespace vc
