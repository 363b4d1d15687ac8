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

// One P-point row of a work list: where it is read, where it is written (may be the
// same row) and the constants of its prime.  32 bytes.
struct RowDesc {
    const uint64_t* in;
    uint64_t* out;
    const PrimeInfo* pi;
    uint64_t reserved;
};

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
    // Work-list mode (FP64 path only): when `table` is set (device memory), row r of
    // the launch is table[r], one P-point row with its own prime, so rows of any
    // polynomials, pools and limb sets with the same P share one launch; the slot
    // arrays, nlimbs, split and batch are then unused.
    const RowDesc* table;
    long long table_rows;
    int table_src_is_dst;  // read table[r].out instead of .in (second pass of a split transform)
};

// Rows one launch of `rows` transforms.
inline long long rowset_rows(const RowSet& rows) {
    return rows.table ? rows.table_rows : (long long)rows.batch * rows.nlimbs * rows.split;
}

// Launch shape of the FP64 transform for one (log2 P, log2 rows) class:
//   tile_bits      low index bits done by one CTA tile (== logP: one pass; else a
//                  radix-2^(logP - tile_bits) column pass first), 8..13;
//   tiles_per_cta  tiles (rows or row segments) one CTA holds at once;
//   ctas_per_sm    0 = one CTA per tile group; k = persistent grid of k x SMs CTAs
//                  walking the tile groups.
// Zero fields mean the built-in choice.  Set by the autotuner through the C ABI.
struct NttSchedule {
    int tile_bits;
    int tiles_per_cta;
    int ctas_per_sm;
};
constexpr int kSchedMaxLogP = 17;
constexpr int kSchedRowBuckets = 32;
bool set_ntt_schedule(int logP, int rows_log2, const NttSchedule& s);
NttSchedule get_ntt_schedule(int logP, long long nrows);
int sm_count();

// Launch the forward (inverse=false) or inverse transform of every row in `rows`.
// Work is enqueued on `stream`; returns a cudaError_t code (0 on success).
int launch_ntt(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream);

// Only the tile pass of an inverse FP64 transform (rows aligned, all primes below
// 2^50) whose tuned schedule is a tile pass + a column pass of K1 <= max_k1 bits:
// the rows are left as centred doubles, and *K1_out / *KT_out receive the column and
// tile bits the caller's fused column pass must cover.  Returns kTilePassUnavailable,
// having enqueued nothing, for any other schedule; else a cudaError_t code.
constexpr int kTilePassUnavailable = -3;
bool ntt_f64_eligible(const RowSet& rows);  // launch_ntt would take the FP64 kernels
int launch_ntt_f64_inverse_tiles(const RowSet& rows, const PrimeInfo* d_primes, int max_k1, int* K1_out, int* KT_out,
                                 cudaStream_t stream);

// Count of kernels this engine has launched (vfhe_cuda_launch_count).  Kernels
// recorded into a CUDA graph are counted at capture; the capturing code takes that
// count back (forget_launches) and notes it again at every replay.
void note_launch(int n = 1);
uint64_t launch_counter();
void forget_launches(uint64_t n);

// Raise the dynamic shared-memory limit of every transform kernel once, outside any
// stream capture, so that launches recorded into graphs make no attribute calls.
int prepare_ntt_kernels();

// Two-pass transform (radix-2^K1 column pass + 2^K-point tiles) as one dataflow launch
// (ntt_flow.cu).  `first` / `second` are the two passes' row sets as launch_ntt_f64
// builds them.  Returns kFlowUnavailable, having enqueued nothing, where the launch
// cannot be made (stream capture, no counter buffer under FlowNoAlloc, an unsupported
// shape); the caller then runs the two kernels.
constexpr int kFlowUnavailable = -2;
bool flow_supported(int K, int K1);
// `per`: work items (one CTA's worth of columns or tiles) per ticket: 1 or 2 (0 = two).
int flow_dispatch(int K, int K1, const RowSet& first, const RowSet& second, const PrimeInfo* d_primes, bool inverse,
                  int per, cudaStream_t stream);
// While one lives on this thread, transform launches allocate no device memory.
struct FlowNoAlloc {
    FlowNoAlloc();
    ~FlowNoAlloc();
    FlowNoAlloc(const FlowNoAlloc&) = delete;
    FlowNoAlloc& operator=(const FlowNoAlloc&) = delete;
};
// The flag a dataflow launch raises when a wait for its first pass gave up (0 = never).
int read_flow_fault(int* out);
int clear_flow_fault();

// Copy the device flag that persistent transform kernels raise when a bounded wait
// for a tile copy gave up (0 = never).
int read_tile_fault(int* out);
int clear_tile_fault();

// Kernel attributes of the batched CKKS kernels (the staged key-switch MAC's shared
// memory), set once; prepare_ntt_kernels calls it too.
int prepare_ckks_kernels();

// Copy the device flag that the staged key-switch MAC raises when a bounded wait for
// a bulk copy gave up (0 = never).
int read_mac_fault(int* out);
int clear_mac_fault();

// The flag the persistent work-list kernel raises when a grid-barrier wait gave up.
int read_wl_fault(int* out);
int clear_wl_fault();

// Launch a one-thread kernel whose bounded mbarrier wait can never be satisfied (a
// transaction count no copy delivers) with a limit of `tries` attempts; on return
// *gave_up is 1 when the wait gave up and raised the staged-MAC fault flag.
int bounded_wait_selfcheck(int tries, int* gave_up);

}  // namespace vc
