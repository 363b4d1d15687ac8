// Internal definitions of the cuda engine: object layouts behind the public
// handles, the device context, and the kernel launchers shared by the ABI files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "../../include/vfhe_cuda.h"
#include "chacha.cuh"
#include "modarith.cuh"
#include "ntt.cuh"

// Private transform descriptor behind NTT_proc.  The first two fields match the
// reference's struct _NTT_proc (modules/arith/c/include/arith.h:29-33) so C code
// that reads ->n or ->q keeps working.
struct _NTT_proc {
    uint64_t n;
    uint64_t q;
    uint64_t root_of_unity;
    uint64_t inv_root_of_unity;
};

namespace vc {

// ---------------------------------------------------------------- context
struct Context {
    int device = -1;
    int sms = 0;  // streaming multiprocessors of the device
    cudaStream_t stream = nullptr;
    bool ready = false;
    std::recursive_mutex mu;
};
Context& ctx();
// Initialise the device and stream on first use; returns false (and records an
// error) when no CUDA device is usable.  Every ABI entry point calls this first.
bool ensure_ready();
cudaStream_t stream();

// Error recording (first error wins until vfhe_cuda_clear_error).
void set_error(const char* where, const char* what);
bool check_cuda(int code, const char* where);  // true when code == cudaSuccess
// Synchronise the engine stream and record any asynchronous fault.
bool sync(const char* where);

// ---------------------------------------------------------------- memory
// Managed (host+device addressable) blocks from a size-bucketed cache.
void* managed_alloc(size_t bytes);
void managed_free(void* p);
// Device-only scratch from a size-bucketed cache.
void* device_alloc(size_t bytes);
void device_free(void* p);
// Ask the driver to move a managed range to the GPU before kernels touch it.
void prefetch_to_device(const void* p, size_t bytes);

// ---------------------------------------------------------------- objects
struct IncNtt {
    _incNTT pub;  // public prefix; must stay first
    uint64_t P = 0;
    int logP = 0;
    std::vector<PrimeInfo> info;      // host copy; table pointers are device pointers
    std::vector<_NTT_proc*> procs;    // what pub.ntt points at
    std::vector<void*> dev_blocks;    // device table storage to release
    PrimeInfo* d_info = nullptr;      // device copy of `info`
    size_t d_info_cap = 0;
};

struct Poly {
    _RNS_Polynomial pub;  // public prefix; must stay first
    uint64_t* base = nullptr;  // managed block, allocated_l * N residues
};

struct Mlwe {
    _RNS_MLWE pub;  // public prefix
};

struct LweSample {
    _LWE pub;
    uint64_t* block = nullptr;  // managed: l*n (a) followed by l (b)
};

struct LweKey {
    _LWE_Key pub;
    uint64_t* block = nullptr;  // managed: l*n
};

struct IntPoly {
    uint64_t* coeffs;
    uint64_t N;
};

struct MlweKey {
    _RNS_MLWE_Key pub;
};

inline IncNtt* as_ntt(void* p) { return reinterpret_cast<IncNtt*>(p); }
inline Poly* as_poly(void* p) { return reinterpret_cast<Poly*>(p); }
inline RNS_MLWE as_mlwe(void* p) { return reinterpret_cast<RNS_MLWE>(p); }

// Allow the FP64 butterfly kernels for a row set when all its primes are below 2^50.
inline void mark_fp64(RowSet& rs, const IncNtt* t) {
    int ok = 1;
    for (int k = 0; k < rs.nlimbs; ++k)
        if (!t->info[rs.prime[k]].fp64) ok = 0;
    rs.fp64 = ok;
}

IncNtt* ntt_create(const uint64_t* primes, uint64_t split, uint64_t N, uint64_t count);
bool ntt_extend(IncNtt* t, const uint64_t* primes, uint64_t count);
Poly* poly_create(uint64_t N, uint64_t mask, IncNtt* t);
void poly_destroy(Poly* p);

// Host number theory used to build tables (tables.cu).
uint64_t host_pow_mod(uint64_t b, uint64_t e, uint64_t q);
uint64_t host_inv_mod(uint64_t a, uint64_t q);
uint64_t host_mul_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t host_shoup(uint64_t w, uint64_t q);
// Fill PrimeInfo (and upload tables) for prime q at transform size P.
bool build_prime(IncNtt* t, uint64_t q, PrimeInfo* out, _NTT_proc* proc,
                 std::vector<uint64_t>& twist_host);
bool upload_prime_info(IncNtt* t);

// ---------------------------------------------------------------- launchers
enum EwOp : int {
    EW_COPY = 0,
    EW_ZERO,
    EW_ADD,
    EW_SUB,
    EW_NEG,
    EW_MUL,
    EW_MUL_ADDTO,
    EW_MUL_SUBTO,
    EW_SCALE,         // out = a * s
    EW_SCALE_ADDTO,   // out = out + a * s
    EW_ADD_SCALAR,    // out = a + s
    EW_REDUCE,        // out = a mod q (a arbitrary 64-bit)
};

struct EwSet {
    uint64_t* out[kMaxLimbs];
    const uint64_t* a[kMaxLimbs];
    const uint64_t* b[kMaxLimbs];
    uint32_t prime[kMaxLimbs];
    uint64_t s[kMaxLimbs];
    uint64_t s_sh[kMaxLimbs];
    int nlimbs;
    long long n;             // elements per limb
    int batch;
    long long batch_stride;  // elements
};

int launch_ew(EwOp op, const EwSet& set, const PrimeInfo* d_primes, cudaStream_t st);

// Copy a small host array (pointers, Galois elements) into device memory through
// kernel parameters: stream-ordered and asynchronous for the host, unlike a
// cudaMemcpyAsync from pageable memory, which first waits for the stream to drain.
// Values go 256 per launch.
int upload_small(uint64_t* d_dst, const uint64_t* h_src, uint64_t n, cudaStream_t st);

// Incomplete (split-degree) product, rns_polynomial.c:311-435.  mode: 0 set, 1 add, 2 sub.
int launch_inc_product(int mode, const EwSet& set, int split, int logP, const PrimeInfo* d_primes,
                       cudaStream_t st);

// NTT -> product -> INTT of batch x nlimbs rows ([batch][nlimbs][N], 16-byte aligned)
// in one kernel (chain.cu): FP64 primes, N <= 2^13, 2^9 <= P <= 2^13.  Returns
// kChainUnavailable, having enqueued nothing, for other shapes; else a cudaError_t.
constexpr int kChainUnavailable = -2;
int launch_chain(IncNtt* t, uint64_t* out, const uint64_t* a, const uint64_t* b, uint64_t batch,
                 const uint32_t* limbs, uint32_t nlimbs, cudaStream_t st);
// Shared-memory attributes of the chain kernels, set once outside any stream capture.
int prepare_chain_kernels();

// The packing key switch's inner product for one sample over nd digits (ckks.cu):
// acc [2][ne][N] = -sum_d D_d (*) K_d, D [nd][ne][N] and keys [nd][2][ne][N] contiguous,
// NTT domain, (*) the ring's incomplete product; ext: the ne limbs' pool indices;
// keyptr: device scratch for one pointer.
int mac_one_sample(IncNtt* t, uint64_t* acc, const uint64_t* D, const uint64_t* keys, uint64_t* keyptr,
                   const uint32_t* ext, int nd, int ne, cudaStream_t st);

// Galois permutation x -> x^gen (rns_polynomial.c:996-1035).
int launch_permute(const EwSet& set, uint64_t N, int split, uint64_t gen, const PrimeInfo* d_primes,
                   cudaStream_t st);

// Multiplication by X^a (minus1: by X^a - 1), split_degree 1 (rns_polynomial.c:1048-1180).
int launch_mul_xai(const EwSet& set, uint64_t N, uint64_t a, bool minus1, const PrimeInfo* d_primes,
                   cudaStream_t st);

// Rounded (round=true) or floored division by the prime of limb `drop`, applied to
// the limbs listed in `set` (rns_polynomial.c:905-976).  set.a[k] must be the
// dropped limb's row for every k; set.out[k] the limb rows to update.
struct DivideArgs {
    uint64_t* drop_row;
    uint64_t half_drop;      // floor(p/2) (0 for floor division)
    uint64_t p;              // dropped prime
    uint32_t drop_prime;     // its pool index
};
int launch_divide(const EwSet& set, const DivideArgs& d, const PrimeInfo* d_primes, cudaStream_t st);

// Uniform residues / rounded Gaussian integers from the engine's counter PRNG.
int launch_sample_uniform(const EwSet& set, const PrngKey& key, uint64_t counter,
                          const PrimeInfo* d_primes, cudaStream_t st);
int launch_sample_gaussian(const EwSet& set, double sigma, const PrngKey& key, uint64_t counter,
                           const PrimeInfo* d_primes, cudaStream_t st);

// Engine randomness (chacha.cuh): the ChaCha20 key (256 bits from /dev/urandom, or
// expanded from the seed given to vfhe_prng_set_deterministic_seed) and the next free
// block counter; prng_advance reserves `blocks` consecutive blocks and returns the first.
PrngKey prng_key();
uint64_t prng_advance(uint64_t blocks);
void prng_set(uint64_t seed, bool deterministic);

}  // namespace vc
