// NTT pass kernel and launcher; conventions are documented in ntt.cuh.
#include <cuda_runtime.h>

#include "ntt.cuh"

namespace vc {

namespace {

// One pass over the index bits [bit_lo, bit_lo + k) of every row.
// Residues entering a forward pass lie in [0, 4q); entering an inverse pass in [0, 2q).
template <bool INV>
__global__ void __launch_bounds__(1024) k_ntt_pass(const __grid_constant__ RowSet rows,
                                                   const PrimeInfo* __restrict__ primes, int bit_lo,
                                                   int k, int logC, int last) {
    extern __shared__ uint64_t tile[];
    const int logP = rows.logP;
    const int P = 1 << logP;
    const int C = 1 << logC;
    const int T = 1 << (k + logC);
    const int ncb = (1 << bit_lo) >> logC;   // column blocks per hi value
    const int nhi = P >> (bit_lo + k);       // hi values per row
    const long long tiles_per_row = (long long)nhi * ncb;

    const long long tid_tile = blockIdx.x;
    const long long row = tid_tile / tiles_per_row;
    const int tr = (int)(tid_tile - row * tiles_per_row);
    const int hi = tr / ncb;
    const int cb = tr - hi * ncb;

    const int per_poly = rows.nlimbs * rows.split;
    const long long b = row / per_poly;
    const int rem = (int)(row - b * per_poly);
    const int slot = rem / rows.split;
    const int blk = rem - slot * rows.split;

    const PrimeInfo* pi = primes + rows.prime[slot];
    const uint64_t q = pi->q;
    const uint64_t q2 = pi->two_q;
    const long long off = (long long)blk * P;
    const uint64_t* __restrict__ src = rows.in[slot] + b * rows.in_batch_stride + off;
    uint64_t* __restrict__ dst = rows.out[slot] + b * rows.batch_stride + off;

    const int base = (hi << (bit_lo + k)) + (cb << logC);
    if (rows.reduce_input && !INV) {
        const PrimeInfo pr = *pi;
        for (int e = threadIdx.x; e < T; e += blockDim.x)
            tile[e] = reduce64(src[base + ((e >> logC) << bit_lo) + (e & (C - 1))], pr);
    } else {
        for (int e = threadIdx.x; e < T; e += blockDim.x)
            tile[e] = src[base + ((e >> logC) << bit_lo) + (e & (C - 1))];
    }
    __syncthreads();

    const ulonglong2* __restrict__ tw =
        reinterpret_cast<const ulonglong2*>(INV ? pi->inv : pi->fwd);
    const int half = T >> 1;
    for (int step = 0; step < k; ++step) {
        const int p = INV ? step : (k - 1 - step);
        const int bit = bit_lo + p;
        const int twbase = INV ? (P >> (bit + 1)) : (1 << (logP - 1 - bit));
        const bool final_stage = INV && last && (step == k - 1);
        for (int bf = threadIdx.x; bf < half; bf += blockDim.x) {
            const int c = bf & (C - 1);
            const int m2 = bf >> logC;
            const int mid = ((m2 >> p) << (p + 1)) | (m2 & ((1 << p) - 1));
            const int grp = (hi << (k - p - 1)) | (mid >> (p + 1));
            const int e0 = (mid << logC) | c;
            const int e1 = e0 + (1 << (p + logC));
            uint64_t x0 = tile[e0];
            uint64_t x1 = tile[e1];
            if (!INV) {
                const ulonglong2 w = tw[twbase + grp];
                const uint64_t u = csub(x0, q2);
                const uint64_t v = shoup_lazy(x1, w.x, w.y, q);
                x0 = u + v;
                x1 = u + q2 - v;
            } else if (!final_stage) {
                const ulonglong2 w = tw[twbase + grp];
                const uint64_t u = x0, v = x1;
                x0 = csub(u + v, q2);
                x1 = shoup_lazy(u + q2 - v, w.x, w.y, q);
            } else {
                const uint64_t u = x0, v = x1;
                x0 = shoup(u + v, pi->p_inv, pi->p_inv_sh, q);
                x1 = shoup(u + q2 - v, pi->inv_last, pi->inv_last_sh, q);
            }
            tile[e0] = x0;
            tile[e1] = x1;
        }
        __syncthreads();
    }

    for (int e = threadIdx.x; e < T; e += blockDim.x) {
        uint64_t x = tile[e];
        if (last && !INV) x = csub(csub(x, q2), q);
        dst[base + ((e >> logC) << bit_lo) + (e & (C - 1))] = x;
    }
}

template <bool INV>
int run_pass(const RowSet& rows, const PrimeInfo* d_primes, int bit_lo, int k, int logC, bool last,
             cudaStream_t stream) {
    static bool attr_set = false;
    const int T = 1 << (k + logC);
    const size_t smem = sizeof(uint64_t) * (size_t)T;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_ntt_pass<INV>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        if (e != cudaSuccess) return (int)e;
        attr_set = true;
    }
    const long long P = 1LL << rows.logP;
    const long long tiles_per_row = (P >> (bit_lo + k)) * ((1LL << bit_lo) >> logC);
    const long long nrows = (long long)rows.batch * rows.nlimbs * rows.split;
    const long long grid = nrows * tiles_per_row;
    if (grid <= 0) return 0;
    int threads = T / 2;
    if (threads > 1024) threads = 1024;
    if (threads < 32) threads = 32;
    k_ntt_pass<INV><<<(unsigned)grid, threads, smem, stream>>>(rows, d_primes, bit_lo, k, logC,
                                                              last ? 1 : 0);
    note_launch();
    return (int)cudaGetLastError();
}

}  // namespace

int launch_ntt_rb(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream);
int launch_ntt_f64(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream);

namespace {
// The register-blocked kernels use 16-byte vector accesses on row segments.
bool rows_aligned16(const RowSet& rows) {
    if ((rows.batch_stride | rows.in_batch_stride) & 1) return false;
    for (int k = 0; k < rows.nlimbs; ++k)
        if ((((uintptr_t)rows.out[k]) | ((uintptr_t)rows.in[k])) & 15) return false;
    return true;
}
int g_force_generic = -1;
int g_force_int = -1;
}  // namespace

namespace {
void read_force_flags() {
    if (g_force_generic < 0) {
        const char* s = getenv("VFHE_CUDA_NTT_GENERIC");
        g_force_generic = (s && atoi(s)) ? 1 : 0;
    }
    if (g_force_int < 0) {
        const char* s = getenv("VFHE_CUDA_NTT_INT");
        g_force_int = (s && atoi(s)) ? 1 : 0;
    }
}
}  // namespace

bool ntt_f64_eligible(const RowSet& rows) {
    read_force_flags();
    return !rows.table && rows.batch > 0 && rows.nlimbs > 0 && !g_force_generic && !g_force_int && rows.fp64 &&
           rows.logP >= 8 && rows.logP <= 17 && rows_aligned16(rows);
}

int launch_ntt(const RowSet& rows, const PrimeInfo* d_primes, bool inverse, cudaStream_t stream) {
    const int logP = rows.logP;
    if (rows.table) {
        // work lists are built only from FP64-eligible, 16-byte aligned rows
        if (rows.table_rows <= 0) return 0;
        const int e = launch_ntt_f64(rows, d_primes, inverse, stream);
        return e == -1 ? (int)cudaErrorInvalidValue : e;
    }
    if (rows.batch <= 0 || rows.nlimbs <= 0) return 0;
    read_force_flags();
    if (!g_force_generic && logP >= 8 && logP <= 17 && rows_aligned16(rows)) {
        if (rows.fp64 && !g_force_int) {
            const int e = launch_ntt_f64(rows, d_primes, inverse, stream);
            if (e != -1) return e;
        }
        const int e = launch_ntt_rb(rows, d_primes, inverse, stream);
        if (e != -1) return e;
    }
    if (logP <= 14) {
        return inverse ? run_pass<true>(rows, d_primes, 0, logP, 0, true, stream)
                       : run_pass<false>(rows, d_primes, 0, logP, 0, true, stream);
    }
    // Two passes: the low 12 index bits form contiguous 4096-point chunks; the high
    // bits form columns, handled with 2^(12-k1) adjacent columns per tile.
    const int k_lo = 12;
    const int k_hi = logP - k_lo;
    const int logC = k_lo - k_hi;
    // the second pass works in place on the first pass's output
    RowSet second = rows;
    for (int i = 0; i < rows.nlimbs; ++i) second.in[i] = rows.out[i];
    second.in_batch_stride = rows.batch_stride;
    second.reduce_input = 0;
    int err;
    if (!inverse) {
        err = run_pass<false>(rows, d_primes, k_lo, k_hi, logC, false, stream);
        if (err) return err;
        return run_pass<false>(second, d_primes, 0, k_lo, 0, true, stream);
    }
    err = run_pass<true>(rows, d_primes, 0, k_lo, 0, false, stream);
    if (err) return err;
    return run_pass<true>(second, d_primes, k_lo, k_hi, logC, true, stream);
}

}  // namespace vc
