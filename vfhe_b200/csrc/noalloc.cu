// Allocation-free variant of the batched NTT -> product -> INTT chain.
//
// vfhe_cuda_ntt_mul_intt_batch needs scratch for the transformed second operand and
// takes it from device memory the engine allocates.  Some callers cannot let a
// library allocate on the GPU: code that builds a CUDA graph by stream capture (a
// cudaMalloc during capture is an error), host runtimes that own the device memory
// themselves (a JVM or Go service that pre-reserves its HBM budget through one
// allocator), and latency-bound serving loops for which a cudaMalloc, which can
// synchronise the device, is not acceptable.  This entry point serves them: its
// scratch is a fixed array in the library's device image, so it calls no cudaMalloc,
// cudaFree or other allocating routine.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "abi_common.cuh"

namespace {

// 2^20 residues (8 MiB).  Every GPU that loads the library holds this array until
// the process exits.
constexpr uint64_t kScratchWords = 1ULL << 20;
static __device__ __align__(256) uint64_t g_noalloc_scratch[kScratchWords];

// Device address of the array per device ordinal.  The array's name in host code is
// only a host-side stand-in for the symbol, never a device address: it is resolved
// with cudaGetSymbolAddress, once per device, with that device current.
constexpr int kMaxDevices = 64;
uint64_t* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

uint64_t* scratch_for_current_device(const char* where) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        vc::set_error(where, "no current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            vc::set_error(where, "cudaGetSymbolAddress of the static scratch array failed");
            return nullptr;
        }
        g_scratch_addr[dev] = (uint64_t*)p;
    }
    return g_scratch_addr[dev];
}

}  // namespace

extern "C" {

int vfhe_cuda_ntt_mul_intt_batch_noalloc(void* ntt, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                                         uint64_t batch, const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    static const char* const where = "vfhe_cuda_ntt_mul_intt_batch_noalloc";
    using namespace vc;
    // ensure_ready only selects the device and creates the engine's stream; it
    // allocates no device memory
    if (!ensure_ready()) return 1;
    // transform schedules that would allocate a counter buffer fall back to kernels that do not
    const FlowNoAlloc no_alloc;
    IncNtt* t = as_ntt(ntt);
    if (!t || !limbs || !d_out || !d_a || !d_b || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs || batch == 0) {
        set_error(where, "bad pool, buffers or limb list");
        return 1;
    }
    const uint64_t N = t->pub.N;
    if (batch > kScratchWords / N / nlimbs) {
        set_error(where, "batch * nlimbs * N exceeds the 2^20-residue (8 MiB) static scratch; "
                         "split the batch or use vfhe_cuda_ntt_mul_intt_batch");
        return 1;
    }
    for (uint32_t k = 0; k < nlimbs; ++k)
        if (limbs[k] >= t->pub.l) {
            set_error(where, "limb index outside the pool");
            return 1;
        }
    {
        int dev = -1;
        if (cudaGetDevice(&dev) != cudaSuccess || dev != ctx().device) {
            set_error(where, "call with the engine's device current (its tables live there)");
            return 1;
        }
    }
    uint64_t* scratch = scratch_for_current_device(where);
    if (!scratch) return 1;
    cudaStream_t st = (cudaStream_t)stream_;

    // transforms: scratch <- NTT(b), out <- NTT(a); the scratch is fully overwritten by
    // the first transform before anything reads it, so it needs no clearing
    RowSet rs;
    memset(&rs, 0, sizeof rs);
    for (uint32_t k = 0; k < nlimbs; ++k) {
        rs.in[k] = d_b + (uint64_t)k * N;
        rs.out[k] = scratch + (uint64_t)k * N;
        rs.prime[k] = limbs[k];
    }
    rs.nlimbs = (int)nlimbs;
    rs.split = (int)t->pub.split_degree;
    rs.logP = t->logP;
    rs.batch = (int)batch;
    rs.batch_stride = (long long)(nlimbs * N);
    rs.in_batch_stride = rs.batch_stride;
    mark_fp64(rs, t);
    if (!check_cuda(launch_ntt(rs, t->d_info, false, st), where)) return 1;
    for (uint32_t k = 0; k < nlimbs; ++k) {
        rs.in[k] = d_a + (uint64_t)k * N;
        rs.out[k] = d_out + (uint64_t)k * N;
    }
    if (!check_cuda(launch_ntt(rs, t->d_info, false, st), where)) return 1;

    // out <- out * scratch (incomplete product), then out <- INTT(out)
    EwSet s = empty_set((long long)N);
    for (uint32_t k = 0; k < nlimbs; ++k) {
        s.out[k] = d_out + (uint64_t)k * N;
        s.a[k] = d_out + (uint64_t)k * N;
        s.b[k] = scratch + (uint64_t)k * N;
        s.prime[k] = limbs[k];
    }
    s.nlimbs = (int)nlimbs;
    s.batch = (int)batch;
    s.batch_stride = (long long)(nlimbs * N);
    if (!check_cuda(launch_inc_product(0, s, (int)t->pub.split_degree, t->logP, t->d_info, st), where)) return 1;
    for (uint32_t k = 0; k < nlimbs; ++k) rs.in[k] = d_out + (uint64_t)k * N;
    if (!check_cuda(launch_ntt(rs, t->d_info, true, st), where)) return 1;
    return 0;
}

}  // extern "C"
