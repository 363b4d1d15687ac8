// Batched device API (Part 2 of vfhe_cuda.h): plain device pointers and a caller
// stream, no managed memory and no synchronisation.
#include <cuda_runtime.h>
#include <string.h>

#include "abi_common.cuh"

using namespace vc;

namespace vc {

bool batch_rowset(IncNtt* t, uint64_t* d_out, const uint64_t* d_in, uint64_t batch, const uint32_t* limbs,
                  uint32_t nlimbs, RowSet* rs, const char* where) {
    if (!t || !limbs || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs) {
        set_error(where, "bad pool or limb list");
        return false;
    }
    memset(rs, 0, sizeof *rs);
    const uint64_t N = t->pub.N;
    for (uint32_t k = 0; k < nlimbs; ++k) {
        if (limbs[k] >= t->pub.l) {
            set_error(where, "limb index outside the pool");
            return false;
        }
        rs->out[k] = d_out + (uint64_t)k * N;
        rs->in[k] = d_in + (uint64_t)k * N;
        rs->prime[k] = limbs[k];
    }
    rs->nlimbs = (int)nlimbs;
    rs->split = (int)t->pub.split_degree;
    rs->logP = t->logP;
    rs->batch = (int)batch;
    rs->batch_stride = (long long)(nlimbs * N);
    return true;
}

}  // namespace vc

extern "C" {

int vfhe_cuda_ntt_batch(void* ntt, int inverse, uint64_t* d_out, const uint64_t* d_in, uint64_t batch,
                        const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    RowSet rs;
    if (!batch_rowset(as_ntt(ntt), d_out, d_in, batch, limbs, nlimbs, &rs, "vfhe_cuda_ntt_batch")) return 1;
    const int e = launch_ntt(rs, as_ntt(ntt)->d_info, inverse != 0, (cudaStream_t)stream_);
    return check_cuda(e, "vfhe_cuda_ntt_batch") ? 0 : 1;
}

int vfhe_cuda_poly_mul_batch(void* ntt, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                             uint64_t batch, const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    IncNtt* t = as_ntt(ntt);
    if (!t || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs) {
        set_error("vfhe_cuda_poly_mul_batch", "bad pool or limb list");
        return 1;
    }
    const uint64_t N = t->pub.N;
    EwSet s = empty_set((long long)N);
    for (uint32_t k = 0; k < nlimbs; ++k) {
        s.out[k] = d_out + (uint64_t)k * N;
        s.a[k] = d_a + (uint64_t)k * N;
        s.b[k] = d_b + (uint64_t)k * N;
        s.prime[k] = limbs[k];
    }
    s.nlimbs = (int)nlimbs;
    s.batch = (int)batch;
    s.batch_stride = (long long)(nlimbs * N);
    const int e = launch_inc_product(0, s, (int)t->pub.split_degree, t->logP, t->d_info, (cudaStream_t)stream_);
    return check_cuda(e, "vfhe_cuda_poly_mul_batch") ? 0 : 1;
}

int vfhe_cuda_ntt_mul_intt_batch(void* ntt, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                                 uint64_t batch, const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    IncNtt* t = as_ntt(ntt);
    if (!t) return 1;
    const uint64_t elems = batch * nlimbs * t->pub.N;
    uint64_t* tmp = (uint64_t*)device_alloc(elems * 8);
    if (!tmp) return 1;
    cudaStream_t st = (cudaStream_t)stream_;
    int rc = vfhe_cuda_ntt_batch(ntt, 0, tmp, d_b, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_ntt_batch(ntt, 0, d_out, d_a, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_poly_mul_batch(ntt, d_out, d_out, tmp, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_ntt_batch(ntt, 1, d_out, d_out, batch, limbs, nlimbs, stream_);
    // the scratch may only be recycled once the stream has consumed it
    cudaStreamSynchronize(st);
    device_free(tmp);
    return rc;
}

uint64_t vfhe_cuda_ckks_mul_workspace_bytes(void* ntt, uint64_t batch, uint32_t nlimbs) {
    (void)ntt; (void)batch; (void)nlimbs;
    return 0;
}

int vfhe_cuda_ckks_mul_relin_rescale_batch(void* ntt, uint64_t* d_out, const uint64_t* d_ct1, const uint64_t* d_ct2,
                                           uint64_t batch, const uint32_t* limbs, uint32_t nlimbs,
                                           uint32_t special, const uint64_t* d_rlk, void* workspace,
                                           void* stream_) {
    (void)ntt; (void)d_out; (void)d_ct1; (void)d_ct2; (void)batch; (void)limbs; (void)nlimbs; (void)special;
    (void)d_rlk; (void)workspace; (void)stream_;
    set_error("vfhe_cuda_ckks_mul_relin_rescale_batch", "not built yet");
    return 1;
}

uint64_t vfhe_cuda_ckks_rotate_workspace_bytes(void* ntt, uint64_t batch, uint32_t nlimbs) {
    (void)ntt; (void)batch; (void)nlimbs;
    return 0;
}

int vfhe_cuda_ckks_rotate_batch(void* ntt, uint64_t* d_out, const uint64_t* d_ct, uint64_t batch,
                                const uint32_t* limbs, uint32_t nlimbs, uint32_t special, uint64_t gen,
                                const uint64_t* d_gk, void* workspace, void* stream_) {
    (void)ntt; (void)d_out; (void)d_ct; (void)batch; (void)limbs; (void)nlimbs; (void)special; (void)gen;
    (void)d_gk; (void)workspace; (void)stream_;
    set_error("vfhe_cuda_ckks_rotate_batch", "not built yet");
    return 1;
}

}  // extern "C"
