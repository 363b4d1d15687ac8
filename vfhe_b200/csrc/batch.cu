// Batched device API (Part 2 of vfhe_cuda.h): plain device pointers and a caller
// stream, no managed memory, no synchronisation unless the engine has to allocate.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "abi_common.cuh"

using namespace vc;

namespace vc {
uint64_t ckks_mul_ws_elems(uint64_t N, uint64_t B, uint64_t L);
uint64_t ckks_rot_ws_elems(uint64_t N, uint64_t B, uint64_t L);
int ckks_mul_relin_rescale(IncNtt* t, uint64_t* out, const uint64_t* ct1, const uint64_t* ct2, uint64_t B,
                           const uint32_t* limbs, uint32_t L, uint32_t special, const uint64_t* rlk, uint64_t* ws,
                           cudaStream_t st);
int ckks_rotate(IncNtt* t, uint64_t* out, const uint64_t* ct, uint64_t B, const uint32_t* limbs, uint32_t L,
                uint32_t special, const uint64_t* gens, const uint64_t* const* gks, uint64_t* ws, cudaStream_t st);
uint64_t cggi_ws_elems(uint64_t N, uint64_t B, uint64_t n, uint32_t L0);
int rlwe_encrypt(IncNtt* t, uint64_t* out, const uint64_t* msg, uint64_t B, const uint32_t* limbs, uint32_t L,
                 const uint64_t* sk, double sigma, cudaStream_t st);
int prng_blocks(uint32_t* out, uint64_t nblocks, const uint32_t* key8, uint64_t counter0, uint64_t nonce,
                cudaStream_t st);
int rlwe_gen_ksk(IncNtt* t, uint64_t* out, const uint64_t* src, uint64_t nsrc, const uint32_t* limbs, uint32_t L,
                 const uint64_t* factors, const uint64_t* sk, double sigma, cudaStream_t st);
int cggi_bootstrap(IncNtt* t, uint64_t* out_a, uint64_t* out_b, const uint64_t* in_a, const uint64_t* in_b,
                   uint64_t B, uint32_t n, const uint32_t* limbs, uint32_t L0, uint32_t special, const uint64_t* bk,
                   const uint64_t* tv, uint64_t torus_base, uint64_t* ws, cudaStream_t st);
}  // namespace vc

namespace {

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
    rs->in_batch_stride = rs->batch_stride;
    return true;
}

// Scratch owned by the engine when the caller passes no workspace: one buffer per
// stream, grown on demand.  Calls on one stream are ordered by that stream, so they
// may share its buffer; calls on different streams get different buffers and never
// race on scratch contents.  A buffer is freed only after its own stream has drained.
// The map is guarded by a mutex, so host threads may call concurrently.
uint64_t* engine_workspace(size_t bytes, cudaStream_t st) {
    struct Buf {
        void* p;
        size_t cap;
    };
    static std::mutex mu;
    static std::unordered_map<cudaStream_t, Buf> bufs;
    std::lock_guard<std::mutex> lk(mu);
    Buf& b = bufs[st];
    if (bytes > b.cap) {
        if (b.p) {
            cudaStreamSynchronize(st);
            cudaFree(b.p);
        }
        b.p = nullptr;
        b.cap = 0;
        if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
            b.p = nullptr;
            set_error("workspace", "cudaMalloc failed");
            return nullptr;
        }
        b.cap = bytes;
    }
    return (uint64_t*)b.p;
}

// An empty batch: a successful no-op (nothing is launched and no scratch is touched)
// once the pool and the limb list check out; otherwise the call's usual error.
int empty_batch(void* ntt, const uint32_t* limbs, uint32_t nlimbs, const char* where) {
    IncNtt* t = as_ntt(ntt);
    if (!t || !limbs || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs) {
        set_error(where, "bad pool or limb list");
        return 1;
    }
    for (uint32_t k = 0; k < nlimbs; ++k)
        if (limbs[k] >= t->pub.l) {
            set_error(where, "limb index outside the pool");
            return 1;
        }
    return 0;
}

// Largest batch one pass of the CKKS and key-switch kernels takes: their grids' y
// dimension (at most 65535) counts at most batch x 2 x (nlimbs + 1) rows.  Larger
// batches run as consecutive chunks on the same stream, sharing the workspace.
uint64_t ckks_max_chunk(uint32_t nlimbs) { return 65535 / (2 * ((uint64_t)nlimbs + 1)); }

}  // namespace

extern "C" {

int vfhe_cuda_ntt_batch(void* ntt, int inverse, uint64_t* d_out, const uint64_t* d_in, uint64_t batch,
                        const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    RowSet rs;
    if (!batch_rowset(as_ntt(ntt), d_out, d_in, batch, limbs, nlimbs, &rs, "vfhe_cuda_ntt_batch")) return 1;
    mark_fp64(rs, as_ntt(ntt));
    const int e = launch_ntt(rs, as_ntt(ntt)->d_info, inverse != 0, (cudaStream_t)stream_);
    return check_cuda(e, "vfhe_cuda_ntt_batch") ? 0 : 1;
}

int vfhe_cuda_poly_mul_batch(void* ntt, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                             uint64_t batch, const uint32_t* limbs, uint32_t nlimbs, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_poly_mul_batch");
    IncNtt* t = as_ntt(ntt);
    if (!t || !limbs || nlimbs == 0 || nlimbs > (uint32_t)kMaxLimbs) {
        set_error("vfhe_cuda_poly_mul_batch", "bad pool or limb list");
        return 1;
    }
    const uint64_t N = t->pub.N;
    EwSet s = empty_set((long long)N);
    for (uint32_t k = 0; k < nlimbs; ++k) {
        if (limbs[k] >= t->pub.l) {
            set_error("vfhe_cuda_poly_mul_batch", "limb index outside the pool");
            return 1;
        }
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
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_ntt_mul_intt_batch");
    IncNtt* t = as_ntt(ntt);
    if (!t) return 1;
    cudaStream_t st = (cudaStream_t)stream_;
    if (d_out && d_a && d_b && limbs) {
        // one kernel per chain where the shape allows (chain.cu); the same residues
        const int e = launch_chain(t, d_out, d_a, d_b, batch, limbs, nlimbs, st);
        if (e != kChainUnavailable) return check_cuda(e, "vfhe_cuda_ntt_mul_intt_batch") ? 0 : 1;
    }
    uint64_t* tmp = engine_workspace(batch * nlimbs * t->pub.N * 8, st);
    if (!tmp) return 1;
    int rc = vfhe_cuda_ntt_batch(ntt, 0, tmp, d_b, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_ntt_batch(ntt, 0, d_out, d_a, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_poly_mul_batch(ntt, d_out, d_out, tmp, batch, limbs, nlimbs, stream_);
    if (!rc) rc = vfhe_cuda_ntt_batch(ntt, 1, d_out, d_out, batch, limbs, nlimbs, stream_);
    return rc;
}

uint64_t vfhe_cuda_ckks_mul_workspace_bytes(void* ntt, uint64_t batch, uint32_t nlimbs) {
    IncNtt* t = as_ntt(ntt);
    return t ? 8 * ckks_mul_ws_elems(t->pub.N, batch, nlimbs) : 0;
}

int vfhe_cuda_ckks_mul_relin_rescale_batch(void* ntt, uint64_t* d_out, const uint64_t* d_ct1, const uint64_t* d_ct2,
                                           uint64_t batch, const uint32_t* limbs, uint32_t nlimbs,
                                           uint32_t special, const uint64_t* d_rlk, void* workspace,
                                           void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_ckks_mul_relin_rescale_batch");
    IncNtt* t = as_ntt(ntt);
    if (!t || nlimbs < 2) return ckks_mul_relin_rescale(t, d_out, d_ct1, d_ct2, batch, limbs, nlimbs, special, d_rlk,
                                                        nullptr, (cudaStream_t)stream_);  // records the error
    cudaStream_t st = (cudaStream_t)stream_;
    const uint64_t chunk = std::min<uint64_t>(batch, ckks_max_chunk(nlimbs));
    uint64_t* ws = (uint64_t*)workspace;
    if (!ws) ws = engine_workspace(vfhe_cuda_ckks_mul_workspace_bytes(ntt, chunk, nlimbs), st);
    if (!ws) return 1;
    const uint64_t N = t->pub.N;
    for (uint64_t b0 = 0; b0 < batch; b0 += chunk) {
        const uint64_t n = std::min(chunk, batch - b0);
        const int rc = ckks_mul_relin_rescale(t, d_out + b0 * 2 * (nlimbs - 1) * N, d_ct1 + b0 * 2 * nlimbs * N,
                                              d_ct2 + b0 * 2 * nlimbs * N, n, limbs, nlimbs, special, d_rlk, ws, st);
        if (rc) return rc;
    }
    return 0;
}

int vfhe_cuda_rlwe_encrypt_batch(void* ntt, uint64_t* d_out, const uint64_t* d_msg, uint64_t batch,
                                 const uint32_t* limbs, uint32_t nlimbs, const uint64_t* d_sk, double sigma,
                                 void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_rlwe_encrypt_batch");
    return rlwe_encrypt(as_ntt(ntt), d_out, d_msg, batch, limbs, nlimbs, d_sk, sigma, (cudaStream_t)stream_);
}

int vfhe_cuda_gen_ksk_batch(void* ntt, uint64_t* d_out, const uint64_t* d_src, uint64_t nsrc, const uint32_t* limbs,
                            uint32_t nlimbs, const uint64_t* factors, const uint64_t* d_sk, double sigma,
                            void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (nsrc == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_gen_ksk_batch");
    return rlwe_gen_ksk(as_ntt(ntt), d_out, d_src, nsrc, limbs, nlimbs, factors, d_sk, sigma, (cudaStream_t)stream_);
}

int vfhe_cuda_prng_blocks(uint32_t* d_out, uint64_t nblocks, const uint32_t* key, uint64_t counter0, uint64_t nonce,
                          void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (!d_out || !key) {
        set_error("vfhe_cuda_prng_blocks", "null buffer or key");
        return 1;
    }
    if (nblocks == 0) return 0;
    return prng_blocks(d_out, nblocks, key, counter0, nonce, (cudaStream_t)stream_);
}

uint64_t vfhe_cuda_ckks_rotate_workspace_bytes(void* ntt, uint64_t batch, uint32_t nlimbs) {
    IncNtt* t = as_ntt(ntt);
    return t ? 8 * ckks_rot_ws_elems(t->pub.N, batch, nlimbs) : 0;
}

int vfhe_cuda_ckks_rotate_batch(void* ntt, uint64_t* d_out, const uint64_t* d_ct, uint64_t batch,
                                const uint32_t* limbs, uint32_t nlimbs, uint32_t special, const uint64_t* gens,
                                const uint64_t* const* d_gks, void* workspace, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_ckks_rotate_batch");
    IncNtt* t = as_ntt(ntt);
    if (!t)
        return ckks_rotate(t, d_out, d_ct, batch, limbs, nlimbs, special, gens, d_gks, nullptr,
                           (cudaStream_t)stream_);  // records the error
    if (!d_gks) {
        set_error("vfhe_cuda_ckks_rotate_batch", "no key pointer array");
        return 1;
    }
    cudaStream_t st = (cudaStream_t)stream_;
    const uint64_t chunk = std::min<uint64_t>(batch, ckks_max_chunk(nlimbs));
    uint64_t* ws = (uint64_t*)workspace;
    if (!ws) ws = engine_workspace(vfhe_cuda_ckks_rotate_workspace_bytes(ntt, chunk, nlimbs), st);
    if (!ws) return 1;
    const uint64_t N = t->pub.N;
    for (uint64_t b0 = 0; b0 < batch; b0 += chunk) {
        const uint64_t n = std::min(chunk, batch - b0);
        const int rc = ckks_rotate(t, d_out + b0 * 2 * nlimbs * N, d_ct + b0 * 2 * nlimbs * N, n, limbs, nlimbs,
                                   special, gens ? gens + b0 : nullptr, d_gks + b0, ws, st);
        if (rc) return rc;
    }
    return 0;
}

uint64_t vfhe_cuda_cggi_workspace_bytes(void* ntt, uint64_t batch, uint32_t n, uint32_t nlimbs) {
    IncNtt* t = as_ntt(ntt);
    return t ? 8 * cggi_ws_elems(t->pub.N, batch, n, nlimbs) : 0;
}

int vfhe_cuda_cggi_bootstrap_batch(void* ntt, uint64_t* d_out_a, uint64_t* d_out_b, const uint64_t* d_in_a,
                                   const uint64_t* d_in_b, uint64_t batch, uint32_t n, const uint32_t* limbs,
                                   uint32_t nlimbs, uint32_t special, const uint64_t* d_bk, const uint64_t* d_tv,
                                   uint64_t torus_base, void* workspace, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_cggi_bootstrap_batch");
    IncNtt* t = as_ntt(ntt);
    cudaStream_t st = (cudaStream_t)stream_;
    uint64_t* ws = (uint64_t*)workspace;
    if (!ws) ws = engine_workspace(vfhe_cuda_cggi_workspace_bytes(ntt, batch, n, nlimbs), st);
    if (!ws) return 1;
    return cggi_bootstrap(t, d_out_a, d_out_b, d_in_a, d_in_b, batch, n, limbs, nlimbs, special, d_bk, d_tv,
                          torus_base, ws, st);
}

uint64_t vfhe_cuda_keyswitch_workspace_bytes(void* ntt, uint64_t batch, uint32_t nlimbs) {
    return vfhe_cuda_ckks_rotate_workspace_bytes(ntt, batch, nlimbs);
}

int vfhe_cuda_keyswitch_batch(void* ntt, uint64_t* d_out, const uint64_t* d_ct, uint64_t batch,
                              const uint32_t* limbs, uint32_t nlimbs, uint32_t special, const uint64_t* d_ksk,
                              void* workspace, void* stream_) {
    if (!vc::ensure_ready()) return 1;
    if (batch == 0) return empty_batch(ntt, limbs, nlimbs, "vfhe_cuda_keyswitch_batch");
    IncNtt* t = as_ntt(ntt);
    cudaStream_t st = (cudaStream_t)stream_;
    const uint64_t chunk = std::min<uint64_t>(batch, ckks_max_chunk(nlimbs));
    std::vector<const uint64_t*> keys(chunk, d_ksk);
    if (!t) return ckks_rotate(t, d_out, d_ct, batch, limbs, nlimbs, special, nullptr, keys.data(), nullptr, st);
    uint64_t* ws = (uint64_t*)workspace;
    if (!ws) ws = engine_workspace(vfhe_cuda_keyswitch_workspace_bytes(ntt, chunk, nlimbs), st);
    if (!ws) return 1;
    const uint64_t N = t->pub.N;
    for (uint64_t b0 = 0; b0 < batch; b0 += chunk) {
        const uint64_t n = std::min(chunk, batch - b0);
        const int rc = ckks_rotate(t, d_out + b0 * 2 * nlimbs * N, d_ct + b0 * 2 * nlimbs * N, n, limbs, nlimbs,
                                   special, nullptr, keys.data(), ws, st);
        if (rc) return rc;
    }
    return 0;
}

int vfhe_cuda_device_faults(void) {
    if (!vc::ensure_ready()) return -1;
    int f = 0;
    if (!check_cuda(read_tile_fault(&f), "vfhe_cuda_device_faults")) return -1;
    int m = 0;
    if (!check_cuda(read_mac_fault(&m), "vfhe_cuda_device_faults")) return -1;
    int w = 0;
    if (!check_cuda(read_wl_fault(&w), "vfhe_cuda_device_faults")) return -1;
    int d = 0;
    if (!check_cuda(read_flow_fault(&d), "vfhe_cuda_device_faults")) return -1;
    return f | m | w | d;
}

int vfhe_cuda_clear_device_faults(void) {
    if (!vc::ensure_ready()) return 1;
    if (!check_cuda(clear_tile_fault(), "vfhe_cuda_clear_device_faults")) return 1;
    if (!check_cuda(clear_mac_fault(), "vfhe_cuda_clear_device_faults")) return 1;
    if (!check_cuda(clear_wl_fault(), "vfhe_cuda_clear_device_faults")) return 1;
    if (!check_cuda(clear_flow_fault(), "vfhe_cuda_clear_device_faults")) return 1;
    return 0;
}

int vfhe_cuda_selfcheck_bounded_wait(int32_t tries) {
    if (!vc::ensure_ready()) return -1;
    if (tries <= 0) {
        set_error("vfhe_cuda_selfcheck_bounded_wait", "tries must be positive");
        return -1;
    }
    int gave_up = 0;
    if (!check_cuda(bounded_wait_selfcheck((int)tries, &gave_up), "vfhe_cuda_selfcheck_bounded_wait")) return -1;
    return gave_up;
}

int vfhe_cuda_ntt_set_schedule(uint32_t logP, uint32_t rows_log2, int32_t tile_bits, int32_t tiles_per_cta,
                               int32_t ctas_per_sm) {
    const NttSchedule s = {tile_bits, tiles_per_cta, ctas_per_sm};
    if (!set_ntt_schedule((int)logP, (int)rows_log2, s)) {
        set_error("vfhe_cuda_ntt_set_schedule", "schedule outside the supported shapes");
        return 1;
    }
    return 0;
}

int vfhe_cuda_ntt_get_schedule(uint32_t logP, uint64_t rows, int32_t* out3) {
    if (!out3) return 1;
    const NttSchedule s = get_ntt_schedule((int)logP, (long long)rows);
    out3[0] = s.tile_bits;
    out3[1] = s.tiles_per_cta;
    out3[2] = s.ctas_per_sm;
    return 0;
}

}  // extern "C"
