// misc.cdef / vfhe_cpu.cdef surface, RNS base conversion, and the parts of the
// reference surface that lie outside this engine's hot path (multiprecision, field
// extensions, GP25).  The latter exist so that a cffi module built
// from the reference cdefs links against this library; calling one records an error.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include "abi_common.cuh"

using namespace vc;

namespace {

void unsupported(const char* where) {
    set_error(where, "outside the cuda engine's hot path (use the portable or avx512ifma engine)");
}

struct BaseConv {
    uint64_t in_mask, out_mask;
    std::vector<uint32_t> D, P;              // source / target limb indices
    std::vector<uint64_t> Dhat, Dhat_sh;     // (prod_{k!=j} q_k)^-1 mod q_j
    std::vector<uint64_t> DmodP;             // [v][w]: prod_{k!=j} q_k mod p_i
    uint64_t* d_tab = nullptr;               // device copy: Dhat, Dhat_sh, DmodP
};

// Fast base extension (rns_polynomial.c:738-822): for every target limb i,
// out_i = sum_j ((in_j * Dhat_j mod q_j) mod p_i) * DmodP[i][j] mod p_i.
__global__ void k_base_conv(const __grid_constant__ EwSet set, const uint64_t* __restrict__ tab, int w,
                            const PrimeInfo* __restrict__ primes, const uint32_t* __restrict__ src_prime) {
    const int i = blockIdx.y;  // target slot
    const PrimeInfo pt = primes[set.prime[i]];
    const uint64_t* dhat = tab;
    const uint64_t* dhat_sh = tab + w;
    const uint64_t* dmodp = tab + 2 * w + (long long)i * w;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < set.n;
         x += (long long)gridDim.x * blockDim.x) {
        uint64_t acc = 0;
        for (int j = 0; j < w; ++j) {
            const PrimeInfo& ps = primes[src_prime[j]];
            const uint64_t v = shoup(set.b[j][x], dhat[j], dhat_sh[j], ps.q);
            acc = add_mod(acc, mul_mod(reduce64(v, pt), dmodp[j], pt), pt.q);
        }
        set.out[i][x] = acc;
    }
}

}  // namespace

extern "C" {

const char* vfhe_engine_active(void) { return "cuda"; }

void vfhe_prng_set_deterministic_seed(uint64_t seed) { prng_set(seed, true); }

void vfhe_prng_clear_deterministic_seed(void) { prng_set(0, false); }

int vfhe_cpu_supports(const char* capability) {
    // The cuda engine needs no CPU feature; it answers for the GPU instead.
    if (capability && strcmp(capability, "cuda") == 0) {
        int n = 0;
        return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    }
    return 0;
}

void* init_base_conversion_params(void* ntt, uint64_t in_mask, uint64_t out_mask) {
    VC_ENTER_RET("init_base_conversion_params", nullptr);
    IncNtt* t = as_ntt(ntt);
    BaseConv* bc = new BaseConv();
    bc->in_mask = in_mask;
    bc->out_mask = out_mask;
    const uint64_t l = t->pub.l;
    for (uint64_t i = 0; i < l && i < 64; ++i)
        if (in_mask & (1ULL << i)) bc->D.push_back((uint32_t)i);
    for (uint64_t i = 0; i < l && i < 64; ++i)
        if ((out_mask & (1ULL << i)) && !(in_mask & (1ULL << i))) bc->P.push_back((uint32_t)i);
    const size_t w = bc->D.size(), v = bc->P.size();
    if (v == 0) return bc;
    if (w == 0) {
        set_error(vc_where_, "no source limbs (rns_polynomial.c:668)");
        delete bc;
        return nullptr;
    }
    for (size_t j = 0; j < w; ++j) {
        const uint64_t qj = t->info[bc->D[j]].q;
        uint64_t prod = 1;
        for (size_t k = 0; k < w; ++k)
            if (k != j) prod = host_mul_mod(prod, t->info[bc->D[k]].q % qj, qj);
        bc->Dhat.push_back(host_inv_mod(prod, qj));
        bc->Dhat_sh.push_back(host_shoup(bc->Dhat.back(), qj));
    }
    for (size_t i = 0; i < v; ++i) {
        const uint64_t pi = t->info[bc->P[i]].q;
        for (size_t j = 0; j < w; ++j) {
            uint64_t prod = 1;
            for (size_t k = 0; k < w; ++k)
                if (k != j) prod = host_mul_mod(prod, t->info[bc->D[k]].q % pi, pi);
            bc->DmodP.push_back(prod);
        }
    }
    std::vector<uint64_t> tab;
    tab.insert(tab.end(), bc->Dhat.begin(), bc->Dhat.end());
    tab.insert(tab.end(), bc->Dhat_sh.begin(), bc->Dhat_sh.end());
    tab.insert(tab.end(), bc->DmodP.begin(), bc->DmodP.end());
    std::vector<uint64_t> srcp(bc->D.begin(), bc->D.end());
    tab.insert(tab.end(), srcp.begin(), srcp.end());
    if (!VC_CHECK(cudaMalloc(&bc->d_tab, tab.size() * 8)) ||
        !VC_CHECK(cudaMemcpy(bc->d_tab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice)) ||
        !VC_CHECK(cudaStreamSynchronize(0))) {  // the upload has landed before engine-stream kernels read it
        delete bc;
        return nullptr;
    }
    return bc;
}

void free_base_conversion_params(void* params) {
    BaseConv* bc = (BaseConv*)params;
    if (!bc) return;
    if (bc->d_tab) cudaFree(bc->d_tab);
    delete bc;
}

void polynomial_base_conversion_RNSc(void* out, void* in, void* params) {
    VC_ENTER("polynomial_base_conversion_RNSc");
    Poly* o = as_poly(out);
    Poly* i = as_poly(in);
    const uint64_t in_mask = i->pub.rns_mask, out_mask = o->pub.rns_mask;
    if (o != i) {
        EwSet s = poly_set(o, i, nullptr, in_mask & out_mask);
        prefetch_poly(i);
        prefetch_poly(o);
        VC_CHECK(launch_ew(EW_COPY, s, pool_of(o)->d_info, stream()));
    }
    BaseConv* bc = (BaseConv*)params;
    bool own = false;
    if (!bc) {
        bc = (BaseConv*)init_base_conversion_params(o->pub.ntt, in_mask, out_mask);
        own = true;
    } else if (bc->in_mask != in_mask || bc->out_mask != out_mask) {
        set_error(vc_where_, "parameters were built for other masks (rns_polynomial.c:749-750)");
        return;
    }
    if (bc && !bc->P.empty()) {
        const int w = (int)bc->D.size(), v = (int)bc->P.size();
        if (w > kMaxLimbs || v > kMaxLimbs) {
            set_error(vc_where_, "too many limbs");
        } else {
            EwSet s = empty_set((long long)o->pub.ntt->N);
            for (int t = 0; t < v; ++t) {
                s.out[t] = o->pub.coeffs[bc->P[t]];
                s.prime[t] = bc->P[t];
            }
            for (int j = 0; j < w; ++j) s.b[j] = i->pub.coeffs[bc->D[j]];
            s.nlimbs = v;
            long long blocks = (s.n + 255) / 256;
            if (blocks > 1024) blocks = 1024;
            const uint32_t* d_src = nullptr;
            // source prime indices are stored after the tables as uint64; stage as uint32
            std::vector<uint32_t> src(bc->D.begin(), bc->D.end());
            uint32_t* d_src_buf = (uint32_t*)device_alloc(src.size() * 4);
            VC_CHECK(cudaMemcpyAsync(d_src_buf, src.data(), src.size() * 4, cudaMemcpyHostToDevice, stream()));
            d_src = d_src_buf;
            k_base_conv<<<dim3((unsigned)blocks, (unsigned)v), 256, 0, stream()>>>(
                s, bc->d_tab, w, pool_of(o)->d_info, d_src);
            VC_CHECK(cudaGetLastError());
            vc::sync(vc_where_);
            device_free(d_src_buf);
        }
    }
    o->pub.rns_mask = out_mask;
    if (own) free_base_conversion_params(bc);
    VC_FINISH();
}

// ---- complex FFT (CKKS encoding): complex_fft.cu

// ---- multiprecision (portable layout: one uint64 per digit vector)
int get_mp_vector_size(void) { return 1; }
void mp_scale(void* out, void* in, void* m) { (void)out; (void)in; (void)m; unsupported("mp_scale"); }
void mp_sub(void* out, void* a, void* b) { (void)out; (void)a; (void)b; unsupported("mp_sub"); }
void* mp_load(uint64_t* in, uint64_t d) { (void)in; (void)d; unsupported("mp_load"); return nullptr; }
mp_vector_t* load_m512(uint64_t in) { (void)in; unsupported("load_m512"); return nullptr; }
void* new_mp_polynomial(uint64_t N, uint64_t d) { (void)N; (void)d; unsupported("new_mp_polynomial"); return nullptr; }
void mp_polynomial_from_RNS(void* out, void* in, MPScalar* PW, void* q, mp_vector_t* m, uint64_t k) {
    (void)out; (void)in; (void)PW; (void)q; (void)m; (void)k;
    unsupported("mp_polynomial_from_RNS");
}
void mp_polynomial_to_RNSc(void* out, void* in) { (void)out; (void)in; unsupported("mp_polynomial_to_RNSc"); }

// ---- field extensions
void* field_new_proc(uint64_t q) { (void)q; unsupported("field_new_proc"); return nullptr; }
void field_ext_add(uint64_t* c, const uint64_t* a, const uint64_t* b, uint64_t d, uint64_t q) {
    (void)c; (void)a; (void)b; (void)d; (void)q; unsupported("field_ext_add");
}
void field_ext_sub(uint64_t* c, const uint64_t* a, const uint64_t* b, uint64_t d, uint64_t q) {
    (void)c; (void)a; (void)b; (void)d; (void)q; unsupported("field_ext_sub");
}
void field_ext_neg(uint64_t* c, const uint64_t* a, uint64_t d, uint64_t q) {
    (void)c; (void)a; (void)d; (void)q; unsupported("field_ext_neg");
}
void field_ext_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, uint64_t d, uint64_t w, void* proc) {
    (void)c; (void)a; (void)b; (void)d; (void)w; (void)proc; unsupported("field_ext_mul");
}
void field_ext_pow(uint64_t* res, const uint64_t* base, uint64_t exp_lo, uint64_t exp_hi, uint64_t d, uint64_t w,
                   void* proc) {
    (void)res; (void)base; (void)exp_lo; (void)exp_hi; (void)d; (void)w; (void)proc; unsupported("field_ext_pow");
}
int field_ext_inv(uint64_t* ainv, const uint64_t* a, uint64_t d, uint64_t w, void* proc) {
    (void)ainv; (void)a; (void)d; (void)w; (void)proc; unsupported("field_ext_inv");
    return 0;
}
void field_sample_random_element(uint64_t* a, const uint8_t* seed, uint64_t seed_len, uint64_t d, uint64_t mod) {
    (void)a; (void)seed; (void)seed_len; (void)d; (void)mod; unsupported("field_sample_random_element");
}
void field_hash_element(uint8_t* out, const uint64_t* a, uint64_t d) {
    (void)out; (void)a; (void)d; unsupported("field_hash_element");
}
int field_ext_is_equal(const uint64_t* a, const uint64_t* b, uint64_t d) {
    if (!a || !b) return 0;
    return memcmp(a, b, d * sizeof(uint64_t)) == 0;
}
void field_base_conversion(uint64_t* out, const uint64_t* in, uint64_t source_component,
                           uint64_t target_component, uint64_t d, uint64_t poly_size, const uint64_t* w_i,
                           void* proc) {
    (void)out; (void)in; (void)source_component; (void)target_component; (void)d; (void)poly_size; (void)w_i;
    (void)proc;
    unsupported("field_base_conversion");
}
void ntt_free_proc(void* proc) { (void)proc; }
uint64_t inverse_mod_eea(uint64_t a, uint64_t p) { return p ? host_inv_mod(a % p, p) : 0; }

}  // extern "C"
