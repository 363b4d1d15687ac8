// mlwe.cdef surface of the cuda engine (modules/mlwe/python/cdef/mlwe.cdef): LWE and
// MLWE samples, GHS hybrid key switching, tensor product / relinearising multiply,
// automorphisms, MGSW external product and CMUX.
//
// The composite operations follow the reference's algorithms step by step
// (modules/mlwe/c/src/mlwe.c, gadget.c, mgsw.c, lwe.c); each step is an engine kernel
// over all active limbs, and only the outermost call synchronises.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "abi_common.cuh"

using namespace vc;

namespace {

RNS_MLWE new_mlwe(uint64_t N, uint64_t r, uint64_t mask, IncNtt* t) {
    RNS_MLWE m = (RNS_MLWE)calloc(1, sizeof(struct _RNS_MLWE));
    m->a = (RNS_Polynomial*)calloc(r ? r : 1, sizeof(RNS_Polynomial));
    for (uint64_t i = 0; i < r; ++i) m->a[i] = (RNS_Polynomial)poly_create(N, mask, t);
    m->b = (RNS_Polynomial)poly_create(N, mask, t);
    m->r = r;
    return m;
}

void del_mlwe(RNS_MLWE m) {
    if (!m) return;
    for (uint64_t i = 0; i < m->r; ++i) poly_destroy((Poly*)m->a[i]);
    free(m->a);
    poly_destroy((Poly*)m->b);
    free(m);
}

inline Poly* P_(RNS_Polynomial p) { return reinterpret_cast<Poly*>(p); }
inline IncNtt* pool(RNS_MLWE m) { return reinterpret_cast<IncNtt*>(m->b->ntt); }

void prefetch_mlwe(RNS_MLWE m) {
    if (!m) return;
    for (uint64_t i = 0; i < m->r; ++i) prefetch_poly(P_(m->a[i]));
    prefetch_poly(P_(m->b));
}

uint64_t all_rows(Poly* p) {
    return p->pub.allocated_l >= 64 ? ~0ULL : ((1ULL << p->pub.allocated_l) - 1);
}

// mlwe_RNS_trivial_sample_of_zero (mlwe.c:302-312): every row of every component zeroed.
void zero_mlwe(RNS_MLWE m, const char* where) {
    for (uint64_t i = 0; i < m->r; ++i) op_zero_rows(P_(m->a[i]), all_rows(P_(m->a[i])), where);
    op_zero_rows(P_(m->b), all_rows(P_(m->b)), where);
}

// gadget_mul_{add,sub}to_polynomial (gadget.c:5-36): digit j = limb j of the
// coefficient-domain `poly`, lifted to the key's extended limbs, transformed, and
// multiplied into `out` with ksk[digit].
void gadget_mac(RNS_MLWE out, RNS_MLWE* ksk, Poly* poly, int mode, const char* where) {
    IncNtt* t = pool(out);
    Poly* tmp = poly_create(0, ksk[0]->b->rns_mask, reinterpret_cast<IncNtt*>(ksk[0]->b->ntt));
    uint64_t k = 0;
    for (uint64_t j = 0; j < t->pub.l && j < 64; ++j) {
        if (!(poly->pub.rns_mask & (1ULL << j))) continue;
        polynomial_RNSc_mod_reduce_lifted(tmp, poly, j);
        polynomial_RNSc_to_RNS(tmp, tmp);
        RNS_MLWE key = ksk[k++];
        for (uint64_t i = 0; i < out->r; ++i) op_product(P_(out->a[i]), P_(key->a[i]), tmp, mode, where);
        op_product(P_(out->b), P_(key->b), tmp, mode, where);
    }
    poly_destroy(tmp);
}

void set_masks(RNS_MLWE m, uint64_t mask) {
    for (uint64_t i = 0; i < m->r; ++i) m->a[i]->rns_mask = mask;
    m->b->rns_mask = mask;
}

// Gaussian integers (truncated Box-Muller draws), four per ChaCha20 block from ctr on.
__global__ void k_gauss_int(int64_t* out, long long n, double sigma, const __grid_constant__ PrngKey key,
                            uint64_t ctr) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; 4 * j < n;
         j += (long long)gridDim.x * blockDim.x) {
        uint32_t blk[16];
        chacha20_block(key, ctr + j, kStreamInteger, blk);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (4 * j + e >= n) break;
            out[4 * j + e] = (int64_t)(sigma * sqrt(-2.0 * log(unit_open_low(block_u64(blk, 2 * e)))) *
                                       cospi(2.0 * unit_closed_low(block_u64(blk, 2 * e + 1))));
        }
    }
}

// LWE helpers over managed rows.
// lwe_phase (lwe.c:141-156): out[i] = b_i - sum_j a_ij s_ij mod q_i, one CTA per limb.
__global__ void k_lwe_phase(uint64_t* out, const uint64_t* const* a, const uint64_t* b,
                            const uint64_t* const* s, const PrimeInfo* __restrict__ primes, long long n) {
    const int i = blockIdx.x;
    const PrimeInfo pi = primes[i];
    __shared__ uint64_t part[256];
    uint64_t acc = 0;
    for (long long j = threadIdx.x; j < n; j += blockDim.x)
        acc = add_mod(acc, mul_mod(a[i][j], s[i][j], pi), pi.q);
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] = add_mod(part[threadIdx.x], part[threadIdx.x + w], pi.q);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = sub_mod(b[i], part[0], pi.q);
}

// lwe_subto (lwe.c:158-167)
__global__ void k_lwe_subto(uint64_t* const* oa, uint64_t* ob, const uint64_t* const* ia, const uint64_t* ib,
                            const PrimeInfo* __restrict__ primes, long long n) {
    const int i = blockIdx.y;
    const uint64_t q = primes[i].q;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x)
        oa[i][j] = sub_mod(oa[i][j], ia[i][j], q);
    if (blockIdx.x == 0 && threadIdx.x == 0) ob[i] = sub_mod(ob[i], ib[i], q);
}

// lwe_sample (lwe.c:95-121) with the engine's PRNG: uniform a, rounded Gaussian e.
__global__ void k_lwe_uniform(uint64_t* const* a, const PrimeInfo* __restrict__ primes, long long n,
                              const __grid_constant__ PrngKey key, uint64_t ctr) {
    const int i = blockIdx.y;
    const uint64_t q = primes[i].q;
    const long long per_row = (n + 3) / 4;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < per_row;
         j += (long long)gridDim.x * blockDim.x) {
        uint32_t blk[16];
        chacha20_block(key, ctr + (uint64_t)i * per_row + j, kStreamUniform, blk);
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (4 * j + e < n) a[i][4 * j + e] = uniform_mod(block_u64(blk, 2 * e), block_u64(blk, 2 * e + 1), q);
    }
}

dim3 grid2(long long n, int y) {
    long long blocks = (n + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    return dim3((unsigned)blocks, (unsigned)y, 1);
}

// Device array of row pointers for the LWE kernels (managed, cached).
template <typename T>
T* stage_ptrs(const std::vector<T>& v) {
    T* d = (T*)managed_alloc(sizeof(T) * (v.size() ? v.size() : 1));
    if (d) memcpy(d, v.data(), sizeof(T) * v.size());
    return d;
}

// mlwe_extract_LWE (mlwe.c:40-68), one output limb: a[k N + i] = a_k[idx - i] for
// i <= idx, else -a_k[N + idx - i].  One thread per output element.
__global__ void k_extract_rows(uint64_t* out_row, const uint64_t* const* comps, int r, long long N,
                               long long idx, uint64_t q) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)r * N;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / N);
        const long long i = e - (long long)k * N;
        const uint64_t* ak = comps[k];
        out_row[e] = (i <= idx) ? ak[idx - i] : neg_mod(ak[N + idx - i], q);
    }
}

LweSample* new_lwe(uint64_t n, uint64_t l, void* ntt) {
    LweSample* c = new LweSample();
    c->block = (uint64_t*)managed_alloc(sizeof(uint64_t) * (l * n + l));
    c->pub.a = (uint64_t**)malloc(sizeof(uint64_t*) * (l ? l : 1));
    for (uint64_t i = 0; i < l; ++i) c->pub.a[i] = c->block + i * n;
    c->pub.b = c->block + l * n;
    c->pub.n = n;
    c->pub.l = l;
    c->pub.ntt = (incNTT)ntt;
    return c;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ lwe
void* lwe_alloc_key(uint64_t n, uint64_t l, void* ntt) {
    VC_ENTER_RET("lwe_alloc_key", nullptr);
    (void)vc_where_;
    LweKey* k = new LweKey();
    k->block = (uint64_t*)managed_alloc(sizeof(uint64_t) * ((l * n) != 0 ? l * n : 1));
    k->pub.s = (uint64_t**)malloc(sizeof(uint64_t*) * (l ? l : 1));
    for (uint64_t i = 0; i < l; ++i) k->pub.s[i] = k->block + i * n;
    k->pub.n = n;
    k->pub.l = l;
    k->pub.ntt = (incNTT)ntt;
    // lwe_alloc_key leaves sigma unset in the reference (lwe.c:6-18); start from 0 here.
    k->pub.sigma = 0.0;
    return k;
}

void* lwe_alloc_sample(uint64_t n, uint64_t l, void* ntt) {
    VC_ENTER_RET("lwe_alloc_sample", nullptr);
    (void)vc_where_;
    return new_lwe(n, l, ntt);
}

void free_lwe_sample(void* c) {
    if (!c) return;
    LweSample* s = (LweSample*)c;
    managed_free(s->block);
    free(s->pub.a);
    delete s;
}

void* lwe_new_key(uint64_t n, uint64_t l, void* ntt, double sec_sigma, double err_sigma) {
    VC_ENTER_RET("lwe_new_key", nullptr);
    LweKey* k = (LweKey*)lwe_alloc_key(n, l, ntt);
    if (!k) return nullptr;
    int64_t* d = (int64_t*)device_alloc(n * 8);
    k_gauss_int<<<grid2((long long)n, 1), 256, 0, stream()>>>(d, (long long)n, sec_sigma, prng_key(),
                                                               prng_advance((n + 3) / 4));
    std::vector<int64_t> h(n);
    VC_CHECK(cudaMemcpyAsync(h.data(), d, n * 8, cudaMemcpyDeviceToHost, stream()));
    vc::sync(vc_where_);
    device_free(d);
    IncNtt* t = as_ntt(ntt);
    for (uint64_t j = 0; j < l; ++j)
        for (uint64_t i = 0; i < n; ++i) k->pub.s[j][i] = host_reduce_signed((uint64_t)h[i], t->info[j].q);
    k->pub.sigma = err_sigma;
    return k;
}

void* lwe_new_sparse_ternary_key(uint64_t n, uint64_t l, void* ntt, uint64_t h, double err_sigma) {
    VC_ENTER_RET("lwe_new_sparse_ternary_key", nullptr);
    (void)vc_where_;
    LweKey* k = (LweKey*)lwe_alloc_key(n, l, ntt);
    if (!k) return nullptr;
    IncNtt* t = as_ntt(ntt);
    std::vector<int> v(n, 0);
    // h distinct positions with random signs, drawn on the host from the engine's
    // ChaCha20 stream (8 draws per block; a position is floor(r n / 2^63), r 63 bits)
    const PrngKey key = prng_key();
    const uint64_t nblocks = n + 16;  // 8 (n + 16) draws: far more than h distinct positions need
    const uint64_t ctr = prng_advance(nblocks);
    uint64_t placed = 0, draw = 0;
    uint32_t blk[16];
    while (placed < h && placed < n && draw < 8 * nblocks) {
        if (draw % 8 == 0) chacha20_block(key, ctr + draw / 8, kStreamTernary, blk);
        const uint64_t r = block_u64(blk, (int)(draw % 8));
        ++draw;
        const uint64_t pos = (uint64_t)(((unsigned __int128)(r >> 1) * n) >> 63);
        if (v[pos]) continue;
        v[pos] = (r & 1) ? 1 : -1;
        ++placed;
    }
    for (uint64_t j = 0; j < l; ++j)
        for (uint64_t i = 0; i < n; ++i)
            k->pub.s[j][i] = v[i] == 1 ? 1 : (v[i] == -1 ? t->info[j].q - 1 : 0);
    k->pub.sigma = err_sigma;
    return k;
}

void lwe_sample(void* c, uint64_t* m, void* key) {
    VC_ENTER("lwe_sample");
    LweSample* s = (LweSample*)c;
    LweKey* k = (LweKey*)key;
    if (!s || !k) return;
    IncNtt* t = (IncNtt*)k->pub.ntt;
    const uint64_t n = k->pub.n, l = k->pub.l;
    std::vector<uint64_t*> rows(s->pub.a, s->pub.a + l);
    uint64_t** d_rows = stage_ptrs(rows);
    k_lwe_uniform<<<grid2((long long)n, (int)l), 256, 0, stream()>>>(d_rows, t->d_info, (long long)n,
                                                                      prng_key(), prng_advance((n + 3) / 4 * l));
    // phase of the fresh (a, b = 0) sample gives -<a, s>; b = e + <a, s> + m
    std::vector<uint64_t> zero(l, 0);
    memcpy(s->pub.b, zero.data(), l * 8);
    std::vector<const uint64_t*> srows(k->pub.s, k->pub.s + l);
    const uint64_t** d_s = stage_ptrs(srows);
    uint64_t* d_out = (uint64_t*)managed_alloc(l * 8);
    k_lwe_phase<<<(unsigned)l, 256, 0, stream()>>>(d_out, (const uint64_t* const*)d_rows, s->pub.b, d_s,
                                                   t->d_info, (long long)n);
    int64_t* d_e = (int64_t*)managed_alloc(8);
    k_gauss_int<<<1, 32, 0, stream()>>>(d_e, 1, k->pub.sigma, prng_key(), prng_advance(1));
    vc::sync(vc_where_);
    for (uint64_t i = 0; i < l; ++i) {
        const uint64_t q = t->info[i].q;
        uint64_t b = host_reduce_signed((uint64_t)d_e[0], q);
        b = (b + (q - d_out[i]) % q) % q;  // + <a, s>
        if (m) b = (b + m[i] % q) % q;
        s->pub.b[i] = b;
    }
    managed_free(d_rows);
    managed_free(d_s);
    managed_free(d_out);
    managed_free(d_e);
}

void* lwe_new_sample(uint64_t* m, void* key) {
    VC_ENTER_RET("lwe_new_sample", nullptr);
    (void)vc_where_;
    LweKey* k = (LweKey*)key;
    LweSample* c = new_lwe(k->pub.n, k->pub.l, k->pub.ntt);
    lwe_sample(c, m, key);
    return c;
}

void* lwe_new_trivial_sample(uint64_t* m, uint64_t n, uint64_t l, void* ntt) {
    VC_ENTER_RET("lwe_new_trivial_sample", nullptr);
    (void)vc_where_;
    LweSample* c = new_lwe(n, l, ntt);
    memset(c->block, 0, sizeof(uint64_t) * l * n);
    for (uint64_t i = 0; i < l; ++i) c->pub.b[i] = m ? m[i] : 0;
    return c;
}

void lwe_phase(uint64_t* out, void* c, void* key) {
    VC_ENTER("lwe_phase");
    LweSample* s = (LweSample*)c;
    LweKey* k = (LweKey*)key;
    if (!s || !k || !out) return;
    IncNtt* t = (IncNtt*)k->pub.ntt;
    const uint64_t l = k->pub.l;
    std::vector<const uint64_t*> arows(s->pub.a, s->pub.a + l), srows(k->pub.s, k->pub.s + l);
    const uint64_t** d_a = stage_ptrs(arows);
    const uint64_t** d_s = stage_ptrs(srows);
    uint64_t* d_out = (uint64_t*)managed_alloc(l * 8);
    k_lwe_phase<<<(unsigned)l, 256, 0, stream()>>>(d_out, d_a, s->pub.b, d_s, t->d_info,
                                                   (long long)k->pub.n);
    VC_CHECK(cudaGetLastError());
    vc::sync(vc_where_);
    memcpy(out, d_out, l * 8);
    managed_free((void*)d_a);
    managed_free((void*)d_s);
    managed_free(d_out);
}

void lwe_subto(void* out, void* in) {
    VC_ENTER("lwe_subto");
    LweSample* o = (LweSample*)out;
    LweSample* i = (LweSample*)in;
    if (!o || !i || o->pub.n != i->pub.n || o->pub.l != i->pub.l) {
        set_error(vc_where_, "LWE shapes differ (lwe.c:160-161)");
        return;
    }
    IncNtt* t = (IncNtt*)o->pub.ntt;
    std::vector<uint64_t*> orows(o->pub.a, o->pub.a + o->pub.l);
    std::vector<const uint64_t*> irows(i->pub.a, i->pub.a + i->pub.l);
    uint64_t** d_o = stage_ptrs(orows);
    const uint64_t** d_i = stage_ptrs(irows);
    k_lwe_subto<<<grid2((long long)o->pub.n, (int)o->pub.l), 256, 0, stream()>>>(
        d_o, o->pub.b, d_i, i->pub.b, t->d_info, (long long)o->pub.n);
    VC_CHECK(cudaGetLastError());
    vc::sync(vc_where_);
    managed_free(d_o);
    managed_free((void*)d_i);
}

// ------------------------------------------------------------------ mlwe samples / keys
void* mlwe_alloc_RNS_sample(uint64_t N, uint64_t r, uint64_t mask, void* ntt) {
    VC_ENTER_RET("mlwe_alloc_RNS_sample", nullptr);
    (void)vc_where_;
    return new_mlwe(N, r, mask, as_ntt(ntt));
}

void* mlwe_alloc_RNS_sample_array(uint64_t size, uint64_t N, uint64_t r, uint64_t mask, void* ntt) {
    VC_ENTER_RET("mlwe_alloc_RNS_sample_array", nullptr);
    (void)vc_where_;
    RNS_MLWE* arr = (RNS_MLWE*)malloc(sizeof(RNS_MLWE) * (size ? size : 1));
    for (uint64_t i = 0; i < size; ++i) arr[i] = new_mlwe(N, r, mask, as_ntt(ntt));
    return arr;
}

void mlwe_copy_RNS_sample(void* out, void* in) {
    VC_ENTER("mlwe_copy_RNS_sample");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_copy_RNS_polynomial(o->a[k], i->a[k]);
    polynomial_copy_RNS_polynomial(o->b, i->b);
    VC_FINISH();
}

void* mlwe_create_copy_array(void* in, uint64_t size) {
    VC_ENTER_RET("mlwe_create_copy_array", nullptr);
    RNS_MLWE* src = (RNS_MLWE*)in;
    if (!src || size == 0) return nullptr;
    RNS_MLWE* arr = (RNS_MLWE*)mlwe_alloc_RNS_sample_array(size, src[0]->b->ntt->N, src[0]->r,
                                                           src[0]->b->rns_mask, src[0]->b->ntt);
    for (uint64_t i = 0; i < size; ++i) mlwe_copy_RNS_sample(arr[i], src[i]);
    VC_FINISH();
    return arr;
}

void free_mlwe_RNS_sample(void* p) {
    std::lock_guard<std::recursive_mutex> lk(vc::ctx().mu);
    del_mlwe(as_mlwe(p));
}

void* mlwe_new_RNS_key_from_array(uint64_t* array, uint64_t N, uint64_t r, uint64_t l, void* ntt,
                                  double sigma) {
    VC_ENTER_RET("mlwe_new_RNS_key_from_array", nullptr);
    IncNtt* t = as_ntt(ntt);
    RNS_MLWE_Key key = (RNS_MLWE_Key)calloc(1, sizeof(struct _RNS_MLWE_Key));
    key->N = N;
    key->r = r;
    key->l = l;
    key->sigma = sigma;
    key->s = (IntPolynomial*)calloc(r ? r : 1, sizeof(IntPolynomial));
    key->s_RNS = (RNS_Polynomial*)calloc(r ? r : 1, sizeof(RNS_Polynomial));
    const uint64_t mask = l >= 64 ? ~0ULL : ((1ULL << l) - 1);
    for (uint64_t i = 0; i < r; ++i) {
        IntPoly* ip = (IntPoly*)malloc(sizeof(IntPoly));
        ip->coeffs = (uint64_t*)malloc(N * 8);
        ip->N = N;
        if (array) memcpy(ip->coeffs, array + i * N, N * 8);
        key->s[i] = (IntPolynomial)ip;
        key->s_RNS[i] = (RNS_Polynomial)poly_create(N, mask, t);
        int_array_to_RNS(key->s_RNS[i], ip->coeffs);
    }
    VC_FINISH();
    return key;
}

void* mlwe_new_RNS_gaussian_key(uint64_t N, uint64_t r, uint64_t l, double key_sigma, void* ntt,
                                double sigma) {
    VC_ENTER_RET("mlwe_new_RNS_gaussian_key", nullptr);
    std::vector<uint64_t> arr(N * r);
    int64_t* d = (int64_t*)device_alloc(N * r * 8);
    k_gauss_int<<<grid2((long long)(N * r), 1), 256, 0, stream()>>>(d, (long long)(N * r), key_sigma,
                                                                     prng_key(), prng_advance((N * r + 3) / 4));
    VC_CHECK(cudaMemcpyAsync(arr.data(), d, N * r * 8, cudaMemcpyDeviceToHost, stream()));
    vc::sync(vc_where_);
    device_free(d);
    return mlwe_new_RNS_key_from_array(arr.data(), N, r, l, ntt, sigma);
}

void free_mlwe_RNS_key(void* k) {
    if (!k) return;
    std::lock_guard<std::recursive_mutex> lk(vc::ctx().mu);
    RNS_MLWE_Key key = (RNS_MLWE_Key)k;
    for (uint64_t i = 0; i < key->r; ++i) {
        IntPoly* ip = (IntPoly*)key->s[i];
        if (ip) {
            free(ip->coeffs);
            free(ip);
        }
        poly_destroy((Poly*)key->s_RNS[i]);
    }
    free(key->s);
    free(key->s_RNS);
    free(key);
}

void mlwe_RNSc_to_RNS(void* out, void* in) {
    VC_ENTER("mlwe_RNSc_to_RNS");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    prefetch_mlwe(i);
    prefetch_mlwe(o);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_RNSc_to_RNS(o->a[k], i->a[k]);
    polynomial_RNSc_to_RNS(o->b, i->b);
    VC_FINISH();
}

void mlwe_RNS_to_RNSc(void* out, void* in) {
    VC_ENTER("mlwe_RNS_to_RNSc");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_RNS_to_RNSc(o->a[k], i->a[k]);
    polynomial_RNS_to_RNSc(o->b, i->b);
    VC_FINISH();
}

void mlwe_RNS_trivial_sample_of_zero(void* out) {
    VC_ENTER("mlwe_RNS_trivial_sample_of_zero");
    zero_mlwe(as_mlwe(out), vc_where_);
    VC_FINISH();
}

void* mlwe_new_RNS_trivial_sample_of_zero(uint64_t N, uint64_t r, uint64_t mask, void* ntt) {
    VC_ENTER_RET("mlwe_new_RNS_trivial_sample_of_zero", nullptr);
    RNS_MLWE m = new_mlwe(N, r, mask, as_ntt(ntt));
    zero_mlwe(m, vc_where_);
    VC_FINISH();
    return m;
}

// mlwe_RNS_sample_of_zero (mlwe.c:190-200)
static void sample_of_zero(RNS_MLWE out, RNS_MLWE_Key key) {
    polynomial_gen_gaussian_RNSc_polynomial(out->b, key->sigma);
    polynomial_RNSc_to_RNS(out->b, out->b);
    for (uint64_t i = 0; i < out->r; ++i) {
        polynomial_gen_random_RNSc_polynomial(out->a[i]);
        polynomial_RNSc_to_RNS(out->a[i], out->a[i]);
        op_product(P_(out->b), P_(key->s_RNS[i]), P_(out->a[i]), 1, "mlwe_RNS_sample_of_zero");
    }
}

void mlwe_RNSc_sample(void* out, void* key, void* m) {
    VC_ENTER("mlwe_RNSc_sample");
    RNS_MLWE o = as_mlwe(out);
    sample_of_zero(o, (RNS_MLWE_Key)key);
    mlwe_RNS_to_RNSc(o, o);
    polynomial_add_RNSc_polynomial(o->b, o->b, m);
    VC_FINISH();
}

void* mlwe_new_RNSc_sample_of_zero(void* key) {
    VC_ENTER_RET("mlwe_new_RNSc_sample_of_zero", nullptr);
    RNS_MLWE_Key k = (RNS_MLWE_Key)key;
    // the reference passes key->l as the mask here (mlwe.c:281-286)
    RNS_MLWE m = new_mlwe(k->N, k->r, k->l, (IncNtt*)k->s_RNS[0]->ntt);
    sample_of_zero(m, k);
    mlwe_RNS_to_RNSc(m, m);
    VC_FINISH();
    return m;
}

void* mlwe_new_RNS_sample_of_zero(void* key) {
    VC_ENTER_RET("mlwe_new_RNS_sample_of_zero", nullptr);
    RNS_MLWE_Key k = (RNS_MLWE_Key)key;
    RNS_MLWE m = new_mlwe(k->N, k->r, k->l, (IncNtt*)k->s_RNS[0]->ntt);
    sample_of_zero(m, k);
    VC_FINISH();
    return m;
}

void mlwe_RNS_phase(void* out, void* in, void* key) {
    VC_ENTER("mlwe_RNS_phase");
    RNS_MLWE i = as_mlwe(in);
    RNS_MLWE_Key k = (RNS_MLWE_Key)key;
    Poly* o = as_poly(out);
    op_product(o, P_(i->a[0]), P_(k->s_RNS[0]), 0, vc_where_);
    for (uint64_t j = 1; j < i->r; ++j) op_product(o, P_(i->a[j]), P_(k->s_RNS[j]), 1, vc_where_);
    polynomial_sub_RNS_polynomial(o, i->b, o);
    VC_FINISH();
}

static void mul_by_poly(void* out, void* in, void* poly, int mode, const char* where) {
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    for (uint64_t k = 0; k < o->r; ++k) op_product(P_(o->a[k]), P_(i->a[k]), as_poly(poly), mode, where);
    op_product(P_(o->b), P_(i->b), as_poly(poly), mode, where);
}

void mlwe_RNS_mul_addto_by_poly(void* out, void* in, void* poly) {
    VC_ENTER("mlwe_RNS_mul_addto_by_poly");
    mul_by_poly(out, in, poly, 1, vc_where_);
    VC_FINISH();
}

void mlwe_RNS_mul_subto_by_poly(void* out, void* in, void* poly) {
    VC_ENTER("mlwe_RNS_mul_subto_by_poly");
    mul_by_poly(out, in, poly, 2, vc_where_);
    VC_FINISH();
}

void mlwe_RNS_mul_by_poly(void* out, void* in, void* poly) {
    VC_ENTER("mlwe_RNS_mul_by_poly");
    mul_by_poly(out, in, poly, 0, vc_where_);
    VC_FINISH();
}

void mlwe_scale_RNS_mlwe_RNS(void* c, uint64_t* scale) {
    VC_ENTER("mlwe_scale_RNS_mlwe_RNS");
    RNS_MLWE m = as_mlwe(c);
    for (uint64_t k = 0; k < m->r; ++k) polynomial_scale_RNS_polynomial_RNS(m->a[k], m->a[k], scale);
    polynomial_scale_RNS_polynomial_RNS(m->b, m->b, scale);
    VC_FINISH();
}

void mlwe_add_RNSc_sample(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_add_RNSc_sample");
    RNS_MLWE o = as_mlwe(out), a = as_mlwe(in1), b = as_mlwe(in2);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_add_RNSc_polynomial(o->a[k], a->a[k], b->a[k]);
    polynomial_add_RNSc_polynomial(o->b, a->b, b->b);
    VC_FINISH();
}

void mlwe_sub_RNSc_sample(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_sub_RNSc_sample");
    RNS_MLWE o = as_mlwe(out), a = as_mlwe(in1), b = as_mlwe(in2);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_sub_RNSc_polynomial(o->a[k], a->a[k], b->a[k]);
    polynomial_sub_RNSc_polynomial(o->b, a->b, b->b);
    VC_FINISH();
}

static void xai(Poly* o, Poly* i, uint64_t a, bool minus1, const char* where) {
    IncNtt* t = pool_of(o);
    const uint64_t N = t->pub.N;
    if (o == i || t->pub.split_degree != 1) {
        set_error(where, "needs out != in and split_degree 1 (rns_polynomial.c:1050-1051)");
        return;
    }
    a &= (2 * N - 1);
    o->pub.rns_mask = i->pub.rns_mask;
    if (a == 0) {
        if (minus1) op_zero_rows(o, all_rows(o), where);
        else polynomial_copy_RNS_polynomial(o, i);
        return;
    }
    prefetch_poly(i);
    prefetch_poly(o);
    EwSet s = poly_set(o, i, nullptr, i->pub.rns_mask);
    check_cuda(launch_mul_xai(s, N, a, minus1, t->d_info, stream()), where);
}

void mlwe_RNSc_mul_by_xai(void* out, void* in, uint64_t a) {
    VC_ENTER("mlwe_RNSc_mul_by_xai");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    for (uint64_t k = 0; k < o->r; ++k) xai(P_(o->a[k]), P_(i->a[k]), a, false, vc_where_);
    xai(P_(o->b), P_(i->b), a, false, vc_where_);
    VC_FINISH();
}

void mlwe_RNSc_mul_by_xai_minus1(void* out, void* in, uint64_t a) {
    VC_ENTER("mlwe_RNSc_mul_by_xai_minus1");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    for (uint64_t k = 0; k < o->r; ++k) xai(P_(o->a[k]), P_(i->a[k]), a, true, vc_where_);
    xai(P_(o->b), P_(i->b), a, true, vc_where_);
    VC_FINISH();
}

void mlwe_add_RNSc_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_add_RNSc_polynomial");
    polynomial_add_RNSc_polynomial(as_mlwe(out)->b, as_mlwe(in1)->b, in2);
    VC_FINISH();
}

void mlwe_sub_RNSc_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_sub_RNSc_polynomial");
    polynomial_sub_RNSc_polynomial(as_mlwe(out)->b, as_mlwe(in1)->b, in2);
    VC_FINISH();
}

void mlwe_RNS_add_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_RNS_add_polynomial");
    polynomial_add_RNS_polynomial(as_mlwe(out)->b, as_mlwe(in1)->b, in2);
    VC_FINISH();
}

void mlwe_RNS_sub_polynomial(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_RNS_sub_polynomial");
    polynomial_sub_RNS_polynomial(as_mlwe(out)->b, as_mlwe(in1)->b, in2);
    VC_FINISH();
}

void mlwe_round_division_RNSc(void* out, uint64_t divide_mask) {
    VC_ENTER("mlwe_round_division_RNSc");
    if (divide_mask == 0) return;
    RNS_MLWE o = as_mlwe(out);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_round_division_RNSc_wo_free(o->a[k], divide_mask);
    polynomial_round_division_RNSc_wo_free(o->b, divide_mask);
    VC_FINISH();
}

void* mlwe_extract_LWE(void* in, uint64_t idx) {
    VC_ENTER_RET("mlwe_extract_LWE", nullptr);
    RNS_MLWE i = as_mlwe(in);
    Poly* a0 = P_(i->a[0]);
    IncNtt* t = pool_of(a0);
    const uint64_t N = t->pub.N, r = i->r;
    if (idx >= N) {
        set_error(vc_where_, "coefficient index outside [0, N)");
        return nullptr;
    }
    uint32_t act[64];
    const int l = mask_indices(a0->pub.rns_mask, a0->pub.allocated_l, act);
    LweSample* c = new_lwe(r * N, (uint64_t)l, t);
    prefetch_mlwe(i);
    std::vector<const uint64_t*> comps(r);
    const uint64_t** d_comps = (const uint64_t**)managed_alloc(sizeof(uint64_t*) * (r ? r : 1) * (l ? l : 1));
    for (int j = 0; j < l; ++j) {
        for (uint64_t k = 0; k < r; ++k) d_comps[j * r + k] = i->a[k]->coeffs[act[j]];
    }
    for (int j = 0; j < l; ++j) {
        k_extract_rows<<<grid2((long long)(r * N), 1), 256, 0, stream()>>>(
            c->pub.a[j], d_comps + j * r, (int)r, (long long)N, (long long)idx, t->info[act[j]].q);
        VC_CHECK(cudaGetLastError());
    }
    vc::sync(vc_where_);
    for (int j = 0; j < l; ++j) c->pub.b[j] = i->b->coeffs[act[j]][idx];
    managed_free((void*)d_comps);
    return c;
}

// ------------------------------------------------------------------ key switching
void mlwe_RNSc_GHS_hybrid_keyswitch(void* out, void* in, void* ksk, uint64_t lvl) {
    VC_ENTER("mlwe_RNSc_GHS_hybrid_keyswitch");
    (void)lvl;
    if (out == in) {
        set_error(vc_where_, "out must differ from in (mlwe.c:560)");
        return;
    }
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    RNS_MLWE** K = (RNS_MLWE**)ksk;
    uint64_t c0 = 0;
    while (c0 < i->r && K[c0] == nullptr) ++c0;
    if (c0 == i->r) {
        set_error(vc_where_, "every key-switch component is NULL");
        return;
    }
    const uint64_t extended = K[c0][0]->b->rns_mask;
    const uint64_t divide_mask = extended & ~i->b->rns_mask;
    set_masks(o, extended);
    zero_mlwe(o, vc_where_);
    for (uint64_t k = 0; k < i->r; ++k)
        if (K[k] != nullptr) gadget_mac(o, K[k], P_(i->a[k]), 2, vc_where_);
    mlwe_RNS_to_RNSc(o, o);
    mlwe_round_division_RNSc(o, divide_mask);
    uint64_t keep = 0;
    for (uint64_t k = 0; k < i->r; ++k) {
        if (K[k] == nullptr) {
            polynomial_add_RNSc_polynomial(o->a[keep], o->a[keep], i->a[k]);
            ++keep;
        }
    }
    polynomial_add_RNSc_polynomial(o->b, o->b, i->b);
    VC_FINISH();
}

void mlwe_automorphism_RNSc_GHS(void* out, void* in, uint64_t gen, void* ksk, uint64_t lvl) {
    VC_ENTER("mlwe_automorphism_RNSc_GHS");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    RNS_MLWE tmp = new_mlwe(o->a[0]->ntt->N, o->r, o->a[0]->rns_mask, pool(o));
    for (uint64_t k = 0; k < o->r; ++k) polynomial_RNSc_permute(tmp->a[k], i->a[k], gen);
    polynomial_RNSc_permute(tmp->b, i->b, gen);
    mlwe_RNSc_GHS_hybrid_keyswitch(out, tmp, ksk, lvl);
    del_mlwe(tmp);
    VC_FINISH();
}

void mlwe_partial_trace(void* out, void* in, uint64_t* gens, void* ksks, uint64_t size, uint64_t lvl) {
    VC_ENTER("mlwe_partial_trace");
    RNS_MLWE o = as_mlwe(out);
    RNS_MLWE tmp = new_mlwe(o->a[0]->ntt->N, o->r, o->a[0]->rns_mask, pool(o));
    mlwe_copy_RNS_sample(tmp, in);
    void** K = (void**)ksks;
    for (uint64_t s = 0; s < size; ++s) {
        mlwe_automorphism_RNSc_GHS(out, tmp, gens[s], K[s], lvl);
        mlwe_add_RNSc_sample(tmp, tmp, out);
    }
    mlwe_copy_RNS_sample(out, tmp);
    del_mlwe(tmp);
    VC_FINISH();
}

void mlwe_trace(void* out, void* in, void* ksks, uint64_t lvl) {
    VC_ENTER("mlwe_trace");
    RNS_MLWE i = as_mlwe(in);
    uint64_t N = i->a[0]->ntt->N, logN = 0;
    while ((1ULL << logN) < N) ++logN;
    std::vector<uint64_t> gens(logN);
    for (uint64_t s = 1; s <= logN; ++s) gens[s - 1] = (1ULL << (logN - s + 1)) + 1;
    mlwe_partial_trace(out, in, gens.data(), ksks, logN, lvl);
    VC_FINISH();
}

uint64_t mlwe_extended_rank(uint64_t r) { return r * (r + 3) / 2; }

static void tensor(RNS_Polynomial* out, RNS_MLWE a, RNS_MLWE b, const char* where) {
    const uint64_t r = a->r;
    const uint64_t R = mlwe_extended_rank(r);
    uint64_t k = 0;
    for (uint64_t i = 0; i < r; ++i) {
        for (uint64_t j = i; j < r; ++j) {
            op_product(P_(out[k]), P_(a->a[i]), P_(b->a[j]), 0, where);
            if (i != j) op_product(P_(out[k]), P_(a->a[j]), P_(b->a[i]), 1, where);
            ++k;
        }
    }
    for (uint64_t i = 0; i < r; ++i) {
        op_product(P_(out[k]), P_(a->a[i]), P_(b->b), 0, where);
        op_product(P_(out[k]), P_(a->b), P_(b->a[i]), 1, where);
        ++k;
    }
    op_product(P_(out[R]), P_(a->b), P_(b->b), 0, where);
}

void mlwe_tensor_product(void* out, void* in1, void* in2) {
    VC_ENTER("mlwe_tensor_product");
    RNS_MLWE a = as_mlwe(in1), b = as_mlwe(in2);
    if (a->r != b->r) {
        set_error(vc_where_, "ranks differ (mlwe.c:680)");
        return;
    }
    tensor((RNS_Polynomial*)out, a, b, vc_where_);
    VC_FINISH();
}

void mlwe_multiply(void* out, void* in1, void* in2, void* ksk) {
    VC_ENTER("mlwe_multiply");
    RNS_MLWE o = as_mlwe(out), a = as_mlwe(in1), b = as_mlwe(in2);
    const uint64_t r = a->r, R = mlwe_extended_rank(r);
    const uint64_t N = a->b->ntt->N, mask = a->b->rns_mask;
    IncNtt* t = pool(a);
    if (ksk == nullptr) {
        if (o->r != R) {
            set_error(vc_where_, "output rank must be the extended rank without a key (mlwe.c:725)");
            return;
        }
        std::vector<RNS_Polynomial> tp(R + 1);
        for (uint64_t j = 0; j < R; ++j) tp[j] = o->a[j];
        tp[R] = o->b;
        tensor(tp.data(), a, b, vc_where_);
        VC_FINISH();
        return;
    }
    if (o->r != r) {
        set_error(vc_where_, "output rank must equal the input rank (mlwe.c:741)");
        return;
    }
    RNS_MLWE ext = new_mlwe(N, R, mask, t);
    std::vector<RNS_Polynomial> tp(R + 1);
    for (uint64_t j = 0; j < R; ++j) tp[j] = ext->a[j];
    tp[R] = ext->b;
    tensor(tp.data(), a, b, vc_where_);
    RNS_MLWE ext_c = new_mlwe(N, R, mask, t);
    mlwe_RNS_to_RNSc(ext_c, ext);
    mlwe_RNSc_GHS_hybrid_keyswitch(o, ext_c, ksk, 0);
    mlwe_RNSc_to_RNS(o, o);
    del_mlwe(ext);
    del_mlwe(ext_c);
    VC_FINISH();
}

// ------------------------------------------------------------------ mgsw
void mgsw_external_product(void* out, void* mgsw, void* in, uint64_t ell, uint64_t special_primes) {
    VC_ENTER("mgsw_external_product");
    RNS_MLWE o = as_mlwe(out), i = as_mlwe(in);
    RNS_MLWE* G = (RNS_MLWE*)mgsw;
    const uint64_t r = i->r;
    const uint64_t extended = G[0]->b->rns_mask;
    set_masks(o, extended);
    zero_mlwe(o, vc_where_);
    for (uint64_t j = 0; j < r; ++j) gadget_mac(o, &G[j * ell], P_(i->a[j]), 1, vc_where_);
    gadget_mac(o, &G[r * ell], P_(i->b), 1, vc_where_);
    if (special_primes > 0) {
        mlwe_RNS_to_RNSc(o, o);
        uint64_t divide_mask = 0, count = 0;
        const uint64_t m = o->b->rns_mask;
        for (int idx = 63; idx >= 0 && count < special_primes; --idx) {
            if (m & (1ULL << idx)) {
                divide_mask |= (1ULL << idx);
                ++count;
            }
        }
        if (divide_mask) mlwe_round_division_RNSc(o, divide_mask);
        mlwe_RNSc_to_RNS(o, o);
    }
    VC_FINISH();
}

void mgsw_CMUX(void* out, void* in1, void* in2, void* mgsw, uint64_t ell, uint64_t special_primes) {
    VC_ENTER("mgsw_CMUX");
    RNS_MLWE a = as_mlwe(in1);
    const uint64_t N = a->b->ntt->N, r = a->r, mask = a->b->rns_mask;
    IncNtt* t = pool(a);
    RNS_MLWE diff = new_mlwe(N, r, mask, t);
    mlwe_sub_RNSc_sample(diff, in2, in1);
    mgsw_external_product(out, mgsw, diff, ell, special_primes);
    RNS_MLWE a_ntt = new_mlwe(N, r, mask, t);
    mlwe_copy_RNS_sample(a_ntt, in1);
    mlwe_RNSc_to_RNS(a_ntt, a_ntt);
    RNS_MLWE o = as_mlwe(out);
    for (uint64_t k = 0; k < o->r; ++k) polynomial_add_RNS_polynomial(o->a[k], o->a[k], a_ntt->a[k]);
    polynomial_add_RNS_polynomial(o->b, o->b, a_ntt->b);
    del_mlwe(diff);
    del_mlwe(a_ntt);
    VC_FINISH();
}

void mgsw_NCMUX(void* out, void* in1, void* in2, void* mgsw, void* ksk, uint64_t ell, uint64_t special_primes) {
    VC_ENTER("mgsw_NCMUX");
    RNS_MLWE a = as_mlwe(in1);
    const uint64_t N = a->b->ntt->N, r = a->r, mask = a->b->rns_mask;
    RNS_MLWE tmp = new_mlwe(N, r, mask, pool(a));
    mlwe_automorphism_RNSc_GHS(tmp, in2, 2 * N - 1, ksk, ell);
    mgsw_CMUX(out, in1, tmp, mgsw, ell, special_primes);
    del_mlwe(tmp);
    VC_FINISH();
}

// ------------------------------------------------------------------ packing (composite)
// pool indices of the extended limbs, passed by value to the digit kernel
struct PackPrimes {
    uint32_t p[kMaxLimbs];
};

// The packing key switch's digits for digits d0 .. d0 + nd - 1, d = i lwe_l + l: row e of
// digit d is the polynomial whose coefficient k < size is sample k's mask entry i of
// limb l (M [in_n][lwe_l][size]) reduced modulo extended prime e, zero above `size`
// (polynomial_RNSc_mod_reduce_lifted of the reference's tmp polynomial).
__global__ void k_pack_digits(uint64_t* __restrict__ D, const uint64_t* __restrict__ M, long long d0, int nd,
                              int lwe_l, int size, int ne, const __grid_constant__ PackPrimes lp,
                              const PrimeInfo* __restrict__ primes, long long N) {
    const int de = blockIdx.y;  // (digit, extended limb)
    const int dd = de / ne, e = de - dd * ne;
    const long long d = d0 + dd;
    const PrimeInfo& pi = primes[lp.p[e]];
    const uint64_t* src = M + d * size;  // [i][l] rows of `size` entries, d = i lwe_l + l
    uint64_t* row = D + ((long long)dd * ne + e) * N;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N; x += (long long)gridDim.x * blockDim.x)
        row[x] = x < size ? reduce64(src[x], pi) : 0;
    (void)lwe_l;
    (void)nd;
}

// Copy rows through a pointer table: rows[r] (N residues) -> dst + r N.
__global__ void k_gather_rows(uint64_t* __restrict__ dst, const uint64_t* const* __restrict__ rows, long long N) {
    const uint64_t* src = rows[blockIdx.y];
    uint64_t* o = dst + (long long)blockIdx.y * N;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N; x += (long long)gridDim.x * blockDim.x)
        o[x] = src[x];
}

// mlwe_full_packing_keyswitch's inner product over every (mask entry i, limb l) digit
// at once: the mask entries are gathered on the host in one pass, the digit rows built,
// transformed and multiplied into the key on the GPU in a few launches per chunk of
// digits, instead of a host write of the digit polynomial and a synchronisation per
// mask entry.  Digits of the target's limbs past the samples' lwe_l are zero and are
// skipped (they add nothing).  Exact modular arithmetic throughout, so the result is
// the sequential form's.  Writes -sum into out's a[0] and b rows of the extended limbs
// and returns true; false (nothing written) where it does not apply: rank other than
// 1, more than 64 extended limbs, or a failed allocation.
static bool packing_inner_product_batched(RNS_MLWE o, LWE* lw, RNS_MLWE** K, uint64_t size, uint64_t in_n,
                                          uint64_t lwe_l, uint64_t extended, const char* where) {
    // VFHE_CUDA_PACKING_SEQUENTIAL=1: the sequential form below (same residues; tests compare)
    const char* seq = getenv("VFHE_CUDA_PACKING_SEQUENTIAL");
    if (seq && atoi(seq) != 0) return false;
    if (o->r != 1 || K[0][0]->r != 1) return false;
    IncNtt* t = pool(o);
    const uint64_t N = o->b->ntt->N;
    std::vector<uint32_t> ext;
    for (uint32_t j = 0; j < 64; ++j)
        if ((extended >> j) & 1) ext.push_back(j);
    const int ne = (int)ext.size();
    if (ne == 0 || ne > kMaxLimbs || size > N || in_n == 0 || lwe_l == 0) return false;
    // the samples' mask entries, M[i][l][k] = sample k's entry i of limb l
    std::vector<uint64_t> M(in_n * lwe_l * size);
    for (uint64_t k = 0; k < size; ++k)
        for (uint64_t l = 0; l < lwe_l; ++l)
            for (uint64_t i = 0; i < in_n; ++i) M[(i * lwe_l + l) * size + k] = lw[k]->a[l][i];
    const uint64_t ndig = in_n * lwe_l;
    // digits per chunk: D and the gathered keys within ~256 MB
    const uint64_t per_digit = 3ULL * ne * N * sizeof(uint64_t);
    uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(ndig, (256ULL << 20) / per_digit));
    chunk = std::min<uint64_t>(chunk, 65535 / (2 * (uint64_t)ne));  // the gather grid's y dimension
    uint64_t *dM = nullptr, *dD = nullptr, *dK = nullptr, *dacc = nullptr, *dtmp = nullptr, *dptr = nullptr;
    const uint64_t** drows = nullptr;
    auto release = [&]() {
        cudaFree(dM);
        cudaFree(dD);
        cudaFree(dK);
        cudaFree(dacc);
        cudaFree(dtmp);
        cudaFree(dptr);
        cudaFree(drows);
    };
    if (cudaMalloc(&dM, M.size() * 8) != cudaSuccess || cudaMalloc(&dD, chunk * ne * N * 8) != cudaSuccess ||
        cudaMalloc(&dK, chunk * 2 * ne * N * 8) != cudaSuccess || cudaMalloc(&dacc, 2 * ne * N * 8) != cudaSuccess ||
        cudaMalloc(&dtmp, 2 * ne * N * 8) != cudaSuccess || cudaMalloc(&dptr, 8) != cudaSuccess ||
        cudaMalloc(&drows, chunk * 2 * ne * sizeof(uint64_t*)) != cudaSuccess) {
        cudaGetLastError();
        release();
        return false;
    }
    cudaStream_t st = stream();
    // on the engine stream, so that the digit kernels below are ordered after it
    bool ok = check_cuda(cudaMemcpyAsync(dM, M.data(), M.size() * 8, cudaMemcpyHostToDevice, st), where);
    PackPrimes lp;
    memset(&lp, 0, sizeof lp);
    for (int e = 0; e < ne; ++e) lp.p[e] = ext[e];
    std::vector<const uint64_t*> rows(chunk * 2 * ne);
    for (uint64_t d0 = 0; ok && d0 < ndig; d0 += chunk) {
        const int nd = (int)std::min(chunk, ndig - d0);
        // keys of these digits, [dd][component][e][N]
        for (int dd = 0; dd < nd; ++dd) {
            const uint64_t d = d0 + dd, i = d / lwe_l, l = d % lwe_l;
            RNS_MLWE k = K[i][l];
            for (int e = 0; e < ne; ++e) {
                rows[((size_t)dd * 2 + 0) * ne + e] = k->a[0]->coeffs[ext[e]];
                rows[((size_t)dd * 2 + 1) * ne + e] = k->b->coeffs[ext[e]];
            }
        }
        ok = check_cuda(cudaMemcpyAsync(drows, rows.data(), (size_t)nd * 2 * ne * sizeof(uint64_t*),
                                        cudaMemcpyHostToDevice, st), where);
        if (!ok) break;
        const unsigned gx = (unsigned)std::min<uint64_t>(64, (N + 255) / 256);
        k_gather_rows<<<dim3(gx, (unsigned)(nd * 2 * ne)), 256, 0, st>>>(dK, drows, (long long)N);
        k_pack_digits<<<dim3(gx, (unsigned)(nd * ne)), 256, 0, st>>>(dD, dM, (long long)d0, nd, (int)lwe_l, (int)size,
                                                                     ne, lp, t->d_info, (long long)N);
        ok = check_cuda(cudaGetLastError(), where);
        if (!ok) break;
        RowSet rs;
        memset(&rs, 0, sizeof rs);
        for (int e = 0; e < ne; ++e) {
            rs.in[e] = dD + (size_t)e * N;
            rs.out[e] = dD + (size_t)e * N;
            rs.prime[e] = ext[e];
        }
        rs.nlimbs = ne;
        rs.split = (int)t->pub.split_degree;
        rs.logP = t->logP;
        rs.batch = nd;
        rs.batch_stride = (long long)ne * N;
        rs.in_batch_stride = rs.batch_stride;
        mark_fp64(rs, t);
        ok = check_cuda(launch_ntt(rs, t->d_info, false, st), where) &&
             check_cuda(mac_one_sample(t, d0 ? dtmp : dacc, dD, dK, dptr, ext.data(), nd, ne, st), where);
        if (ok && d0) {
            // acc += tmp, row by row (both components)
            EwSet es = empty_set((long long)N);
            for (int c = 0; c < 2 && ok; ++c) {
                for (int e = 0; e < ne; ++e) {
                    es.out[e] = dacc + ((size_t)c * ne + e) * N;
                    es.a[e] = dacc + ((size_t)c * ne + e) * N;
                    es.b[e] = dtmp + ((size_t)c * ne + e) * N;
                    es.prime[e] = ext[e];
                }
                es.nlimbs = ne;
                ok = check_cuda(launch_ew(EW_ADD, es, t->d_info, st), where);
            }
        }
        // the host rewrites `rows` for the next chunk only after this chunk's copy of it
        if (ok && d0 + chunk < ndig) ok = check_cuda(cudaStreamSynchronize(st), where);
    }
    if (ok) {
        for (int e = 0; e < ne && ok; ++e) {
            ok = check_cuda(cudaMemcpyAsync(o->a[0]->coeffs[ext[e]], dacc + (size_t)e * N, N * 8,
                                            cudaMemcpyDeviceToDevice, st), where) &&
                 check_cuda(cudaMemcpyAsync(o->b->coeffs[ext[e]], dacc + ((size_t)ne + e) * N, N * 8,
                                            cudaMemcpyDeviceToDevice, st), where);
        }
    }
    check_cuda(cudaStreamSynchronize(st), where);
    release();
    return ok;
}

// Packing of `size` LWE samples into one MLWE (mlwe_full_packing_keyswitch, mlwe.c:343-430):
// out = sum over mask coefficients i of -(the polynomial of the samples' i-th mask
// entries, one coefficient per sample) lifted per limb and times ksk[i][limb], computed
// over the extended limbs of the key, then divided down to the output's limbs, plus
// the polynomial of the bodies.  The same sequence of engine operations as the
// reference, each on the GPU.
void mlwe_full_packing_keyswitch(void* out, void* in, uint64_t size, void* ksk, uint64_t lvl) {
    VC_ENTER("mlwe_full_packing_keyswitch");
    (void)lvl;
    RNS_MLWE o = as_mlwe(out);
    LWE* lw = (LWE*)in;
    RNS_MLWE** K = (RNS_MLWE**)ksk;
    if (!o || !lw || !K || size == 0 || !lw[0]) {
        set_error(vc_where_, "null output, samples or keys, or no samples");
        return;
    }
    const uint64_t N = o->b->ntt->N, in_n = lw[0]->n, lwe_l = lw[0]->l;
    if (size > N) {
        set_error(vc_where_, "more samples than ring coefficients");
        return;
    }
    const uint64_t target = o->b->rns_mask, extended = K[0][0]->b->rns_mask;
    const uint64_t divide = extended & ~target;
    // pool index of the limb-th active limb of the target mask
    std::vector<uint64_t> active;
    for (uint64_t j = 0; j < 64; ++j)
        if ((target >> j) & 1) active.push_back(j);
    if (active.size() < lwe_l) {
        set_error(vc_where_, "the output has fewer limbs than the samples");
        return;
    }
    for (uint64_t k = 0; k < o->r; ++k) o->a[k]->rns_mask = extended;
    o->b->rns_mask = extended;
    mlwe_RNS_trivial_sample_of_zero(out);
    IncNtt* t = pool(o);
    void* tmp = polynomial_new_RNS_polynomial(N, target, t);
    void* tmp_red = polynomial_new_RNS_polynomial(N, extended, t);
    void* tmp_rns = polynomial_new_RNS_polynomial(N, extended, t);
    RNS_Polynomial tp = (RNS_Polynomial)tmp;
    const bool batched = packing_inner_product_batched(o, lw, K, size, in_n, lwe_l, extended, vc_where_);
    for (uint64_t i = 0; i < in_n && !batched; ++i) {
        vc::sync(vc_where_);  // the rows are written from the host below
        for (uint64_t j : active) memset(tp->coeffs[j], 0, N * sizeof(uint64_t));
        for (uint64_t limb = 0; limb < lwe_l; ++limb)
            for (uint64_t k = 0; k < size; ++k) tp->coeffs[active[limb]][k] = lw[k]->a[limb][i];
        uint64_t idx = 0;
        for (uint64_t j : active) {
            polynomial_RNSc_mod_reduce_lifted(tmp_red, tmp, j);
            polynomial_RNSc_to_RNS(tmp_rns, tmp_red);
            mlwe_RNS_mul_subto_by_poly(out, K[i][idx++], tmp_rns);
        }
    }
    vc::sync(vc_where_);
    for (uint64_t j : active) memset(tp->coeffs[j], 0, N * sizeof(uint64_t));
    for (uint64_t limb = 0; limb < lwe_l; ++limb)
        for (uint64_t k = 0; k < size; ++k) tp->coeffs[active[limb]][k] = lw[k]->b[limb];
    mlwe_RNS_to_RNSc(out, out);
    if (divide) {
        for (uint64_t j = 0; j < o->r; ++j) polynomial_round_division_RNSc_wo_free(o->a[j], divide);
        polynomial_round_division_RNSc_wo_free(o->b, divide);
    }
    polynomial_add_RNSc_polynomial(o->b, o->b, tmp);
    mlwe_RNSc_to_RNS(out, out);
    free_RNS_polynomial(tmp);
    free_RNS_polynomial(tmp_red);
    free_RNS_polynomial(tmp_rns);
    VC_FINISH();
}

static void packing_rec(RNS_MLWE* vec, uint64_t ell, RNS_MLWE*** ksks, uint64_t lvl) {
    if (ell == 0) return;
    const uint64_t half = 1ULL << (ell - 1);
    std::vector<RNS_MLWE> even(half), odd(half);
    for (uint64_t i = 0; i < half; ++i) {
        even[i] = vec[2 * i];
        odd[i] = vec[2 * i + 1];
    }
    packing_rec(even.data(), ell - 1, ksks, lvl);
    packing_rec(odd.data(), ell - 1, ksks, lvl);
    RNS_MLWE C = even[0];
    const uint64_t N = vec[0]->b->ntt->N, r = vec[0]->r;
    IncNtt* t = pool(vec[0]);
    RNS_MLWE tmp = new_mlwe(N, r, vec[0]->b->rns_mask, t);
    const uint64_t extended = ksks[ell - 1][0][0]->b->rns_mask;
    RNS_MLWE tmp2 = new_mlwe(N, r, extended, t);
    mlwe_RNSc_mul_by_xai(tmp, odd[0], N >> ell);
    mlwe_sub_RNSc_sample(C, even[0], tmp);
    mlwe_automorphism_RNSc_GHS(tmp2, C, (1ULL << ell) + 1, ksks[ell - 1], lvl);
    for (uint64_t k = 0; k < tmp->r; ++k) polynomial_scale_RNSc_polynomial(tmp->a[k], tmp->a[k], 2);
    polynomial_scale_RNSc_polynomial(tmp->b, tmp->b, 2);
    mlwe_add_RNSc_sample(C, C, tmp2);
    mlwe_add_RNSc_sample(C, C, tmp);
    del_mlwe(tmp);
    del_mlwe(tmp2);
}

void mlwe_full_packing_keyswitch_scaled(void* vec, uint64_t ell, void* ksks, uint64_t lvl) {
    VC_ENTER("mlwe_full_packing_keyswitch_scaled");
    packing_rec((RNS_MLWE*)vec, ell, (RNS_MLWE***)ksks, lvl);
    VC_FINISH();
}

// ------------------------------------------------------------------ GP25 (composite)
// GP25's sparse-amortised bootstrap steps (modules/fhe/c/src/gp25.c:68-336) as the same
// sequence of engine operations, each on the GPU.  The reference's thread count is
// a CPU work split and does not change results; the _mt entry points take it and run
// the single sequence.

// out = ExtProd(mgsw, in2 - in1) to the coefficient domain, + in1 (mgsw_CMUX_to_coeff,
// modules/mlwe/c/src/mgsw.c:103-119: equal to CMUX followed by an inverse transform).
static void cmux_to_coeff(void* out, void* in1, void* in2, void* mgsw, uint64_t ell, uint64_t sp) {
    RNS_MLWE a = as_mlwe(in1);
    RNS_MLWE diff = new_mlwe(a->b->ntt->N, a->r, a->b->rns_mask, pool(a));
    mlwe_sub_RNSc_sample(diff, in2, in1);
    mgsw_external_product(out, mgsw, diff, ell, sp);
    mlwe_RNS_to_RNSc(out, out);
    mlwe_add_RNSc_sample(out, out, in1);
    del_mlwe(diff);
}

// CMUX with in2 first mapped by X -> X^(2N-1) (mgsw_NCMUX_to_coeff, mgsw.c:121-136).
static void ncmux_to_coeff(void* out, void* in1, void* in2, void* mgsw, void* ksk, uint64_t ell, uint64_t sp) {
    RNS_MLWE a = as_mlwe(in1);
    const uint64_t N = a->b->ntt->N;
    RNS_MLWE tmp = new_mlwe(N, a->r, a->b->rns_mask, pool(a));
    mlwe_automorphism_RNSc_GHS(tmp, in2, 2 * N - 1, ksk, ell);
    cmux_to_coeff(out, in1, tmp, mgsw, ell, sp);
    del_mlwe(tmp);
}

// gp25_RGSW_monomial_mul (gp25.c:68-128): r_prec rounds of (N)CMUXes over the in_N
// accumulators, ping-ponging between p0 and a scratch array.
void gp25_RGSW_monomial_mul(void* p0v, uint64_t in_N, void* ev, uint64_t r_prec, void* ksk, uint64_t ell,
                            uint64_t special_primes) {
    VC_ENTER("gp25_RGSW_monomial_mul");
    RNS_MLWE* p0 = (RNS_MLWE*)p0v;
    RNS_MLWE* e = (RNS_MLWE*)ev;
    if (!p0 || !e || in_N == 0) {
        set_error(vc_where_, "null accumulators or keys");
        return;
    }
    const uint64_t N = p0[0]->b->ntt->N, r = p0[0]->r, mask = p0[0]->b->rns_mask;
    std::vector<RNS_MLWE> p1(in_N);
    for (uint64_t i = 0; i < in_N; ++i) p1[i] = new_mlwe(N, r, mask, pool(p0[0]));
    RNS_MLWE* p[2] = {p0, p1.data()};
    for (uint64_t i = 0; i < r_prec; ++i) {
        const uint64_t power = 1ULL << i;
        const uint64_t out_idx = (i + 1) & 1, in_idx = out_idx ^ 1;
        const void* ei = ((void* const*)e)[i];
        for (uint64_t j = 0; j < power; ++j)
            ncmux_to_coeff(p[out_idx][j], p[in_idx][j], p[in_idx][in_N - power + j], (void*)ei, ksk, ell,
                           special_primes);
        for (uint64_t j = 0; j + power < in_N; ++j)
            cmux_to_coeff(p[out_idx][j + power], p[in_idx][j + power], p[in_idx][j], (void*)ei, ell,
                          special_primes);
    }
    if (r_prec & 1)
        for (uint64_t i = 0; i < in_N; ++i) mlwe_copy_RNS_sample(p0[i], p1[i]);
    for (uint64_t i = 0; i < in_N; ++i) del_mlwe(p1[i]);
    VC_FINISH();
}

void gp25_RGSW_monomial_mul_mt(void* p0, uint64_t in_N, void* e, uint64_t r_prec, void* ksk, uint64_t ell,
                               uint64_t special_primes, uint64_t num_threads) {
    (void)num_threads;
    gp25_RGSW_monomial_mul(p0, in_N, e, r_prec, ksk, ell, special_primes);
}

// gp25_sub_a_mt (gp25.c:278-336): p[k] <- p[k] X^a_k + s_sign (x) (p[k] X^a_k (X^(-2 a_k) - 1)).
void gp25_sub_a_mt(void* p0v, uint64_t in_N, uint64_t* a, void* s_sign, uint64_t ell, uint64_t special_primes,
                   uint64_t N, uint64_t num_threads) {
    VC_ENTER("gp25_sub_a_mt");
    (void)num_threads;
    RNS_MLWE* p0 = (RNS_MLWE*)p0v;
    if (!p0 || !a || !s_sign || in_N == 0) {
        set_error(vc_where_, "null accumulators, rotations or key");
        return;
    }
    const uint64_t twoN = 2 * N, r = p0[0]->r, mask = p0[0]->b->rns_mask;
    IncNtt* t = pool(p0[0]);
    RNS_MLWE pax = new_mlwe(N, r, mask, t), tmp = new_mlwe(N, r, mask, t);
    RNS_MLWE ext = new_mlwe(N, r, mask, t), pax_ntt = new_mlwe(N, r, mask, t);
    for (uint64_t k = 0; k < in_N; ++k) {
        mlwe_RNSc_mul_by_xai(pax, p0[k], a[k]);
        const uint64_t m2a = (twoN - (2 * a[k]) % twoN) % twoN;
        mlwe_RNSc_mul_by_xai_minus1(tmp, pax, m2a);
        mgsw_external_product(ext, s_sign, tmp, ell, special_primes);
        mlwe_copy_RNS_sample(pax_ntt, pax);
        mlwe_RNSc_to_RNS(pax_ntt, pax_ntt);
        for (uint64_t i = 0; i < r; ++i) polynomial_add_RNS_polynomial(ext->a[i], ext->a[i], pax_ntt->a[i]);
        polynomial_add_RNS_polynomial(ext->b, ext->b, pax_ntt->b);
        mlwe_RNS_to_RNSc(p0[k], ext);
    }
    del_mlwe(pax);
    del_mlwe(tmp);
    del_mlwe(ext);
    del_mlwe(pax_ntt);
    VC_FINISH();
}

}  // extern "C"
