// Device context, error recording, memory caches, PRNG state and transform tables.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <atomic>
#include <map>
#include <string>

#include "engine.cuh"

namespace vc {

// ---------------------------------------------------------------- context / errors
Context& ctx() {
    static Context c;
    return c;
}

namespace {
std::mutex g_err_mu;
int g_status = 0;
char g_error[512];  // fixed buffer: recording an error never allocates
}  // namespace

void set_error(const char* where, const char* what) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (g_status == 0) {
        g_status = 1;
        snprintf(g_error, sizeof g_error, "%s: %s", where, what);
        if (getenv("VFHE_CUDA_QUIET") == nullptr) fprintf(stderr, "vfhe cuda engine: %s\n", g_error);
    }
}

bool check_cuda(int code, const char* where) {
    if (code == cudaSuccess) return true;
    set_error(where, cudaGetErrorString((cudaError_t)code));
    return false;
}

int sm_count() {
    const int n = ctx().sms;
    return n > 0 ? n : 148;
}

bool ensure_ready() {
    Context& c = ctx();
    if (c.ready) return true;
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    if (c.ready) return true;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_error("init", "no CUDA device is available (the cuda engine has no CPU fallback)");
        return false;
    }
    int dev = 0;
    if (const char* s = getenv("VFHE_CUDA_DEVICE")) dev = atoi(s);
    if (!check_cuda(cudaSetDevice(dev), "init: cudaSetDevice")) return false;
    if (!check_cuda(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "init: stream"))
        return false;
    c.device = dev;
    if (cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c.sms <= 0) c.sms = 148;
    c.ready = true;
    return true;
}

cudaStream_t stream() { return ctx().stream; }

bool sync(const char* where) {
    cudaError_t e = cudaStreamSynchronize(ctx().stream);
    if (e != cudaSuccess) return check_cuda(e, where);
    return true;
}

// ---------------------------------------------------------------- memory caches
namespace {
struct Cache {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;
    std::map<void*, size_t> sizes;
};
Cache& managed_cache() {
    static Cache c;
    return c;
}
Cache& device_cache() {
    static Cache c;
    return c;
}
size_t round_bytes(size_t b) {
    if (b < 4096) return 4096;
    // round to 1/8 of the next power of two to bound waste and keep reuse high
    size_t p = 1;
    while (p < b) p <<= 1;
    size_t step = p >> 3;
    return (b + step - 1) / step * step;
}
void* cache_alloc(Cache& c, size_t bytes, bool managed) {
    size_t rb = round_bytes(bytes);
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.free_blocks.find(rb);
        if (it != c.free_blocks.end()) {
            void* p = it->second;
            c.free_blocks.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = managed ? cudaMallocManaged(&p, rb, cudaMemAttachGlobal) : cudaMalloc(&p, rb);
    if (e != cudaSuccess) {
        check_cuda(e, managed ? "cudaMallocManaged" : "cudaMalloc");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(c.mu);
    c.sizes[p] = rb;
    return p;
}
void cache_free(Cache& c, void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.sizes.find(p);
    if (it == c.sizes.end()) return;
    c.free_blocks.emplace(it->second, p);
}
}  // namespace

void* managed_alloc(size_t bytes) {
    if (!ensure_ready()) return nullptr;
    return cache_alloc(managed_cache(), bytes, true);
}
void managed_free(void* p) { cache_free(managed_cache(), p); }
void* device_alloc(size_t bytes) {
    if (!ensure_ready()) return nullptr;
    return cache_alloc(device_cache(), bytes, false);
}
void device_free(void* p) { cache_free(device_cache(), p); }

// A prefetch costs a fixed 70-85 us of driver time on B200 even when the pages already
// sit on the device, and saves 50-70 us against the kernel's own page faults for a
// host-written block of up to 1 MB, 175 us at 4 MB, 1.1 ms at 16 MB.  Blocks below
// VFHE_CUDA_PREFETCH_MIN_BYTES (default 2 MiB) are therefore left to the faults: most
// of them are intermediates that never leave the device.  VFHE_CUDA_PREFETCH=0 turns
// every prefetch off.
void prefetch_to_device(const void* p, size_t bytes) {
    if (!p || bytes == 0) return;
    struct Policy {
        bool enabled;
        size_t min_bytes;
    };
    static const Policy policy = [] {  // read once; a function-local static initialises thread-safely
        const char* s = getenv("VFHE_CUDA_PREFETCH");
        const char* m = getenv("VFHE_CUDA_PREFETCH_MIN_BYTES");
        return Policy{s == nullptr || atoi(s) != 0, m ? (size_t)strtoull(m, nullptr, 10) : ((size_t)2 << 20)};
    }();
    if (!policy.enabled || bytes < policy.min_bytes) return;
    cudaMemPrefetchAsync(p, bytes, ctx().device, ctx().stream);
    cudaGetLastError();  // a refused prefetch only costs speed
}

// ---------------------------------------------------------------- PRNG state
namespace {
PrngKey g_key;
uint64_t g_counter = 0;
bool g_seeded = false;
std::mutex g_prng_mu;

uint64_t splitmix_next(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

PrngKey expand_seed(uint64_t seed) {
    PrngKey k;
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
        const uint64_t v = splitmix_next(x);
        k.w[2 * i] = (uint32_t)v;
        k.w[2 * i + 1] = (uint32_t)(v >> 32);
    }
    return k;
}

// 256 bits from the operating system's entropy source; without one the key still
// differs per process (address, time) and the engine records an error.
PrngKey entropy_key() {
    PrngKey k;
    memset(&k, 0, sizeof k);
    FILE* f = fopen("/dev/urandom", "rb");
    bool ok = false;
    if (f) {
        ok = fread(k.w, sizeof k.w, 1, f) == 1;
        fclose(f);
    }
    if (!ok) {
        set_error("prng", "/dev/urandom unavailable: key from process address and time only");
        k = expand_seed((uint64_t)(uintptr_t)&k ^ (uint64_t)time(nullptr));
    }
    return k;
}
}  // namespace

PrngKey prng_key() {
    std::lock_guard<std::mutex> lk(g_prng_mu);
    if (!g_seeded) {
        g_key = entropy_key();
        g_counter = 0;
        g_seeded = true;
    }
    return g_key;
}
uint64_t prng_advance(uint64_t blocks) {
    prng_key();
    std::lock_guard<std::mutex> lk(g_prng_mu);
    const uint64_t c = g_counter;
    g_counter += blocks;
    return c;
}
// Deterministic mode (tests): the 64-bit seed expanded to a key by splitmix64.
void prng_set(uint64_t seed, bool det) {
    const PrngKey k = det ? expand_seed(seed) : entropy_key();
    std::lock_guard<std::mutex> lk(g_prng_mu);
    g_key = k;
    g_counter = 0;
    g_seeded = true;
}

// ---------------------------------------------------------------- number theory
uint64_t host_mul_mod(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((unsigned __int128)a * b) % q);
}
uint64_t host_pow_mod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = host_mul_mod(r, b, q);
        b = host_mul_mod(b, b, q);
        e >>= 1;
    }
    return r;
}
uint64_t host_inv_mod(uint64_t a, uint64_t q) {
    // extended Euclid on signed 128-bit to stay exact for q < 2^63
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr != 0) {
        __int128 quo = r / nr;
        __int128 tmp = t - quo * nt;
        t = nt;
        nt = tmp;
        tmp = r - quo * nr;
        r = nr;
        nr = tmp;
    }
    if (t < 0) t += q;
    return (uint64_t)t;
}
uint64_t host_shoup(uint64_t w, uint64_t q) {
    return (uint64_t)((((unsigned __int128)w) << 64) / q);
}

static uint64_t brv(uint64_t x, int bits) {
    uint64_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

static int bit_length(uint64_t x) {
    int b = 0;
    while (x) {
        ++b;
        x >>= 1;
    }
    return b;
}

// The reference's deterministic root search (ntt_new_proc, ntt_portable.c:137-154):
// the first g = 2, 3, ... whose (q-1)/2P power has order exactly 2P.
static uint64_t find_root(uint64_t P, uint64_t q) {
    for (uint64_t g = 2; g < q; ++g) {
        uint64_t c = host_pow_mod(g, (q - 1) / (2 * P), q);
        if (host_pow_mod(c, P, q) == q - 1) return c;
    }
    return 0;
}

bool build_prime(IncNtt* t, uint64_t q, PrimeInfo* out, _NTT_proc* proc,
                 std::vector<uint64_t>& twist_host) {
    const uint64_t P = t->P;
    const int logP = t->logP;
    if (q < 3 || q >= (1ULL << 61) || ((q - 1) % (2 * P)) != 0) {
        set_error("new_incomplete_ntt_list", "prime must be below 2^61 and congruent to 1 mod 2N/split");
        return false;
    }
    const uint64_t psi = find_root(P, q);
    const uint64_t psi_inv = host_inv_mod(psi, q);
    proc->n = P;
    proc->q = q;
    proc->root_of_unity = psi;
    proc->inv_root_of_unity = psi_inv;

    std::vector<uint64_t> fwd(2 * P), inv(2 * P), tw(2 * P);
    // forward / inverse twiddles: table[brv(i)] = psi^(+-i)   (ntt_portable.c:18-62)
    uint64_t pf = 1, pi = 1;
    for (uint64_t i = 0; i < P; ++i) {
        uint64_t idx = brv(i, logP);
        fwd[2 * idx] = pf;
        fwd[2 * idx + 1] = host_shoup(pf, q);
        inv[2 * idx] = pi;
        inv[2 * idx + 1] = host_shoup(pi, q);
        pf = host_mul_mod(pf, psi, q);
        pi = host_mul_mod(pi, psi_inv, q);
    }
    // split-product twist: w[k] = psi^(2 brv(k) + 1)   (rns_polynomial.c:19-27, misc.c:186-192)
    twist_host.resize(P);
    for (uint64_t kk = 0; kk < P; ++kk) {
        uint64_t w = host_pow_mod(psi, 2 * brv(kk, logP) + 1, q);
        twist_host[kk] = w;
        tw[2 * kk] = w;
        tw[2 * kk + 1] = host_shoup(w, q);
    }
    // FP64 twiddles: centred w and fl(w / q) (see fp64mod.cuh for why this is exact)
    const bool fp64 = q < (1ULL << 50);
    std::vector<double> fwd_d(2 * P), inv_d(2 * P);
    auto centred = [q](uint64_t v) -> double {
        return v > q / 2 ? -(double)(q - v) : (double)v;
    };
    for (uint64_t i = 0; i < P && fp64; ++i) {
        fwd_d[2 * i] = centred(fwd[2 * i]);
        fwd_d[2 * i + 1] = fwd_d[2 * i] / (double)q;
        inv_d[2 * i] = centred(inv[2 * i]);
        inv_d[2 * i + 1] = inv_d[2 * i] / (double)q;
    }
    // lane-major copies of the bit 0..3 twiddles (layout described with PrimeInfo)
    const uint64_t nblk = P / 16, lane_pairs = ((nblk + 31) / 32) * 15 * 32;
    std::vector<double> fwd_l(2 * lane_pairs, 0.0), inv_l(2 * lane_pairs, 0.0);
    for (uint64_t g = 0; g < nblk && fp64; ++g)
        for (int b = 0; b < 4; ++b)
            for (uint64_t h = 0; h < (1u << (3 - b)); ++h) {
                const uint64_t src = (P >> (b + 1)) + (g << (3 - b)) + h;
                const uint64_t dst = (((g >> 5) * 15 + ((1u << (3 - b)) - 1) + h) << 5) + (g & 31);
                fwd_l[2 * dst] = fwd_d[2 * src];
                fwd_l[2 * dst + 1] = fwd_d[2 * src + 1];
                inv_l[2 * dst] = inv_d[2 * src];
                inv_l[2 * dst + 1] = inv_d[2 * src + 1];
            }
    // the same for the stages at bits 2..5, by 64-residue group G (layout described
    // with PrimeInfo)
    const uint64_t ngrp = P / 64, mid_pairs = ((ngrp + 31) / 32) * 15 * 32;
    std::vector<double> fwd_m(2 * mid_pairs, 0.0), inv_m(2 * mid_pairs, 0.0);
    for (uint64_t g = 0; g < ngrp && fp64; ++g)
        for (int bb = 0; bb < 4; ++bb)
            for (uint64_t h = 0; h < (1u << (3 - bb)); ++h) {
                const uint64_t src = (P >> (bb + 3)) + (g << (3 - bb)) + h;
                const uint64_t dst = (((g >> 5) * 15 + ((1u << (3 - bb)) - 1) + h) << 5) + (g & 31);
                fwd_m[2 * dst] = fwd_d[2 * src];
                fwd_m[2 * dst + 1] = fwd_d[2 * src + 1];
                inv_m[2 * dst] = inv_d[2 * src];
                inv_m[2 * dst + 1] = inv_d[2 * src + 1];
            }
    void* blk = nullptr;
    const size_t bytes = sizeof(uint64_t) * (10 * P + 4 * lane_pairs + 4 * mid_pairs);
    if (!check_cuda(cudaMalloc(&blk, bytes), "table alloc")) return false;
    uint64_t* d = (uint64_t*)blk;
    if (!check_cuda(cudaMemcpy(d, fwd.data(), 16 * P, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 2 * P, inv.data(), 16 * P, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 4 * P, tw.data(), 16 * P, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 6 * P, fwd_d.data(), 16 * P, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 8 * P, inv_d.data(), 16 * P, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 10 * P, fwd_l.data(), 16 * lane_pairs, cudaMemcpyHostToDevice), "table upload") ||
        !check_cuda(cudaMemcpy(d + 10 * P + 2 * lane_pairs, inv_l.data(), 16 * lane_pairs, cudaMemcpyHostToDevice),
                    "table upload"))
        return false;
    uint64_t* dm = d + 10 * P + 4 * lane_pairs;
    if (mid_pairs && (!check_cuda(cudaMemcpy(dm, fwd_m.data(), 16 * mid_pairs, cudaMemcpyHostToDevice), "table upload") ||
                      !check_cuda(cudaMemcpy(dm + 2 * mid_pairs, inv_m.data(), 16 * mid_pairs, cudaMemcpyHostToDevice),
                                  "table upload")))
        return false;
    t->dev_blocks.push_back(blk);

    PrimeInfo& o = *out;
    memset(&o, 0, sizeof o);
    o.q = q;
    o.two_q = 2 * q;
    const int b = bit_length(q);
    o.bar_shift = (uint32_t)(b - 2);
    o.bar_mu = (uint64_t)((((unsigned __int128)1) << (b + 62)) / q);
    o.log_p = (uint32_t)logP;
    o.p_inv = host_inv_mod(P % q, q);
    o.p_inv_sh = host_shoup(o.p_inv, q);
    const uint64_t last_tw = P >= 2 ? inv[2 * 1] : 1;
    o.inv_last = host_mul_mod(last_tw, o.p_inv, q);
    o.inv_last_sh = host_shoup(o.inv_last, q);
    o.fwd = d;
    o.inv = d + 2 * P;
    o.twist = d + 4 * P;
    o.fwd_d = reinterpret_cast<const double*>(d + 6 * P);
    o.inv_d = reinterpret_cast<const double*>(d + 8 * P);
    o.fwd_lane = reinterpret_cast<const double*>(d + 10 * P);
    o.inv_lane = reinterpret_cast<const double*>(d + 10 * P + 2 * lane_pairs);
    o.fwd_mid = mid_pairs ? reinterpret_cast<const double*>(dm) : nullptr;
    o.inv_mid = mid_pairs ? reinterpret_cast<const double*>(dm + 2 * mid_pairs) : nullptr;
    o.fp64 = fp64 ? 1 : 0;
    o.qd = (double)q;
    o.qinv = 1.0 / (double)q;
    o.pinv_d = centred(o.p_inv);
    o.pinv_q = o.pinv_d / (double)q;
    o.ilast_d = centred(o.inv_last);
    o.ilast_q = o.ilast_d / (double)q;
    return true;
}

bool upload_prime_info(IncNtt* t) {
    const size_t n = t->info.size();
    if (n > t->d_info_cap) {
        size_t cap = n < 64 ? 64 : n;
        PrimeInfo* d = nullptr;
        if (!check_cuda(cudaMalloc(&d, cap * sizeof(PrimeInfo)), "prime info alloc")) return false;
        if (t->d_info) {
            // the old table may still be read by queued kernels: drain first
            cudaStreamSynchronize(ctx().stream);
            cudaFree(t->d_info);
        }
        t->d_info = d;
        t->d_info_cap = cap;
    }
    if (!check_cuda(cudaMemcpy(t->d_info, t->info.data(), n * sizeof(PrimeInfo), cudaMemcpyHostToDevice),
                    "prime info upload"))
        return false;
    // the last of a pool's uploads (tables of every added prime, then this one):
    // a pageable upload on the legacy stream may return before its DMA lands, and the
    // kernels that read it run on non-blocking streams: wait for the legacy stream
    return check_cuda(cudaStreamSynchronize(0), "prime info upload");
}

static bool add_primes(IncNtt* t, const uint64_t* primes, uint64_t count) {
    const uint64_t P = t->P;
    for (uint64_t i = 0; i < count; ++i) {
        PrimeInfo pi;
        _NTT_proc* proc = (_NTT_proc*)calloc(1, sizeof(_NTT_proc));
        std::vector<uint64_t> tw;
        if (!build_prime(t, primes[i], &pi, proc, tw)) {
            free(proc);
            return false;
        }
        uint64_t* w_row = (uint64_t*)aligned_alloc(64, ((P * 8 + 63) / 64) * 64);
        memcpy(w_row, tw.data(), P * 8);
        t->info.push_back(pi);
        t->procs.push_back(proc);
        // public arrays are reallocated as the pool grows
        t->pub.ntt = (NTT_proc*)realloc(t->pub.ntt, sizeof(NTT_proc) * t->procs.size());
        t->pub.w = (uint64_t**)realloc(t->pub.w, sizeof(uint64_t*) * t->procs.size());
        t->pub.ntt[t->procs.size() - 1] = proc;
        t->pub.w[t->procs.size() - 1] = w_row;
    }
    t->pub.l = t->procs.size();
    return upload_prime_info(t);
}

IncNtt* ntt_create(const uint64_t* primes, uint64_t split, uint64_t N, uint64_t count) {
    if (!ensure_ready()) return nullptr;
    if (split == 0 || N == 0 || (N & (N - 1)) || (split & (split - 1)) || split > N) {
        set_error("new_incomplete_ntt_list", "N and split_degree must be powers of two with split <= N");
        return nullptr;
    }
    IncNtt* t = new IncNtt();
    t->pub.ntt = nullptr;
    t->pub.w = nullptr;
    t->pub.N = N;
    t->pub.split_degree = split;
    t->pub.l = 0;
    t->P = N / split;
    int lp = 0;
    while ((1ULL << lp) < t->P) ++lp;
    t->logP = lp;
    if (lp > 17) {
        set_error("new_incomplete_ntt_list", "N/split_degree above 2^17 is not supported");
        delete t;
        return nullptr;
    }
    if (count > (uint64_t)kMaxLimbs) {
        set_error("new_incomplete_ntt_list", "at most 64 primes per pool (rns_mask is 64-bit)");
        delete t;
        return nullptr;
    }
    if (!add_primes(t, primes, count)) {
        delete t;
        return nullptr;
    }
    return t;
}

bool ntt_extend(IncNtt* t, const uint64_t* primes, uint64_t count) {
    if (t->procs.size() + count > (uint64_t)kMaxLimbs) {
        set_error("incNTT_extend_with_primes", "at most 64 primes per pool (rns_mask is 64-bit)");
        return false;
    }
    return add_primes(t, primes, count);
}

Poly* poly_create(uint64_t N, uint64_t mask, IncNtt* t) {
    if (!t) {
        set_error("polynomial_new_RNS_polynomial", "null incNTT");
        return nullptr;
    }
    Poly* p = new Poly();
    const uint64_t l = t->pub.l;
    p->base = (uint64_t*)managed_alloc(sizeof(uint64_t) * l * t->pub.N);
    p->pub.coeffs = (uint64_t**)malloc(sizeof(uint64_t*) * (l ? l : 1));
    for (uint64_t i = 0; i < l; ++i) p->pub.coeffs[i] = p->base ? p->base + i * t->pub.N : nullptr;
    p->pub.ntt = &t->pub;
    p->pub.rns_mask = mask;
    p->pub.allocated_l = l;
    (void)N;
    return p;
}

void poly_destroy(Poly* p) {
    if (!p) return;
    managed_free(p->base);
    free(p->pub.coeffs);
    delete p;
}

}  // namespace vc

namespace vc {
namespace {
std::atomic<uint64_t> g_launches{0};
}
void note_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
uint64_t launch_counter() { return g_launches.load(); }
void forget_launches(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
}  // namespace vc

// ---------------------------------------------------------------- status ABI
extern "C" {

uint64_t vfhe_cuda_launch_count(void) { return vc::g_launches.load(); }

int vfhe_cuda_status(void) { return vc::g_status; }

const char* vfhe_cuda_last_error(void) { return vc::g_error; }

void vfhe_cuda_clear_error(void) {
    std::lock_guard<std::mutex> lk(vc::g_err_mu);
    vc::g_status = 0;
    vc::g_error[0] = '\0';
}

int vfhe_cuda_device(void) {
    if (!vc::ensure_ready()) return -1;
    return vc::ctx().device;
}

int vfhe_cuda_synchronize(void) {
    if (!vc::ensure_ready()) return 1;
    return vc::sync("vfhe_cuda_synchronize") ? 0 : 1;
}

}  // extern "C"
