// CKKS special FFT on the GPU: the complex-FFT entry points of the cdef
// (arith.cdef:84-93; modules/arith/c/src/complex.c) and a batched encoder.
//
// Layout (as the reference): a complex polynomial of n slots is 2n doubles, the n real
// parts then the n imaginary parts.  Twiddle tables (load_rous_CT / load_rous_GS) are
// indexed like the reference's scalar build, ws[m + i] for stage m.  The butterflies
// use exactly the reference's scalar operation order (complex.c:389-440): a complex
// product is re = ar*br - ai*bi, im = ar*bi + br*ai, each product and sum rounded
// separately (no fused multiply-add), so every result is bit-identical to the
// reference's portable engine.
//
// The caller's buffers are host memory (safe_aligned_malloc); each entry point copies
// in, runs the stages as kernels and copies back before returning (synchronous, like
// every cdef call).  complex_polys_ifft_scale_round_to_RNS_batch runs a whole batch of
// encodings in one pass over the device.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "abi_common.cuh"

namespace vc {

struct RouTable {
    uint64_t size = 0;
    double* d_re = nullptr;
    double* d_im = nullptr;
};

namespace {

// exact reference rounding: separate products and sums
__device__ __forceinline__ void cmul_ref(double& cr, double& ci, double ar, double ai, double br, double bi) {
    ci = __dadd_rn(__dmul_rn(ar, bi), __dmul_rn(br, ai));
    cr = __dsub_rn(__dmul_rn(ar, br), __dmul_rn(ai, bi));
}

// one Cooley-Tukey stage (m groups, half-size t) on `count` arrays of n complex values
__global__ void k_ct_stage(double* __restrict__ x, const double* __restrict__ wr, const double* __restrict__ wi,
                           long long n, long long m, long long t, long long count) {
    const long long half = n / 2, total = half * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long a = e / half, k = e - a * half;
        const long long i = k / t, j = 2 * i * t + (k - i * t);
        double* re = x + a * 2 * n;
        double* im = re + n;
        double vr, vi;
        cmul_ref(vr, vi, re[j + t], im[j + t], wr[m + i], wi[m + i]);
        const double ur = re[j], ui = im[j];
        re[j + t] = __dsub_rn(ur, vr);
        im[j + t] = __dsub_rn(ui, vi);
        re[j] = __dadd_rn(ur, vr);
        im[j] = __dadd_rn(ui, vi);
    }
}

// one Gentleman-Sande stage (h groups, half-size t)
__global__ void k_gs_stage(double* __restrict__ x, const double* __restrict__ wr, const double* __restrict__ wi,
                           long long n, long long h, long long t, long long count) {
    const long long half = n / 2, total = half * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long a = e / half, k = e - a * half;
        const long long i = k / t, j = 2 * i * t + (k - i * t);
        double* re = x + a * 2 * n;
        double* im = re + n;
        const double vr = __dsub_rn(re[j], re[j + t]), vi = __dsub_rn(im[j], im[j + t]);
        re[j] = __dadd_rn(re[j], re[j + t]);
        im[j] = __dadd_rn(im[j], im[j + t]);
        double cr, ci;
        cmul_ref(cr, ci, vr, vi, wr[h + i], wi[h + i]);
        re[j + t] = cr;
        im[j + t] = ci;
    }
}

// the reference's 20-bit reversal (complex.c:13-24), then >> (20 - prec)
__host__ __device__ __forceinline__ uint32_t brv20(uint32_t x, uint32_t prec) {
    uint32_t r = 0;
    for (int b = 0; b < 20; ++b) r |= ((x >> b) & 1u) << (19 - b);
    return r >> (20 - prec);
}

// dst[a][brv(i)] = src[a][i] for both halves
__global__ void k_bit_reverse(double* __restrict__ dst, const double* __restrict__ src, long long n, uint32_t prec,
                              long long count) {
    const long long total = 2 * n * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long a = e / (2 * n), r = e - a * 2 * n;
        const long long h = r / n, i = r - h * n;
        dst[a * 2 * n + h * n + brv20((uint32_t)i, prec)] = src[e];
    }
}

__global__ void k_scale(double* __restrict__ x, double s, long long total) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x)
        x[e] = __dmul_rn(x[e], s);
}

// llrint of the first nc values of each array (the ring degree), two's complement
__global__ void k_round(int64_t* __restrict__ out, const double* __restrict__ x, long long n2, long long nc,
                        long long count) {
    const long long total = nc * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long a = e / nc, i = e - a * nc;
        out[e] = __double2ll_rn(x[a * n2 + i]);
    }
}

unsigned grid_of(long long work) {
    long long b = (work + 255) / 256;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)b;
}

int run_ct(double* d, const RouTable* w, long long n, long long count, cudaStream_t st) {
    long long t = n, m = 1;
    while (m < n) {
        t >>= 1;
        k_ct_stage<<<grid_of(n / 2 * count), 256, 0, st>>>(d, w->d_re, w->d_im, n, m, t, count);
        note_launch();
        const int e = (int)cudaGetLastError();
        if (e) return e;
        m <<= 1;
    }
    return 0;
}

int run_gs(double* d, const RouTable* w, long long n, long long count, cudaStream_t st) {
    long long t = 1, m = n;
    while (m > 1) {
        const long long h = m >> 1;
        k_gs_stage<<<grid_of(n / 2 * count), 256, 0, st>>>(d, w->d_re, w->d_im, n, h, t, count);
        note_launch();
        const int e = (int)cudaGetLastError();
        if (e) return e;
        t <<= 1;
        m >>= 1;
    }
    return 0;
}

int run_brv(double* d, double* tmp, long long n, uint32_t prec, long long count, cudaStream_t st) {
    k_bit_reverse<<<grid_of(2 * n * count), 256, 0, st>>>(tmp, d, n, prec, count);
    note_launch();
    int e = (int)cudaGetLastError();
    if (!e) e = (int)cudaMemcpyAsync(d, tmp, sizeof(double) * 2 * n * count, cudaMemcpyDeviceToDevice, st);
    return e;
}

RouTable* load_rous(const double* re, const double* im, uint64_t size, const char* where) {
    if (!ensure_ready()) return nullptr;
    if (!re || !im || size < 2 || (size & (size - 1))) {
        set_error(where, "table size must be a power of two >= 2");
        return nullptr;
    }
    RouTable* t = new RouTable();
    t->size = size;
    if (cudaMalloc(&t->d_re, size * 8) != cudaSuccess || cudaMalloc(&t->d_im, size * 8) != cudaSuccess ||
        cudaMemcpy(t->d_re, re, size * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(t->d_im, im, size * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess) {  // the uploads have landed before engine-stream kernels read them
        cudaFree(t->d_re);
        cudaFree(t->d_im);
        delete t;
        set_error(where, "device allocation failed");
        return nullptr;
    }
    return t;
}

// host buffer in -> device -> fn -> host buffer out
template <typename F>
void on_device(double* host, long long doubles, const char* where, F fn) {
    double* d = (double*)device_alloc(doubles * 8);
    if (!d) return;
    cudaStream_t st = stream();
    int e = (int)cudaMemcpyAsync(d, host, doubles * 8, cudaMemcpyHostToDevice, st);
    if (!e) e = fn(d, st);
    if (!e) e = (int)cudaMemcpyAsync(host, d, doubles * 8, cudaMemcpyDeviceToHost, st);
    if (!e) e = (int)cudaStreamSynchronize(st);
    check_cuda(e, where);
    device_free(d);
}

bool valid_handle(void* p, const char* where) {
    if (!p) {
        set_error(where, "null polynomial handle");
        return false;
    }
    return true;
}

bool valid_table(void* ws, uint64_t n, const char* where) {
    const RouTable* w = (const RouTable*)ws;
    if (!w || n < 2 || (n & (n - 1)) || w->size < n) {
        set_error(where, "twiddle table smaller than the transform, or n not a power of two");
        return false;
    }
    return true;
}

}  // namespace

// Scatter of signed 64-bit integers into every active limb of `out` followed by its
// forward transform (int_array_to_RNS semantics), from a device array; abi_arith.cu.
int int_array_to_RNS_device(void* out, const int64_t* d_in, cudaStream_t st);

}  // namespace vc

using namespace vc;

extern "C" {

void* load_rous_CT(double* rous_real, double* rous_imag, uint64_t size) {
    return load_rous(rous_real, rous_imag, size, "load_rous_CT");
}

void* load_rous_GS(double* rous_real, double* rous_imag, uint64_t size) {
    return load_rous(rous_real, rous_imag, size, "load_rous_GS");
}

void CT_NR(double* x, void* ws, uint64_t n) {
    if (!ensure_ready() || !x || !valid_table(ws, n, "CT_NR")) return;
    on_device(x, 2 * (long long)n, "CT_NR",
              [&](double* d, cudaStream_t st) { return run_ct(d, (const RouTable*)ws, (long long)n, 1, st); });
}

void GS_RN(double* x, void* ws, uint64_t n) {
    if (!ensure_ready() || !x || !valid_table(ws, n, "GS_RN")) return;
    on_device(x, 2 * (long long)n, "GS_RN",
              [&](double* d, cudaStream_t st) { return run_gs(d, (const RouTable*)ws, (long long)n, 1, st); });
}

void bit_reverse_array(double* v, uint64_t N, uint32_t prec) {
    if (!ensure_ready() || !v) return;
    if (prec > 20 || (N > (1ULL << prec))) {
        set_error("bit_reverse_array", "N must be at most 2^prec and prec at most 20");
        return;
    }
    double* tmp = (double*)device_alloc(16 * N);
    if (!tmp) return;
    on_device(v, 2 * (long long)N, "bit_reverse_array",
              [&](double* d, cudaStream_t st) { return run_brv(d, tmp, (long long)N, prec, 1, st); });
    device_free(tmp);
}

void complex_poly_scale_double(double* v, double scale, uint64_t N) {
    if (!ensure_ready() || !v) return;
    on_device(v, 2 * (long long)N, "complex_poly_scale_double", [&](double* d, cudaStream_t st) {
        k_scale<<<grid_of(2 * (long long)N), 256, 0, st>>>(d, scale, 2 * (long long)N);
        note_launch();
        return (int)cudaGetLastError();
    });
}

void complex_poly_round_to_RNS(void* out, double* in, uint64_t N) {
    (void)N;
    VC_ENTER("complex_poly_round_to_RNS");
    if (!valid_handle(out, vc_where_) || !in) return;
    const long long n = (long long)pool_of(as_poly(out))->pub.N;
    double* d = (double*)device_alloc(n * 8);
    int64_t* r = (int64_t*)device_alloc(n * 8);
    if (!d || !r) return;
    VC_CHECK(cudaMemcpyAsync(d, in, n * 8, cudaMemcpyHostToDevice, stream()));
    k_round<<<grid_of(n), 256, 0, stream()>>>(r, d, n, n, 1);
    note_launch();
    VC_CHECK(cudaGetLastError());
    VC_CHECK(int_array_to_RNS_device(out, r, stream()));
    VC_FINISH();
    device_free(d);
    device_free(r);
}

void complex_polys_ifft_scale_round_to_RNS_batch(void** rows_in, void** outs_rns, uint64_t count,
                                                 uint64_t n_complex, uint32_t log_prec, void* gs_ws,
                                                 double temp_delta) {
    VC_ENTER("complex_polys_ifft_scale_round_to_RNS_batch");
    if (!rows_in || !outs_rns || count == 0) return;
    if (!valid_table(gs_ws, n_complex, vc_where_)) return;
    for (uint64_t i = 0; i < count; ++i)
        if (!valid_handle(outs_rns[i], vc_where_) || !rows_in[i]) return;
    const long long n = (long long)n_complex, n2 = 2 * n, B = (long long)count;
    const long long nc = (long long)pool_of(as_poly(outs_rns[0]))->pub.N;
    if (nc > n2) {
        set_error(vc_where_, "ring degree above 2 n_complex");
        return;
    }
    double* d = (double*)device_alloc(B * n2 * 8);
    double* tmp = (double*)device_alloc(B * n2 * 8);
    int64_t* r = (int64_t*)device_alloc(B * nc * 8);
    if (!d || !tmp || !r) return;
    cudaStream_t st = stream();
    for (long long i = 0; i < B; ++i)
        VC_CHECK(cudaMemcpyAsync(d + i * n2, rows_in[i], n2 * 8, cudaMemcpyHostToDevice, st));
    // per row: bit reversal, GS_RN, scale by temp_delta / n, round (complex.c batch thread)
    VC_CHECK(run_brv(d, tmp, n, log_prec, B, st));
    VC_CHECK(run_gs(d, (const RouTable*)gs_ws, n, B, st));
    k_scale<<<grid_of(B * n2), 256, 0, st>>>(d, temp_delta / (double)n_complex, B * n2);
    note_launch();
    k_round<<<grid_of(B * nc), 256, 0, st>>>(r, d, n2, nc, B);
    note_launch();
    VC_CHECK(cudaGetLastError());
    for (long long i = 0; i < B; ++i) {
        VC_CHECK(int_array_to_RNS_device(outs_rns[i], r + i * nc, st));
        // the reference transforms the caller's rows in place
        VC_CHECK(cudaMemcpyAsync(rows_in[i], d + i * n2, n2 * 8, cudaMemcpyDeviceToHost, st));
    }
    VC_FINISH();
    device_free(d);
    device_free(tmp);
    device_free(r);
}

}  // extern "C"
