/*
 * vfhe_cuda.h -- C ABI of the B200 `cuda` engine for vfhe's RNS polynomial hot path.
 *
 * Part 1 is the drop-in surface: the functions and struct prefixes that vfhe's
 * cffi layer binds for every engine.  Names, argument order and meaning follow the
 * reference cdefs line by line:
 *   modules/arith/python/cdef/arith.cdef   (cited as arith.cdef:<line>)
 *   modules/misc/python/cdef/misc.cdef     (misc.cdef:<line>)
 *   modules/misc/python/cdef/vfhe_cpu.cdef (vfhe_cpu.cdef:<line>)
 *   modules/mlwe/python/cdef/mlwe.cdef     (mlwe.cdef:<line>)
 *   modules/fhe/python/cdef/fhe.cdef       (fhe.cdef:<line>)
 * Handles are `void *`; outputs are caller-allocated out-params, first.  Calls are
 * synchronous: when a function returns, its results are readable from the host
 * through the coefficient pointers (coefficient rows live in CUDA managed memory).
 *
 * Part 2 is new: a batched device API over plain device pointers and a CUDA
 * stream, for callers that keep ciphertexts and keys resident in HBM.
 *
 * Errors: the reference aborts on contract violations.  This engine records the
 * first error instead (vfhe_cuda_last_error) and returns; batched entry points
 * also return a nonzero status.
 *
 * This header is also the cffi cdef source: keep it free of macros other than the
 * include guard and the extern "C" block.
 */
#ifndef VFHE_CUDA_H
#define VFHE_CUDA_H

#include <stdbool.h>
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ===================================================================== *
 * Part 1: drop-in surface                                                *
 * ===================================================================== */

/* Opaque per-prime transform descriptor (arith.cdef:8; modules/arith/c/include/arith.h:29-46).
 * Its first two fields are the transform size n and the prime q, as in the reference. */
typedef struct _NTT_proc *NTT_proc;

/* Pool of primes for one (N, split_degree) (arith.cdef:10-16; arith.h:48-54).
 * w[i] holds the split-product twist row of prime i (N/split_degree values, host-readable). */
typedef struct _incNTT {
  NTT_proc *ntt;
  uint64_t split_degree;
  uint64_t **w;
  uint64_t N;
  uint64_t l;
} *incNTT;

/* RNS polynomial (arith.cdef:18-23; arith.h:72-78): one row of N residues per limb of
 * the pool, rns_mask selects the active limbs.  Rows are host-dereferenceable. */
typedef struct _RNS_Polynomial {
  uint64_t **coeffs;
  incNTT ntt;
  uint64_t rns_mask;
  uint64_t allocated_l;
} *RNS_Polynomial;

/* --- misc --- */
void *safe_aligned_malloc(uint64_t size);                                            /* arith.cdef:26 */

/* --- ntt / base conversion --- */
void *new_incomplete_ntt_list(uint64_t *primes, uint64_t split_degree, uint64_t N, uint64_t count); /* arith.cdef:29 */
void incNTT_extend_with_primes(void *ntt, uint64_t *new_primes, uint64_t count);   /* arith.cdef:30 */
uint64_t **incNTT_get_rou_matrix(void *ntt);                                       /* arith.cdef:31 */
void *init_base_conversion_params(void *ntt, uint64_t in_mask, uint64_t out_mask);  /* arith.cdef:32 */
void free_base_conversion_params(void *params);                                    /* arith.cdef:33 */

/* --- polynomial lifecycle / io --- */
void *polynomial_new_RNS_polynomial(uint64_t N, uint64_t rns_mask, void *ntt);      /* arith.cdef:36 */
void polynomial_copy_RNS_polynomial(void *out, void *in);                          /* arith.cdef:37 */
void free_RNS_polynomial(void *p);                                                 /* arith.cdef:38 */
void int_array_to_RNS(void *out, uint64_t *in);                                    /* arith.cdef:39 */
void array_to_RNS(void *out, uint64_t **in);                                       /* arith.cdef:40 */

/* --- sampling (engine-specific random stream, as in the reference) --- */
void polynomial_gen_random_RNSc_polynomial(void *out);                             /* arith.cdef:43 */
void polynomial_gen_gaussian_RNSc_polynomial(void *out, double sigma);             /* arith.cdef:44 */

/* --- arithmetic --- */
void polynomial_mul_RNS_polynomial(void *out, void *in1, void *in2);               /* arith.cdef:47 */
void polynomial_multo_RNS_polynomial(void *out, void *in);                         /* arith.cdef:48 */
void polynomial_sub_RNS_polynomial(void *out, void *in1, void *in2);               /* arith.cdef:49 */
void polynomial_sub_RNSc_polynomial(void *out, void *in1, void *in2);              /* arith.cdef:50 */
void polynomial_add_RNSc_polynomial(void *out, void *in1, void *in2);              /* arith.cdef:51 */
void polynomial_add_RNS_polynomial(void *out, void *in1, void *in2);               /* arith.cdef:52 */
void polynomial_scale_RNSc_polynomial(void *out, void *in1, uint64_t scale);       /* arith.cdef:53 */
void polynomial_scale_RNS_polynomial_RNS(void *out, void *in1, uint64_t *scale);   /* arith.cdef:54 */
void polynomial_RNSc_negate(void *out, void *in);                                  /* arith.cdef:55 */
void polynomial_RNSc_add_integer(void *out, void *in1, uint64_t in2);              /* arith.cdef:56 */
void polynomial_RNS_add_integer(void *out, void *in1, uint64_t in2);               /* arith.cdef:57 */

/* --- automorphism / domain conversion --- */
void polynomial_RNSc_permute(void *out, void *in, uint64_t gen);                   /* arith.cdef:60 */
void polynomial_RNSc_to_RNS(void *out, void *in);                                  /* arith.cdef:61 */
void polynomial_RNS_to_RNSc(void *out, void *in);                                  /* arith.cdef:62 */

/* --- tower --- */
void polynomial_base_conversion_RNSc(void *out, void *in, void *params);           /* arith.cdef:65 */
void polynomial_RNSc_mod_reduce(void *out, void *in);                              /* arith.cdef:66 */
void polynomial_RNSc_mod_reduce_lifted(void *out, void *in, uint64_t idx);         /* arith.cdef:67 */
void polynomial_round_division_RNSc_wo_free(void *out, uint64_t divide_mask);      /* arith.cdef:68 */
void polynomial_floor_division_RNSc_wo_free(void *out, uint64_t divide_mask);      /* arith.cdef:69 */
void polynomial_RNSc_scaled_lift(void *out, void *in, uint64_t *delta);            /* arith.cdef:70 */

/* --- slots / inverse / eq --- */
int polynomial_RNS_inverse(void *out, void *in);                                   /* arith.cdef:73 */
bool polynomial_eq(void *a, void *b);                                              /* arith.cdef:74 */
void polynomial_RNS_broadcast_slot(void *out, void *in, uint64_t slot_idx);        /* arith.cdef:75 */
void polynomial_RNS_rotate_slot(void *out, void *in, uint64_t rot);                /* arith.cdef:76 */
void polynomial_RNS_copy_slot(void *out, uint64_t dst, void *in, uint64_t src);    /* arith.cdef:77 */

/* --- hashing: BLAKE3 is not part of this engine; these record an error --- */
void polynomial_RNS_get_hash(uint64_t *out, void *p);                              /* arith.cdef:80 */
uint64_t *polynomial_RNS_get_hash_p(void *p);                                      /* arith.cdef:81 */

/* --- complex FFT (CKKS encoding) --- */
void *load_rous_CT(double *rous_real, double *rous_imag, uint64_t size);           /* arith.cdef:84 */
void *load_rous_GS(double *rous_real, double *rous_imag, uint64_t size);           /* arith.cdef:85 */
void CT_NR(double *x, void *ws, uint64_t n);                                       /* arith.cdef:86 */
void GS_RN(double *x, void *ws, uint64_t n);                                       /* arith.cdef:87 */
void bit_reverse_array(double *v, uint64_t N, uint32_t prec);                      /* arith.cdef:88 */
void complex_poly_scale_double(double *v, double scale, uint64_t N);               /* arith.cdef:89 */
void complex_poly_round_to_RNS(void *out, double *in, uint64_t N);                 /* arith.cdef:90 */
void complex_polys_ifft_scale_round_to_RNS_batch(void **rows_in, void **outs_rns, uint64_t count,
                                                 uint64_t n_complex, uint32_t log_prec, void *gs_ws,
                                                 double temp_delta);                /* arith.cdef:91-93 */

/* --- multiprecision (outside the hot path; present so the surface links) --- */
typedef struct _mp_vector mp_vector_t;                                             /* arith.cdef:101 */
typedef struct _MPScalar { mp_vector_t *digits; uint64_t d; } *MPScalar;           /* arith.cdef:102 */
typedef struct _MPPolynomial { uint64_t **coeffs; uint64_t N; uint64_t d; } *MPPolynomial; /* arith.cdef:103 */
int get_mp_vector_size(void);                                                      /* arith.cdef:104 */
void mp_scale(void *out, void *in, void *m);                                       /* arith.cdef:105 */
void mp_sub(void *out, void *a, void *b);                                          /* arith.cdef:106 */
void *mp_load(uint64_t *in, uint64_t d);                                           /* arith.cdef:107 */
mp_vector_t *load_m512(uint64_t in);                                               /* arith.cdef:108 */
void *new_mp_polynomial(uint64_t N, uint64_t d);                                   /* arith.cdef:109 */
void mp_polynomial_from_RNS(void *out, void *in, MPScalar *PW, void *q, mp_vector_t *m, uint64_t k); /* arith.cdef:110 */
void mp_polynomial_to_RNSc(void *out, void *in);                                   /* arith.cdef:111 */

/* --- field extensions (outside the hot path; present so the surface links) --- */
void *field_new_proc(uint64_t q);                                                  /* arith.cdef:114 */
void field_ext_add(uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t d, uint64_t q); /* arith.cdef:115 */
void field_ext_sub(uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t d, uint64_t q); /* arith.cdef:116 */
void field_ext_neg(uint64_t *c, const uint64_t *a, uint64_t d, uint64_t q);        /* arith.cdef:117 */
void field_ext_mul(uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t d, uint64_t w, void *proc); /* arith.cdef:118 */
void field_ext_pow(uint64_t *res, const uint64_t *base, uint64_t exp_lo, uint64_t exp_hi, uint64_t d, uint64_t w, void *proc); /* arith.cdef:119 */
int field_ext_inv(uint64_t *ainv, const uint64_t *a, uint64_t d, uint64_t w, void *proc); /* arith.cdef:120 */
void field_sample_random_element(uint64_t *a, const uint8_t *seed, uint64_t seed_len, uint64_t d, uint64_t mod); /* arith.cdef:121 */
void field_hash_element(uint8_t *out, const uint64_t *a, uint64_t d);              /* arith.cdef:122 */
int field_ext_is_equal(const uint64_t *a, const uint64_t *b, uint64_t d);          /* arith.cdef:123 */
void field_base_conversion(uint64_t *out, const uint64_t *in,
                           uint64_t source_component, uint64_t target_component,
                           uint64_t d, uint64_t poly_size, const uint64_t *w_i, void *proc); /* arith.cdef:124-126 */
void ntt_free_proc(void *proc);                                                    /* arith.cdef:127 */
uint64_t inverse_mod_eea(uint64_t a, uint64_t p);                                  /* arith.cdef:128 */

/* --- misc.cdef / vfhe_cpu.cdef --- */
const char *vfhe_engine_active(void);                                              /* misc.cdef:8 */
void vfhe_prng_set_deterministic_seed(uint64_t seed);                              /* misc.cdef:12 */
void vfhe_prng_clear_deterministic_seed(void);                                     /* misc.cdef:13 */
int vfhe_cpu_supports(const char *capability);                                     /* vfhe_cpu.cdef:7 */
/* misc.cdef:17 binds libc free(); safe_aligned_malloc above returns libc memory. */

/* --- mlwe.cdef --- */
typedef struct _IntPolynomial *IntPolynomial;                                      /* mlwe.cdef:9 */

typedef struct _LWE_Key {                                                          /* mlwe.cdef:11-17 */
  uint64_t **s;
  uint64_t n;
  uint64_t l;
  incNTT ntt;
  double sigma;
} *LWE_Key;

typedef struct _LWE {                                                              /* mlwe.cdef:19-25 */
  uint64_t **a;
  uint64_t *b;
  uint64_t n;
  uint64_t l;
  incNTT ntt;
} *LWE;

typedef struct _RNS_MLWE {                                                         /* mlwe.cdef:27-31 */
  RNS_Polynomial *a;
  RNS_Polynomial b;
  uint64_t r;
} *RNS_MLWE;

typedef struct _RNS_MLWE_Key {                                                     /* mlwe.cdef:33-40 */
  IntPolynomial *s;
  RNS_Polynomial *s_RNS;
  uint64_t N;
  uint64_t l;
  uint64_t r;
  double sigma;
} *RNS_MLWE_Key;

/* lwe */
void *lwe_alloc_key(uint64_t n, uint64_t l, void *ntt);                            /* mlwe.cdef:43 */
void *lwe_alloc_sample(uint64_t n, uint64_t l, void *ntt);                         /* mlwe.cdef:44 */
void free_lwe_sample(void *c);                                                     /* mlwe.cdef:45 */
void *lwe_new_key(uint64_t n, uint64_t l, void *ntt, double sec_sigma, double err_sigma); /* mlwe.cdef:46 */
void *lwe_new_sparse_ternary_key(uint64_t n, uint64_t l, void *ntt, uint64_t h, double err_sigma); /* mlwe.cdef:47 */
void lwe_sample(void *c, uint64_t *m, void *key);                                  /* mlwe.cdef:48 */
void *lwe_new_sample(uint64_t *m, void *key);                                      /* mlwe.cdef:49 */
void *lwe_new_trivial_sample(uint64_t *m, uint64_t n, uint64_t l, void *ntt);      /* mlwe.cdef:50 */
void lwe_phase(uint64_t *out, void *c, void *key);                                 /* mlwe.cdef:51 */
void lwe_subto(void *out, void *in);                                               /* mlwe.cdef:52 */

/* mlwe (rns) */
void *mlwe_new_RNS_key_from_array(uint64_t *array, uint64_t N, uint64_t r, uint64_t l, void *ntt, double sigma); /* mlwe.cdef:55 */
void *mlwe_new_RNS_gaussian_key(uint64_t N, uint64_t r, uint64_t l, double key_sigma, void *ntt, double sigma);  /* mlwe.cdef:56 */
void *mlwe_alloc_RNS_sample(uint64_t N, uint64_t r, uint64_t mask, void *ntt);     /* mlwe.cdef:57 */
void *mlwe_alloc_RNS_sample_array(uint64_t size, uint64_t N, uint64_t r, uint64_t mask, void *ntt); /* mlwe.cdef:58 */
void *mlwe_create_copy_array(void *in, uint64_t size);                             /* mlwe.cdef:59 */
void free_mlwe_RNS_sample(void *p);                                                /* mlwe.cdef:60 */
void free_mlwe_RNS_key(void *key);                                                 /* mlwe.cdef:61 */

void mlwe_RNSc_sample(void *out, void *key, void *m);                              /* mlwe.cdef:63 */
void mlwe_RNS_phase(void *out, void *in, void *key);                               /* mlwe.cdef:64 */
void mlwe_RNSc_to_RNS(void *out, void *in);                                        /* mlwe.cdef:65 */
void mlwe_RNS_to_RNSc(void *out, void *in);                                        /* mlwe.cdef:66 */
void mlwe_copy_RNS_sample(void *out, void *in);                                    /* mlwe.cdef:67 */
void mlwe_RNS_trivial_sample_of_zero(void *out);                                   /* mlwe.cdef:68 */
void *mlwe_new_RNSc_sample_of_zero(void *key);                                     /* mlwe.cdef:69 */
void *mlwe_new_RNS_sample_of_zero(void *key);                                      /* mlwe.cdef:70 */
void *mlwe_new_RNS_trivial_sample_of_zero(uint64_t N, uint64_t r, uint64_t mask, void *ntt); /* mlwe.cdef:71 */

void mlwe_RNS_mul_addto_by_poly(void *out, void *in, void *poly);                  /* mlwe.cdef:73 */
void mlwe_RNS_mul_subto_by_poly(void *out, void *in, void *poly);                  /* mlwe.cdef:74 */
void mlwe_RNS_mul_by_poly(void *out, void *in, void *poly);                        /* mlwe.cdef:75 */
void mlwe_scale_RNS_mlwe_RNS(void *c, uint64_t *scale);                            /* mlwe.cdef:76 */
void mlwe_add_RNSc_sample(void *out, void *in1, void *in2);                        /* mlwe.cdef:77 */
void mlwe_sub_RNSc_sample(void *out, void *in1, void *in2);                        /* mlwe.cdef:78 */
void mlwe_RNSc_mul_by_xai(void *out, void *in, uint64_t a);                        /* mlwe.cdef:79 */
void mlwe_RNSc_mul_by_xai_minus1(void *out, void *in, uint64_t a);                 /* mlwe.cdef:80 */
void mlwe_add_RNSc_polynomial(void *out, void *in1, void *in2);                    /* mlwe.cdef:81 */
void mlwe_sub_RNSc_polynomial(void *out, void *in1, void *in2);                    /* mlwe.cdef:82 */
void mlwe_RNS_add_polynomial(void *out, void *in1, void *in2);                     /* mlwe.cdef:83 */
void mlwe_RNS_sub_polynomial(void *out, void *in1, void *in2);                     /* mlwe.cdef:84 */
void mlwe_round_division_RNSc(void *out, uint64_t divide_mask);                    /* mlwe.cdef:85 */

void *mlwe_extract_LWE(void *in, uint64_t idx);                                    /* mlwe.cdef:87 */
void mlwe_full_packing_keyswitch(void *out, void *in, uint64_t size, void *ksk, uint64_t lvl); /* mlwe.cdef:88 */
void mlwe_full_packing_keyswitch_scaled(void *vec, uint64_t ell, void *ksks, uint64_t lvl);    /* mlwe.cdef:89 */
void mlwe_RNSc_GHS_hybrid_keyswitch(void *out, void *in, void *ksk, uint64_t lvl); /* mlwe.cdef:90 */
void mlwe_automorphism_RNSc_GHS(void *out, void *in, uint64_t gen, void *ksk, uint64_t lvl); /* mlwe.cdef:91 */
void mlwe_partial_trace(void *out, void *in, uint64_t *gens, void *ksks, uint64_t size, uint64_t lvl); /* mlwe.cdef:92 */
void mlwe_trace(void *out, void *in, void *ksks, uint64_t lvl);                    /* mlwe.cdef:93 */
uint64_t mlwe_extended_rank(uint64_t r);                                           /* mlwe.cdef:94 */
void mlwe_tensor_product(void *out, void *in1, void *in2);                         /* mlwe.cdef:95 */
void mlwe_multiply(void *out, void *in1, void *in2, void *ksk);                    /* mlwe.cdef:96 */

/* mgsw */
void mgsw_external_product(void *out, void *mgsw, void *in, uint64_t ell, uint64_t special_primes); /* mlwe.cdef:99 */
void mgsw_CMUX(void *out, void *in1, void *in2, void *mgsw, uint64_t ell, uint64_t special_primes); /* mlwe.cdef:100 */
void mgsw_NCMUX(void *out, void *in1, void *in2, void *mgsw, void *ksk, uint64_t ell, uint64_t special_primes); /* mlwe.cdef:101 */

/* --- fhe.cdef: GP25 (outside the hot path; present so the surface links) --- */
void gp25_RGSW_monomial_mul(void *p0, uint64_t in_N, void *e, uint64_t r_prec, void *ksk, uint64_t ell, uint64_t special_primes); /* fhe.cdef:8 */
void gp25_RGSW_monomial_mul_mt(void *p0, uint64_t in_N, void *e, uint64_t r_prec, void *ksk, uint64_t ell, uint64_t special_primes, uint64_t num_threads); /* fhe.cdef:9 */
void gp25_sub_a_mt(void *p0, uint64_t in_N, uint64_t *a, void *s_sign, uint64_t ell, uint64_t special_primes, uint64_t N, uint64_t num_threads); /* fhe.cdef:10 */

/* ===================================================================== *
 * Part 2: batched device API (new; no reference counterpart)             *
 * ===================================================================== */

/* The batched CKKS multiply, rotation and key switch take batches of any size: past
 * 65535 / (2 (nlimbs + 1)) ciphertexts (one pass of their kernels' grids) they run as
 * consecutive passes on the same stream, sharing one pass's workspace, with the same
 * residues (a caller-supplied workspace sized for the whole batch also serves).
 * An empty batch (batch = 0, or nsrc = 0 for key generation) is a successful no-op
 * for the batched compute calls below once the pool and limb list check out: nothing
 * is launched and no workspace is touched (vfhe_cuda_ntt_mul_intt_batch_noalloc keeps
 * rejecting it, as documented there). */

/* Engine status: 0 when no error has been recorded since the last clear. */
int vfhe_cuda_status(void);
const char *vfhe_cuda_last_error(void);
void vfhe_cuda_clear_error(void);
/* Device ordinal this engine runs on, and a sync of its internal stream. */
int vfhe_cuda_device(void);
int vfhe_cuda_synchronize(void);
/* Number of transform and batched-CKKS kernels this engine has launched so far. */
uint64_t vfhe_cuda_launch_count(void);

/* Batched negacyclic (incomplete) NTT over a device buffer laid out as
 * [batch][nlimbs][N] uint64 residues; limb slot k uses pool prime limbs[k] of the
 * incNTT `ntt` (same split_degree layout as polynomial_RNSc_to_RNS).
 * inverse = 0: coefficient -> NTT (polynomial_RNSc_to_RNS, rns_polynomial.c:582-597);
 * inverse = 1: NTT -> coefficient (polynomial_RNS_to_RNSc, rns_polynomial.c:599-614).
 * d_out may equal d_in.  `stream` is a cudaStream_t (NULL = legacy default stream). */
int vfhe_cuda_ntt_batch(void *ntt, int inverse, uint64_t *d_out, const uint64_t *d_in,
                        uint64_t batch, const uint32_t *limbs, uint32_t nlimbs, void *stream);

/* Batched incomplete ring product d_out = d_a * d_b over [batch][nlimbs][N] NTT-domain
 * buffers (polynomial_mul_RNS_polynomial, rns_polynomial.c:311-356). */
int vfhe_cuda_poly_mul_batch(void *ntt, uint64_t *d_out, const uint64_t *d_a, const uint64_t *d_b,
                             uint64_t batch, const uint32_t *limbs, uint32_t nlimbs, void *stream);

/* Fused NTT -> incomplete product -> INTT for `batch` pairs of coefficient-domain
 * polynomials [batch][nlimbs][N]: d_out = INTT(NTT(d_a) * NTT(d_b)).  One kernel, no
 * scratch, for primes below 2^50, N <= 2^13, 2^9 <= N / split_degree and 16-byte
 * aligned buffers (one CTA per row); otherwise four launches with engine scratch.
 * Replaces the chain polynomial_RNSc_to_RNS x2, polynomial_mul_RNS_polynomial,
 * polynomial_RNS_to_RNSc (rns_polynomial.c:311-356, 582-614). */
int vfhe_cuda_ntt_mul_intt_batch(void *ntt, uint64_t *d_out, const uint64_t *d_a, const uint64_t *d_b,
                                 uint64_t batch, const uint32_t *limbs, uint32_t nlimbs, void *stream);

/* Same result as vfhe_cuda_ntt_mul_intt_batch, for callers that cannot let a library
 * allocate GPU memory: code building a CUDA graph by stream capture, host runtimes
 * (a JVM or Go service, say) that own the device memory through their own allocator,
 * and serving loops that cannot afford an allocation's device synchronisation.  It
 * calls no cudaMalloc, cudaFree or other allocating routine: its scratch is a static
 * device array of 2^20 residues (8 MiB) inside the library, which every GPU that loads
 * the library holds until the process exits.  batch * nlimbs * N must not exceed 2^20;
 * larger requests are rejected (nonzero return, vfhe_cuda_last_error says why).  The
 * first call on a device resolves the array's device address on that device, so make
 * it before any stream capture.  All calls share the one array: calls whose work
 * overlaps on the GPU (different streams, or a second call before the first has
 * finished on another stream) race on it.  Call with the engine's device current.
 * No counterpart in the reference. */
int vfhe_cuda_ntt_mul_intt_batch_noalloc(void *ntt, uint64_t *d_out, const uint64_t *d_a, const uint64_t *d_b,
                                         uint64_t batch, const uint32_t *limbs, uint32_t nlimbs, void *stream);

/* CKKS evaluation over device-resident ciphertexts.
 *
 * A ciphertext at level with L active limbs is [2][L][N] uint64: component 0 is a,
 * component 1 is b.  limbs[0..L) are the pool indices of the ciphertext primes in
 * increasing order; `special` is the pool index of the special prime.  A key-switch
 * key for L digits is [L][2][L+1][N] in the NTT domain: digit j, component (a,b),
 * extended limbs (limbs[0..L) then `special`) -- the layout of
 * MLWE_Set(...)->obj[0][j] in the reference (modules/mlwe/python/src/vfhe/mlwe/mlwe.py:145-177).
 *
 * vfhe_cuda_ckks_mul_relin_rescale_batch: d_out[i] = rescale(relin(d_ct1[i] x d_ct2[i]))
 * for NTT-domain inputs, coefficient-domain outputs [2][L-1][N]; equal to
 * CKKS_Ciphertext.__mul__ (ckks.py:227-241): mlwe_multiply (mlwe.c:711-760) then
 * the round division of the top prime (mlwe.c:762-772).
 *
 * vfhe_cuda_ckks_rotate_batch: d_out[i] = automorphism(d_ct[i], gens[i]) key-switched
 * with the key at d_gks[i], coefficient domain in and out [2][L][N]
 * (mlwe_automorphism_RNSc_GHS, mlwe.c:314-326).  gens and d_gks are host arrays of
 * `batch` entries (Galois elements, device key pointers).
 *
 * Scratch comes from `workspace` (device memory of at least the size returned by the
 * matching *_workspace_bytes call); pass NULL to let the engine allocate it.  Engine-
 * owned scratch is one buffer per stream, shared by every NULL-workspace call and every
 * vfhe_cuda_ntt_mul_intt_batch call on that stream (stream order keeps them apart);
 * calls on different streams use different buffers.  Growing a stream's buffer
 * synchronises that stream. */
uint64_t vfhe_cuda_ckks_mul_workspace_bytes(void *ntt, uint64_t batch, uint32_t nlimbs);
int vfhe_cuda_ckks_mul_relin_rescale_batch(void *ntt, uint64_t *d_out, const uint64_t *d_ct1,
                                           const uint64_t *d_ct2, uint64_t batch,
                                           const uint32_t *limbs, uint32_t nlimbs, uint32_t special,
                                           const uint64_t *d_rlk, void *workspace, void *stream);
uint64_t vfhe_cuda_ckks_rotate_workspace_bytes(void *ntt, uint64_t batch, uint32_t nlimbs);
int vfhe_cuda_ckks_rotate_batch(void *ntt, uint64_t *d_out, const uint64_t *d_ct, uint64_t batch,
                                const uint32_t *limbs, uint32_t nlimbs, uint32_t special,
                                const uint64_t *gens, const uint64_t *const *d_gks, void *workspace,
                                void *stream);

/* Batched rank-1 MLWE (RLWE / CKKS) encryption on the GPU, the batched form of
 * mlwe_RNSc_sample (modules/mlwe/c/src/mlwe.c:190-241, reached from
 * CKKS_Scheme.encrypt, modules/fhe/python/src/vfhe/fhe/ckks.py:100-104):
 *   d_out [batch][2][L][N]  coefficient domain: a uniform, b = a s + e + m
 *   d_msg [batch][L][N]     coefficient-domain plaintexts (NULL: encryptions of zero)
 *   d_sk  [L][N]            the secret key limbs in the NTT domain (MLWE_Key.s_RNS)
 * e is a rounded Gaussian of width sigma per coefficient, the same integer in every
 * limb, as polynomial_gen_gaussian_RNSc_polynomial (rns_polynomial.c:255-271).
 * Randomness: the engine's ChaCha20 stream (RFC 8439 block function; keyed from
 * /dev/urandom, or by vfhe_prng_set_deterministic_seed), so outputs match the
 * reference's in distribution, not bit for bit.  1 <= batch * nlimbs <= 65535. */
int vfhe_cuda_rlwe_encrypt_batch(void *ntt, uint64_t *d_out, const uint64_t *d_msg, uint64_t batch,
                                 const uint32_t *limbs, uint32_t nlimbs, const uint64_t *d_sk,
                                 double sigma, void *stream);

/* Key-switching keys generated on the GPU, the batched _gen_ksk_components
 * (modules/mlwe/python/src/vfhe/mlwe/mlwe.py:145-177) behind gen_rlk / gen_ksk /
 * gen_ksk_automorphism: for each of the nsrc source polynomials j and each of the
 * L extended limbs i, digit j L + i is an RLWE encryption under d_sk of
 * src_j (P mod q_i) e_i, written in the NTT domain:
 *   d_out [nsrc * L][2][L][N]   the key tensor layout of the batched CKKS calls
 *   d_src [nsrc][L][N]          source polynomials in the NTT domain (e.g. -s^2, or
 *                               the permuted key for a Galois key)
 *   factors[L]                  host array: P mod q_i (P = product of special primes)
 *   d_sk  [L][N]                the output key's secret limbs, NTT domain
 * Limbs are the extended (special) ring's.  1 <= nsrc * L * L <= 65535. */
int vfhe_cuda_gen_ksk_batch(void *ntt, uint64_t *d_out, const uint64_t *d_src, uint64_t nsrc,
                            const uint32_t *limbs, uint32_t nlimbs, const uint64_t *factors,
                            const uint64_t *d_sk, double sigma, void *stream);

/* Compact wire format for residue rows, for host <-> device copies of ciphertexts:
 * each row of N residues of a b-bit prime (b = bits[r], residues < 2^b) is a
 * little-endian bit stream of N b bits (N b a multiple of 64); an item (e.g. one
 * ciphertext [2][L][N], rows_per_item = 2 L) is its rows in order, items follow each
 * other.  pack: d_rows [items][rows_per_item][N] uint64 -> d_packed; unpack: back.
 * packed_bytes: size of `items` packed items.  1 <= items * rows_per_item <= 65535,
 * rows_per_item <= 128.  No counterpart in the reference (it has no serialisation). */
uint64_t vfhe_cuda_packed_bytes(uint64_t N, const uint32_t *bits, uint32_t rows_per_item, uint64_t items);
int vfhe_cuda_pack_rows(void *d_packed, const uint64_t *d_rows, uint64_t N, const uint32_t *bits,
                        uint32_t rows_per_item, uint64_t items, void *stream);
int vfhe_cuda_unpack_rows(uint64_t *d_rows, const void *d_packed, uint64_t N, const uint32_t *bits,
                          uint32_t rows_per_item, uint64_t items, void *stream);
/* The same format packed and unpacked on the host, for a sender that holds plain uint64
 * rows (h_rows, h_packed: host memory, pinned or not), on nthreads host threads (0 =
 * every hardware thread); synchronous, no GPU needed.  Byte for byte what
 * vfhe_cuda_pack_rows writes and vfhe_cuda_unpack_rows reads.  No counterpart in the
 * reference. */
int vfhe_cuda_pack_rows_host(void *h_packed, const uint64_t *h_rows, uint64_t N, const uint32_t *bits,
                             uint32_t rows_per_item, uint64_t items, uint32_t nthreads);
int vfhe_cuda_unpack_rows_host(uint64_t *h_rows, const void *h_packed, uint64_t N, const uint32_t *bits,
                               uint32_t rows_per_item, uint64_t items, uint32_t nthreads);

/* ChaCha20 keystream blocks counter0 .. counter0 + nblocks - 1 for a 256-bit key
 * (8 little-endian words) and a 64-bit nonce, in the original layout (64-bit block
 * counter in state words 12-13, nonce in 14-15), into d_out[nblocks][16] words: the
 * generator every sampling kernel of the engine uses.  No counterpart in the reference
 * (its generators are AES-CTR and BLAKE3, modules/misc/c/src/prng.c:91-137). */
int vfhe_cuda_prng_blocks(uint32_t *d_out, uint64_t nblocks, const uint32_t *key, uint64_t counter0,
                          uint64_t nonce, void *stream);

/* Batched CGGI16 functional bootstrap with the RNS gadget (CGGI16.functional_bootstrap,
 * modules/fhe/python/src/vfhe/fhe/cggi16.py:46-128, over mgsw_CMUX, mgsw.c:52-72).
 * `batch` LWE ciphertexts of dimension n over the L0 (1 or 2) primes limbs[] are
 * blind-rotated through one bootstrapping key and sample-extracted at coefficient 0.
 *   d_in_a  [batch][L0][n]   LWE masks      d_in_b  [batch][L0]  LWE bodies
 *   d_bk    [n][2*L0][2][L0+1][N]  MGSW of each secret coefficient, NTT domain, in the
 *           order of MGSW_Scheme.encrypt (mgsw.py:18-55): L0 digits of the a row, then L0
 *           of the b row; extended limbs = limbs[] then `special`
 *   d_tv    [2][L0][N]       LUT test vector (rank-1 MLWE), coefficient domain
 *   d_out_a [batch][L0][N]   extracted masks; d_out_b [batch][L0] extracted bodies.
 * torus_base is the LUT size t (rot_b uses floor(Q / 4t), cggi16.py:65).  The n
 * rotation steps run as one CUDA graph, captured at the first call per shape. */
uint64_t vfhe_cuda_cggi_workspace_bytes(void *ntt, uint64_t batch, uint32_t n, uint32_t nlimbs);
int vfhe_cuda_cggi_bootstrap_batch(void *ntt, uint64_t *d_out_a, uint64_t *d_out_b, const uint64_t *d_in_a,
                                   const uint64_t *d_in_b, uint64_t batch, uint32_t n, const uint32_t *limbs,
                                   uint32_t nlimbs, uint32_t special, const uint64_t *d_bk, const uint64_t *d_tv,
                                   uint64_t torus_base, void *workspace, void *stream);

/* Batched GHS key switch of rank-1 samples with one key (mlwe_RNSc_GHS_hybrid_keyswitch,
 * mlwe.c:557-598, with a single key component): for each [2][L][N] coefficient-domain
 * sample (a, b), d_out = (moddown(-sum_j d_j K_j.a), b + moddown(-sum_j d_j K_j.b)),
 * d_j = limb j of a lifted to limbs[] + special.  Key layout as for the CKKS calls. */
uint64_t vfhe_cuda_keyswitch_workspace_bytes(void *ntt, uint64_t batch, uint32_t nlimbs);
int vfhe_cuda_keyswitch_batch(void *ntt, uint64_t *d_out, const uint64_t *d_ct, uint64_t batch,
                              const uint32_t *limbs, uint32_t nlimbs, uint32_t special, const uint64_t *d_ksk,
                              void *workspace, void *stream);

/* Transform launch schedule for one (log2 P, floor(log2 rows-per-launch)) class, as
 * picked by the autotuner: tile_bits (P-point rows are split into a radix-2^(logP -
 * tile_bits) column pass and tiles of 2^tile_bits; == logP for one pass; 8..13),
 * tiles_per_cta (rows or row segments one CTA holds), ctas_per_sm (0: one CTA per tile
 * group; k: persistent grid of k CTAs per SM; -1: the row on a thread-block cluster of
 * 2^(logP - tile_bits) CTAs, tile_bits 11..13; -2: column pass and tile pass as one
 * dataflow launch, tile_bits 10..13 with logP - tile_bits 2..4, outside stream capture,
 * tiles_per_cta then giving the work items per ticket, 1 or 2 (0: two); the two kernels
 * otherwise).  Zero = built-in default.  Schedules
 * never change results.  get_schedule writes the three fields for a launch of `rows`
 * rows.  No counterpart in the reference (its transforms are single-threaded loops). */
int vfhe_cuda_ntt_set_schedule(uint32_t logP, uint32_t rows_log2, int32_t tile_bits, int32_t tiles_per_cta,
                               int32_t ctas_per_sm);
int vfhe_cuda_ntt_get_schedule(uint32_t logP, uint64_t rows, int32_t *out3);

/* Nonzero when a kernel's bounded wait gave up (for a bulk copy in a persistent
 * transform or the staged key-switch MAC, for a grid barrier of the persistent work
 * list, or for the first pass of a dataflow transform; its results are then wrong);
 * -1 when the flags cannot be read.  Stays 0 in normal operation. */
int vfhe_cuda_device_faults(void);

/* Reset the flags vfhe_cuda_device_faults reads.  0 on success. */
int vfhe_cuda_clear_device_faults(void);

/* Self-check of the bounded-wait machinery (no reference counterpart): runs a one-thread
 * kernel that waits, at most `tries` attempts, on an mbarrier that no copy completes.
 * The wait must give up, raise the flag vfhe_cuda_device_faults reads, and return with
 * the context usable.  Returns 1 when it gave up as designed, 0 if it did not, -1 on a
 * CUDA error.  Clear the flag afterwards with vfhe_cuda_clear_device_faults. */
int vfhe_cuda_selfcheck_bounded_wait(int32_t tries);

/* Work list: independent jobs of any mix of ring degree and limb count, run together.
 * Mode 0 (default): when every job has 2^8 <= N/split <= 2^16 and split <= 4, a run is
 * three persistent cooperative kernels whose CTAs walk six phases (forward column
 * passes | forward tile passes; products and key multiply-accumulates; inverse tile
 * passes | inverse column passes | special-prime divisions) over the device-resident
 * row tables of every transform pool, with a bounded grid barrier between the phases of
 * a kernel (a barrier that gives up raises the flag vfhe_cuda_device_faults reads).
 * Mode 1, and mode 0 for other shapes: a CUDA graph with one launch per stage per
 * transform pool.  Jobs:
 *   chain      d_out = INTT(NTT(d_a) * NTT(d_b)), [nlimbs][N] each (as
 *              vfhe_cuda_ntt_mul_intt_batch with batch 1);
 *   keyswitch  as vfhe_cuda_keyswitch_batch with batch 1 (d_ct [2][nlimbs][N],
 *              d_out [2][nlimbs][N], d_ksk [nlimbs][2][nlimbs+1][N]).
 * All primes below 2^50, rows 16-byte aligned, 2^8 <= N/split <= 2^17.  compile (or
 * the first run) allocates the work list's scratch and tables and captures the graph;
 * run replays it on `stream`.  The job buffers must stay allocated at the same
 * addresses while the work list is used; adding a job drops the compiled graph.
 * No counterpart in the reference. */
void *vfhe_cuda_worklist_new(void);
void vfhe_cuda_worklist_free(void *wl);
int vfhe_cuda_worklist_add_chain(void *wl, void *ntt, uint64_t *d_out, const uint64_t *d_a, const uint64_t *d_b,
                                 const uint32_t *limbs, uint32_t nlimbs);
int vfhe_cuda_worklist_add_keyswitch(void *wl, void *ntt, uint64_t *d_out, const uint64_t *d_ct,
                                     const uint32_t *limbs, uint32_t nlimbs, uint32_t special, const uint64_t *d_ksk);
int vfhe_cuda_worklist_compile(void *wl);
int vfhe_cuda_worklist_run(void *wl, void *stream);
uint64_t vfhe_cuda_worklist_device_bytes(void *wl);
int vfhe_cuda_worklist_launches(void *wl);
int vfhe_cuda_worklist_set_mode(void *wl, int mode);
int vfhe_cuda_worklist_is_persistent(void *wl);
/* Persistent path: wall time (ms, device global timer, seen by CTA 0 at the grid
 * barriers) of the last run's six phases -- forward column, forward tile, products and
 * MACs (with the launch gap before it), inverse tile (with its launch gap), inverse
 * column, divisions.  1 when not on the persistent path. */
int vfhe_cuda_worklist_phase_ms(void *wl, double *out6);

/* CGGI over the 32-bit torus with FP64 FFT external products (the TFHE bootstrap,
 * Chillotti et al., J. Cryptology 33, 2020, with the reference's CGGI16 blind-rotation
 * orchestration, cggi16.py:46-128).  Torus values are uint32; a rank-1 GLWE (a, b) of
 * degree N (512, 1024 or 2048) has phase b - a S; gadget: base 2^base_log, `levels`
 * levels (<= 4), signed digits.  No counterpart in the reference: its CGGI16 uses the
 * RNS gadget (vfhe_cuda_cggi_bootstrap_batch above) and its LWE key switch is a stub.
 *
 * to_fourier: spectra d_out [count][N/2] complex doubles (re, im) of rows
 *   d_rows [count][N] read as signed 32-bit coefficients (bootstrapping-key rows).
 * bootstrap_batch: d_in [batch][n+1] LWEs (mask, body) -> d_out [batch][N+1]
 *   extracted LWEs; d_bsk_f [n][2 levels][2][N/2] spectra of GGSW(s_i), row (c, l) at
 *   c * levels + l; d_tv [N] test vector; rotation offset 2^32 / (4 torus_base).
 *   One persistent launch: every CTA runs whole blind rotations with its accumulator
 *   in shared memory.
 * keyswitch_batch: d_in [batch][N+1] -> d_out [batch][n+1] with d_ksk [N][levels][n+1]
 *   (base 2^base_log, signed digits); exact integer arithmetic.
 * external_product: d_out[b] = ExtProd(GGSW spectra d_ggsw_f, GLWE d_c[b] [2][N]) rounded
 *   to integers, and d_frac[b] = the largest distance of an unrounded coefficient to its
 *   integer (NULL to skip), for measuring the FFT error against exact products. */
int vfhe_cuda_cggi_fft_to_fourier(double *d_out, const uint32_t *d_rows, uint64_t count, uint32_t N, void *stream);
int vfhe_cuda_cggi_fft_bootstrap_batch(uint32_t *d_out, const uint32_t *d_in, uint64_t batch, const double *d_bsk_f,
                                       const uint32_t *d_tv, uint32_t n, uint32_t N, uint32_t base_log,
                                       uint32_t levels, uint32_t torus_base, void *stream);
int vfhe_cuda_cggi_fft_keyswitch_batch(uint32_t *d_out, const uint32_t *d_in, uint64_t batch, const uint32_t *d_ksk,
                                       uint32_t N, uint32_t n, uint32_t base_log, uint32_t levels, void *stream);
int vfhe_cuda_cggi_fft_external_product(uint32_t *d_out, const uint32_t *d_c, uint64_t batch, const double *d_ggsw_f,
                                        uint32_t N, uint32_t base_log, uint32_t levels, double *d_frac,
                                        void *stream);
/* Torus keys generated on the GPU from the caller's secret keys d_s [n], d_S [N] (small
 * signed int32, e.g. binary): d_bsk_rows [n][2 bs_levels][2][N] uint32, row (i, c levels
 * + l) = GLWE_S(0) with s_i 2^(32 - bs_base_log (l + 1)) added to coefficient 0 of
 * component c (GGSW(s_i); to_fourier gives the spectra bootstrap_batch reads), and
 * d_ksk [N][ks_levels][n+1] uint32, row (j, l) = LWE_s(S_j 2^(32 - ks_base_log (l + 1))).
 * Masks uniform, noise rounded Gaussians of width sigma 2^32 (lwe_sigma for the key
 * switch, glwe_sigma for the bootstrapping key), drawn from the engine's ChaCha20
 * stream.  The layout is TorusKeys.generate's in vfhe_b200/cggi_fft.py. */
int vfhe_cuda_cggi_fft_gen_keys(uint32_t *d_bsk_rows, uint32_t *d_ksk, const int32_t *d_s, const int32_t *d_S,
                                uint32_t n, uint32_t N, uint32_t bs_base_log, uint32_t bs_levels,
                                uint32_t ks_base_log, uint32_t ks_levels, double lwe_sigma, double glwe_sigma,
                                void *stream);

/* Evaluation-key files (no counterpart in the reference, which keeps keys in process
 * memory only): a versioned 656-byte header (magic "VFHEKEY", format version 1, kind,
 * element size, shape, the moduli of the limb axis, kind-specific aux words, payload
 * size, FNV-1a-64 checksum of the payload over 64-bit words) followed by the key tensor
 * in row-major order.  Host buffers only (no GPU needed); the byte layout is spelled
 * out in vfhe_b200/csrc/keyfile.cu.  Kinds and shapes:
 *   VFHE_KEY_KSK        key-switching key (rlk / Galois), u64 [D][2][L+1][N], NTT domain;
 *                       aux[0] Galois element (0: relinearisation), aux[1] level
 *   VFHE_KEY_MGSW_BSK   RNS CGGI16 bootstrapping key, u64 [n][2 L0][2][L0+1][N], NTT domain
 *   VFHE_KEY_TORUS_BSK  torus bootstrapping-key rows, u32 [n][2 levels][2][N];
 *                       aux[0] base_log, aux[1] levels
 *   VFHE_KEY_TORUS_KSK  torus key-switching key, u32 [N][levels][n+1]; aux as above
 * write: 0 on success.  read_header: fills hdr from the file.  read: validates the
 * header, the payload size and the checksum, fills hdr and host_data (capacity_bytes
 * at least payload_bytes(hdr)); 1 on any mismatch, with the reason in last_error. */
enum {
    VFHE_KEY_KSK = 1,
    VFHE_KEY_MGSW_BSK = 2,
    VFHE_KEY_TORUS_BSK = 3,
    VFHE_KEY_TORUS_KSK = 4
};
typedef struct VfheKeyHeader {
    uint32_t kind;
    uint32_t elem_bytes;
    uint32_t ndims;
    uint32_t nmoduli;
    uint64_t dims[8];
    uint64_t aux[4];
    uint64_t moduli[64];
} VfheKeyHeader;
uint64_t vfhe_cuda_keyfile_payload_bytes(const VfheKeyHeader *hdr);
int vfhe_cuda_keyfile_write(const char *path, const VfheKeyHeader *hdr, const void *host_data);
int vfhe_cuda_keyfile_read_header(const char *path, VfheKeyHeader *hdr);
int vfhe_cuda_keyfile_read(const char *path, VfheKeyHeader *hdr, void *host_data, uint64_t capacity_bytes);

/* Serving loop (continuous batching on one GPU).  Requests name device-resident
 * ciphertexts and keys; a native worker thread queues them per (operation, class),
 * starts a batch whenever one of `nstreams` stream slots is free and the batch's
 * scratch fits the HBM budget left (up to max_batch requests; CGGI requests merge up
 * to the class's max_count ciphertexts), gathers inputs with device-to-device copies
 * into stream-ordered scratch, runs one batched call, scatters the outputs and records
 * a completion event.  Requests arriving meanwhile join the next batches.  CKKS
 * ciphertext pointers must be 16-byte aligned.  reserve grows the server's memory
 * pool ahead of time.  Latency =
 * submission to observed completion (host steady clock).  max_batch = 1 with one
 * stream is the plain one-call-per-request path.  Inputs must be complete on the
 * device when submitted; outputs are complete when wait returns.  Results equal the
 * batched entry points' (vfhe_cuda_ckks_mul_relin_rescale_batch, _rotate_batch,
 * vfhe_cuda_cggi_bootstrap_batch) for every request, alone or mixed.  The worker
 * is the only thread that may launch engine work while the server runs.
 * No counterpart in the reference. */
void *vfhe_cuda_server_new(uint64_t hbm_budget_bytes, uint32_t nstreams, uint32_t max_batch);
void vfhe_cuda_server_free(void *server);
int vfhe_cuda_server_note_resident(void *server, uint64_t bytes);
int vfhe_cuda_server_reserve(void *server, uint64_t bytes);
int vfhe_cuda_server_ckks_class(void *server, void *ntt, const uint32_t *limbs, uint32_t nlimbs, uint32_t special,
                                const uint64_t *d_rlk);
int vfhe_cuda_server_cggi_class(void *server, void *ntt, const uint32_t *limbs, uint32_t nlimbs, uint32_t special,
                                uint32_t n, const uint64_t *d_bk, const uint64_t *d_tv, uint64_t torus_base,
                                uint32_t max_count);
int64_t vfhe_cuda_server_submit_ckks_mul(void *server, int cls, uint64_t *d_out, const uint64_t *d_ct1,
                                         const uint64_t *d_ct2);
int64_t vfhe_cuda_server_submit_ckks_rotate(void *server, int cls, uint64_t *d_out, const uint64_t *d_ct,
                                            uint64_t gen, const uint64_t *d_gk);
int64_t vfhe_cuda_server_submit_cggi(void *server, int cls, uint64_t *d_out_a, uint64_t *d_out_b,
                                     const uint64_t *d_in_a, const uint64_t *d_in_b, uint64_t count);
/* Torus CGGI classes (the FP64-FFT programmable bootstrap with the key switch back to
 * the input key; vfhe_cuda_cggi_fft_bootstrap_batch + _keyswitch_batch): keys are
 * device-resident (spectra, LUT test vector, key-switching key), requests carry
 * `count` uint32 LWEs [count][n+1] in and out.  Class ids share the CGGI list. */
int vfhe_cuda_server_torus_class(void *server, const double *d_bsk_f, const uint32_t *d_tv,
                                 const uint32_t *d_ksk, uint32_t n, uint32_t N, uint32_t bs_base_log,
                                 uint32_t bs_levels, uint32_t ks_base_log, uint32_t ks_levels,
                                 uint32_t torus_base, uint32_t max_count);
int64_t vfhe_cuda_server_submit_torus(void *server, int cls, uint32_t *d_out, const uint32_t *d_in,
                                      uint64_t count);
int vfhe_cuda_server_wait(void *server, int64_t id, double *latency_ms);
int vfhe_cuda_server_stats(void *server, uint64_t *out5);
/* Failure handling (no counterpart in the reference).
 * wait_for: wait at most timeout_ms (< 0: no limit); 0 done, 1 failed or unknown id,
 *   2 time ran out (the request is kept), 3 cancelled.  wait = wait_for without limit.
 * cancel: drop a request no batch has taken yet; 0 cancelled, 1 already running or
 *   finished (it completes normally), -1 unknown id.
 * pause: hold (1) or resume (0) admission of queued requests into batches.
 * set_batch_timeout: the requests of a batch still running after timeout_ms fail; the
 *   batch's stream and scratch are released once its device work has finished.
 * inject_fault (tests; host-side only, no GPU fault): kind 1 the next `count` batch
 *   launches fail, kind 2 the next `count` scratch allocations fail (the batch is
 *   re-queued and retried), kind 3 the next `count` batches' completions go unobserved
 *   until the batch deadline.
 * fault_stats: out[0] batches failed by the deadline, out[1] allocation retries,
 *   out[2] cancelled requests, out[3] injected faults not yet consumed. */
int vfhe_cuda_server_wait_for(void *server, int64_t id, double timeout_ms, double *latency_ms);
int vfhe_cuda_server_cancel(void *server, int64_t id);
int vfhe_cuda_server_pause(void *server, int paused);
int vfhe_cuda_server_set_batch_timeout(void *server, double timeout_ms);
int vfhe_cuda_server_inject_fault(void *server, int kind, uint32_t count);
int vfhe_cuda_server_fault_stats(void *server, uint64_t *out4);

#ifdef __cplusplus
}
#endif

#endif /* VFHE_CUDA_H */
