/*
 * vfhe_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A scalar, unsigned __int128 restatement of the vfhe reference's RNS hot path,
 * used as the correctness checker for the cuda engine.  Only tests, the smoke entry
 * point and bench.py's CPU-baseline leg load it; the engine never does.
 *
 * It exports the subset of the reference cdef surface that the hot path needs
 * (same names and struct prefixes, so the same Python orchestration drives the cuda
 * engine, this oracle and the reference library built under oracle/_ref/).  Each
 * function cites the reference lines whose behaviour it restates.  Arithmetic is
 * exact modular arithmetic on canonical residues; there is no random sampling here
 * (tests inject seeded inputs).
 *
 * Parity pins: tests/test_golden.py and tests/test_oracle_arith.py check this oracle against the golden vectors in
 * tests/golden/ (made by running the reference built from its own sources) and
 * against the reference library itself when it is present.
 */
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ structs */
/* public prefixes: modules/arith/c/include/arith.h:29-78, mlwe/c/include/mlwe.h:20-49 */
typedef struct _NTT_proc {
    uint64_t n, q, root, inv_root;
    uint64_t *fwd; /* fwd[brv(i)] = psi^i   (ntt_portable.c:18-39) */
    uint64_t *inv; /* inv[brv(i)] = psi^-i  (ntt_portable.c:41-62) */
    uint64_t n_inv;
} *NTT_proc;

typedef struct _incNTT {
    NTT_proc *ntt;
    uint64_t split_degree;
    uint64_t **w;
    uint64_t N, l;
} *incNTT;

typedef struct _RNS_Polynomial {
    uint64_t **coeffs;
    incNTT ntt;
    uint64_t rns_mask, allocated_l;
} *RNS_Polynomial;

typedef struct _RNS_MLWE {
    RNS_Polynomial *a, b;
    uint64_t r;
} *RNS_MLWE;

typedef struct _IntPolynomial {
    uint64_t *coeffs;
    uint64_t N;
} *IntPolynomial;

typedef struct _RNS_MLWE_Key {
    IntPolynomial *s;
    RNS_Polynomial *s_RNS;
    uint64_t N, l, r;
    double sigma;
} *RNS_MLWE_Key;

typedef struct _LWE_Key {
    uint64_t **s;
    uint64_t n, l;
    incNTT ntt;
    double sigma;
} *LWE_Key;

typedef struct _LWE {
    uint64_t **a;
    uint64_t *b;
    uint64_t n, l;
    incNTT ntt;
} *LWE;

/* ------------------------------------------------------------------ scalar mod */
static uint64_t mulm(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
static uint64_t addm(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a + b) % q); }
static uint64_t subm(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a + q - (b % q)) % q); }
static uint64_t negm(uint64_t a, uint64_t q) { return (q - a % q) % q; }
static uint64_t powm(uint64_t b, uint64_t e, uint64_t q)
{
    uint64_t r = 1 % q;
    b %= q;
    for (; e; e >>= 1, b = mulm(b, b, q))
        if (e & 1) r = mulm(r, b, q);
    return r;
}
static uint64_t invm(uint64_t a, uint64_t q) { return powm(a % q, q - 2, q); } /* q prime */
/* signed 64-bit to residue (mod_portable.c:120-137) */
static uint64_t sredm(uint64_t v, uint64_t q)
{
    if (v >> 63) {
        uint64_t r = (0 - v) % q;
        return r ? q - r : 0;
    }
    return v % q;
}
static uint64_t brv(uint64_t x, int bits)
{
    uint64_t r = 0;
    for (int i = 0; i < bits; i++, x >>= 1) r = (r << 1) | (x & 1);
    return r;
}
static int ilog2(uint64_t n)
{
    int l = 0;
    while ((1ULL << l) < n) l++;
    return l;
}
static uint64_t mask_bit(uint64_t m, uint64_t i) { return i < 64 ? (m >> i) & 1 : 0; }

/* ------------------------------------------------------------------ NTT */
/* root: first g = 2, 3, ... with g^((q-1)/2n) of order exactly 2n (ntt_portable.c:137-154) */
static NTT_proc proc_new(uint64_t n, uint64_t q)
{
    NTT_proc p = (NTT_proc)calloc(1, sizeof(*p));
    p->n = n;
    p->q = q;
    for (uint64_t g = 2; g < q; g++) {
        uint64_t c = powm(g, (q - 1) / (2 * n), q);
        if (powm(c, n, q) == q - 1) {
            p->root = c;
            break;
        }
    }
    p->inv_root = invm(p->root, q);
    int logn = ilog2(n);
    p->fwd = (uint64_t *)malloc(n * 8);
    p->inv = (uint64_t *)malloc(n * 8);
    uint64_t f = 1, iv = 1;
    for (uint64_t i = 0; i < n; i++) {
        p->fwd[brv(i, logn)] = f;
        p->inv[brv(i, logn)] = iv;
        f = mulm(f, p->root, q);
        iv = mulm(iv, p->inv_root, q);
    }
    p->n_inv = invm(n % q, q);
    return p;
}

/* forward: CT, natural -> bit-reversed (ntt_portable.c:76-100) */
static void ntt_fwd(uint64_t *a, NTT_proc p)
{
    const uint64_t n = p->n, q = p->q;
    for (uint64_t m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1)
        for (uint64_t i = 0; i < m; i++) {
            const uint64_t w = p->fwd[m + i];
            for (uint64_t j = 2 * i * t; j < 2 * i * t + t; j++) {
                const uint64_t u = a[j], v = mulm(a[j + t], w, q);
                a[j] = addm(u, v, q);
                a[j + t] = subm(u, v, q);
            }
        }
}

/* inverse: GS, bit-reversed -> natural, times n^-1 (ntt_portable.c:102-135) */
static void ntt_inv(uint64_t *a, NTT_proc p)
{
    const uint64_t n = p->n, q = p->q;
    for (uint64_t h = n >> 1, t = 1; h >= 1; h >>= 1, t <<= 1) {
        for (uint64_t i = 0; i < h; i++) {
            const uint64_t w = p->inv[h + i];
            for (uint64_t j = 2 * i * t; j < 2 * i * t + t; j++) {
                const uint64_t u = a[j], v = a[j + t];
                a[j] = addm(u, v, q);
                a[j + t] = mulm(subm(u, v, q), w, q);
            }
        }
        if (h == 1) break;
    }
    for (uint64_t i = 0; i < n; i++) a[i] = mulm(a[i], p->n_inv, q);
}

/* ------------------------------------------------------------------ pool */
/* twist w[k] = psi^(2 brv(k) + 1) (rns_polynomial.c:7-31, misc.c:186-192) */
static void pool_add(incNTT t, uint64_t q)
{
    const uint64_t P = t->N / t->split_degree;
    const uint64_t i = t->l;
    t->ntt = (NTT_proc *)realloc(t->ntt, (i + 1) * sizeof(NTT_proc));
    t->w = (uint64_t **)realloc(t->w, (i + 1) * sizeof(uint64_t *));
    t->ntt[i] = proc_new(P, q);
    t->w[i] = (uint64_t *)malloc(P * 8);
    const int logP = ilog2(P);
    for (uint64_t k = 0; k < P; k++) t->w[i][k] = powm(t->ntt[i]->root, 2 * brv(k, logP) + 1, q);
    t->l = i + 1;
}

void *new_incomplete_ntt_list(uint64_t *primes, uint64_t split_degree, uint64_t N, uint64_t count)
{
    incNTT t = (incNTT)calloc(1, sizeof(*t));
    t->N = N;
    t->split_degree = split_degree;
    for (uint64_t i = 0; i < count; i++) pool_add(t, primes[i]);
    return t;
}

void incNTT_extend_with_primes(void *ntt, uint64_t *new_primes, uint64_t count)
{
    for (uint64_t i = 0; i < count; i++) pool_add((incNTT)ntt, new_primes[i]);
}

uint64_t **incNTT_get_rou_matrix(void *ntt) { return ((incNTT)ntt)->w; }

const char *vfhe_engine_active(void) { return "oracle"; }

void *safe_aligned_malloc(uint64_t size)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, size ? size : 64)) return NULL;
    return p;
}

/* ------------------------------------------------------------------ polynomials */
#define NL(p) ((p)->ntt->l < (p)->allocated_l ? (p)->ntt->l : (p)->allocated_l)
#define Q(p, i) ((p)->ntt->ntt[i]->q)
#define ACTIVE(p, i) mask_bit((p)->rns_mask, (i))

void *polynomial_new_RNS_polynomial(uint64_t N, uint64_t rns_mask, void *ntt)
{
    (void)N;
    incNTT t = (incNTT)ntt;
    RNS_Polynomial p = (RNS_Polynomial)calloc(1, sizeof(*p));
    p->coeffs = (uint64_t **)malloc((t->l ? t->l : 1) * sizeof(uint64_t *));
    for (uint64_t i = 0; i < t->l; i++) p->coeffs[i] = (uint64_t *)calloc(t->N, 8);
    p->ntt = t;
    p->rns_mask = rns_mask;
    p->allocated_l = t->l;
    return p;
}

void free_RNS_polynomial(void *pp)
{
    RNS_Polynomial p = (RNS_Polynomial)pp;
    if (!p) return;
    for (uint64_t i = 0; i < p->allocated_l; i++) free(p->coeffs[i]);
    free(p->coeffs);
    free(p);
}

void polynomial_copy_RNS_polynomial(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out, s = (RNS_Polynomial)in;
    o->rns_mask = s->rns_mask;
    if (o == s) return;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i)) memcpy(o->coeffs[i], s->coeffs[i], o->ntt->N * 8);
}

void polynomial_RNSc_to_RNS(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out, s = (RNS_Polynomial)in;
    o->rns_mask = s->rns_mask;
    const uint64_t P = o->ntt->N / o->ntt->split_degree;
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!ACTIVE(o, i)) continue;
        if (o != s) memcpy(o->coeffs[i], s->coeffs[i], o->ntt->N * 8);
        for (uint64_t k = 0; k < o->ntt->split_degree; k++) ntt_fwd(o->coeffs[i] + k * P, o->ntt->ntt[i]);
    }
}

void polynomial_RNS_to_RNSc(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out, s = (RNS_Polynomial)in;
    o->rns_mask = s->rns_mask;
    const uint64_t P = o->ntt->N / o->ntt->split_degree;
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!ACTIVE(o, i)) continue;
        if (o != s) memcpy(o->coeffs[i], s->coeffs[i], o->ntt->N * 8);
        for (uint64_t k = 0; k < o->ntt->split_degree; k++) ntt_inv(o->coeffs[i] + k * P, o->ntt->ntt[i]);
    }
}

/* layout: coefficient j at (j mod s) * P + j / s (rns_polynomial.c:199-238) */
void int_array_to_RNS(void *out, uint64_t *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out;
    const uint64_t s = o->ntt->split_degree, P = o->ntt->N / s;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i))
            for (uint64_t j = 0; j < o->ntt->N; j++) o->coeffs[i][(j % s) * P + j / s] = sredm(in[j], Q(o, i));
    polynomial_RNSc_to_RNS(o, o);
}

void array_to_RNS(void *out, uint64_t **in)
{
    RNS_Polynomial o = (RNS_Polynomial)out;
    const uint64_t s = o->ntt->split_degree, P = o->ntt->N / s;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i))
            for (uint64_t j = 0; j < o->ntt->N; j++) o->coeffs[i][(j % s) * P + j / s] = in[i][j];
    polynomial_RNSc_to_RNS(o, o);
}

/* incomplete product (rns_polynomial.c:311-435): mode 0 set, 1 add, 2 subtract */
static void product(RNS_Polynomial o, RNS_Polynomial a, RNS_Polynomial b, int mode)
{
    const uint64_t s = o->ntt->split_degree, P = o->ntt->N / s, N = o->ntt->N;
    const uint64_t mask = a->rns_mask & b->rns_mask;
    o->rns_mask = mask;
    uint64_t *acc = (uint64_t *)malloc(N * 8);
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!mask_bit(mask, i)) continue;
        const uint64_t q = Q(o, i);
        memset(acc, 0, N * 8);
        for (uint64_t j = 0; j < s; j++)
            for (uint64_t k = 0; k < s; k++)
                for (uint64_t x = 0; x < P; x++) {
                    uint64_t v = mulm(a->coeffs[i][j * P + x], b->coeffs[i][k * P + x], q);
                    uint64_t dst = j + k;
                    if (dst >= s) {
                        v = mulm(v, o->ntt->w[i][x], q);
                        dst -= s;
                    }
                    acc[dst * P + x] = addm(acc[dst * P + x], v, q);
                }
        for (uint64_t e = 0; e < N; e++) {
            if (mode == 0) o->coeffs[i][e] = acc[e];
            else if (mode == 1) o->coeffs[i][e] = addm(o->coeffs[i][e], acc[e], q);
            else o->coeffs[i][e] = subm(o->coeffs[i][e], acc[e], q);
        }
    }
    free(acc);
}

void polynomial_mul_RNS_polynomial(void *out, void *in1, void *in2)
{
    product((RNS_Polynomial)out, (RNS_Polynomial)in1, (RNS_Polynomial)in2, 0);
}

void polynomial_multo_RNS_polynomial(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out;
    RNS_Polynomial tmp = (RNS_Polynomial)polynomial_new_RNS_polynomial(o->ntt->N, o->rns_mask, o->ntt);
    polynomial_copy_RNS_polynomial(tmp, o);
    product(o, (RNS_Polynomial)in, tmp, 0);
    free_RNS_polynomial(tmp);
}

static void binop(void *out, void *in1, void *in2, int sub)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in1, b = (RNS_Polynomial)in2;
    o->rns_mask = a->rns_mask & b->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i))
            for (uint64_t e = 0; e < o->ntt->N; e++)
                o->coeffs[i][e] = sub ? subm(a->coeffs[i][e], b->coeffs[i][e], Q(o, i))
                                      : addm(a->coeffs[i][e], b->coeffs[i][e], Q(o, i));
}

void polynomial_sub_RNS_polynomial(void *o, void *a, void *b) { binop(o, a, b, 1); }
void polynomial_sub_RNSc_polynomial(void *o, void *a, void *b) { binop(o, a, b, 1); }
void polynomial_add_RNS_polynomial(void *o, void *a, void *b) { binop(o, a, b, 0); }
void polynomial_add_RNSc_polynomial(void *o, void *a, void *b) { binop(o, a, b, 0); }

static void scale(RNS_Polynomial o, RNS_Polynomial a, const uint64_t *per, uint64_t uni)
{
    o->rns_mask = a->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i)) {
            const uint64_t q = Q(o, i), sc = (per ? per[i] : uni) % q;
            for (uint64_t e = 0; e < o->ntt->N; e++) o->coeffs[i][e] = mulm(a->coeffs[i][e], sc, q);
        }
}

void polynomial_scale_RNSc_polynomial(void *out, void *in1, uint64_t s)
{
    scale((RNS_Polynomial)out, (RNS_Polynomial)in1, NULL, s);
}
void polynomial_scale_RNS_polynomial_RNS(void *out, void *in1, uint64_t *s)
{
    scale((RNS_Polynomial)out, (RNS_Polynomial)in1, s, 0);
}

void polynomial_RNSc_negate(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    o->rns_mask = a->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i))
            for (uint64_t e = 0; e < o->ntt->N; e++) o->coeffs[i][e] = negm(a->coeffs[i][e], Q(o, i));
}

/* adds the integer to the first `count` residues (rns_polynomial.c:460-500) */
static void add_int(RNS_Polynomial o, RNS_Polynomial a, uint64_t v, uint64_t count)
{
    o->rns_mask = a->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i)) {
            if (o != a) memcpy(o->coeffs[i], a->coeffs[i], o->ntt->N * 8);
            const uint64_t r = sredm(v, Q(o, i));
            for (uint64_t e = 0; e < count; e++) o->coeffs[i][e] = addm(o->coeffs[i][e], r, Q(o, i));
        }
}

void polynomial_RNSc_add_integer(void *o, void *a, uint64_t v) { add_int(o, a, v, 1); }
void polynomial_RNS_add_integer(void *o, void *a, uint64_t v)
{
    RNS_Polynomial p = (RNS_Polynomial)o;
    add_int(p, a, v, p->ntt->N / p->ntt->split_degree);
}

/* x -> x^gen; coefficient c = i + i2 s at row position i P + i2 (rns_polynomial.c:996-1035) */
void polynomial_RNSc_permute(void *out, void *in, uint64_t gen)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    const uint64_t N = o->ntt->N, s = o->ntt->split_degree, P = N / s;
    o->rns_mask = a->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!ACTIVE(o, i)) {
            memset(o->coeffs[i], 0, N * 8);
            continue;
        }
        for (uint64_t c = 0; c < N; c++) {
            const uint64_t src = (c % s) * P + c / s;
            const uint64_t e = (c * gen) % (2 * N);
            const uint64_t d = e % N;
            const uint64_t v = a->coeffs[i][src];
            o->coeffs[i][(d % s) * P + d / s] = e >= N ? negm(v, Q(o, i)) : v;
        }
    }
}

void polynomial_RNSc_mod_reduce(void *out, void *in)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i) && o != a) memcpy(o->coeffs[i], a->coeffs[i], o->ntt->N * 8);
}

/* digit broadcast (rns_polynomial.c:824-843) */
void polynomial_RNSc_mod_reduce_lifted(void *out, void *in, uint64_t idx)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    uint64_t *src = (uint64_t *)malloc(o->ntt->N * 8);
    memcpy(src, a->coeffs[idx], o->ntt->N * 8);
    for (uint64_t i = 0; i < NL(o); i++)
        if (ACTIVE(o, i))
            for (uint64_t e = 0; e < o->ntt->N; e++) o->coeffs[i][e] = src[e] % Q(o, i);
    free(src);
}

/* sequential division by each prime of the mask (rns_polynomial.c:905-976) */
static void divide(RNS_Polynomial o, uint64_t dmask, int round)
{
    const uint64_t m = dmask & o->rns_mask;
    for (uint64_t d = 0; d < NL(o); d++) {
        if (!mask_bit(m, d)) continue;
        const uint64_t p = Q(o, d), half = round ? p / 2 : 0;
        for (uint64_t e = 0; e < o->ntt->N; e++) o->coeffs[d][e] = addm(o->coeffs[d][e], half, p);
        for (uint64_t i = 0; i < NL(o); i++) {
            if (i == d || !ACTIVE(o, i)) continue;
            const uint64_t q = Q(o, i), pinv = invm(p % q, q);
            for (uint64_t e = 0; e < o->ntt->N; e++) {
                uint64_t c = addm(o->coeffs[i][e], half % q, q);
                c = subm(c, o->coeffs[d][e] % q, q);
                o->coeffs[i][e] = mulm(c, pinv, q);
            }
        }
        memset(o->coeffs[d], 0, o->ntt->N * 8);
        o->rns_mask &= ~(1ULL << d);
    }
}

void polynomial_round_division_RNSc_wo_free(void *out, uint64_t m) { divide((RNS_Polynomial)out, m, 1); }
void polynomial_floor_division_RNSc_wo_free(void *out, uint64_t m) { divide((RNS_Polynomial)out, m, 0); }

/* rns_polynomial.c:1463-1525 */
void polynomial_RNSc_scaled_lift(void *out, void *in, uint64_t *delta)
{
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    const uint64_t diff = o->rns_mask & ~a->rns_mask;
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!ACTIVE(o, i)) continue;
        if (!ACTIVE(a, i)) {
            memset(o->coeffs[i], 0, o->ntt->N * 8);
            continue;
        }
        const uint64_t q = Q(o, i);
        uint64_t d = 1 % q;
        if (delta) d = delta[i] % q;
        else
            for (uint64_t j = 0; j < NL(o); j++)
                if (mask_bit(diff, j)) d = mulm(d, Q(o, j) % q, q);
        for (uint64_t e = 0; e < o->ntt->N; e++) o->coeffs[i][e] = mulm(a->coeffs[i][e], d, q);
    }
}

bool polynomial_eq(void *pa, void *pb)
{
    RNS_Polynomial a = (RNS_Polynomial)pa, b = (RNS_Polynomial)pb;
    const uint64_t l = a->ntt->l > b->ntt->l ? a->ntt->l : b->ntt->l;
    for (uint64_t i = 0; i < l; i++) {
        const int aa = i < NL(a) && ACTIVE(a, i), bb = i < NL(b) && ACTIVE(b, i);
        for (uint64_t e = 0; (aa || bb) && e < a->ntt->N; e++) {
            const uint64_t va = aa ? a->coeffs[i][e] : 0, vb = bb ? b->coeffs[i][e] : 0;
            if (va != vb) return false;
        }
    }
    return true;
}

/* fast base extension (rns_polynomial.c:738-822) */
void *init_base_conversion_params(void *ntt, uint64_t in_mask, uint64_t out_mask)
{
    uint64_t *p = (uint64_t *)malloc(3 * 8);
    p[0] = in_mask;
    p[1] = out_mask;
    p[2] = (uint64_t)(uintptr_t)ntt;
    return p;
}
void free_base_conversion_params(void *params) { free(params); }

void polynomial_base_conversion_RNSc(void *out, void *in, void *params)
{
    (void)params;
    RNS_Polynomial o = (RNS_Polynomial)out, a = (RNS_Polynomial)in;
    const uint64_t im = a->rns_mask, om = o->rns_mask, N = o->ntt->N;
    for (uint64_t i = 0; i < NL(o); i++)
        if (mask_bit(im, i) && mask_bit(om, i) && o != a) memcpy(o->coeffs[i], a->coeffs[i], N * 8);
    for (uint64_t t = 0; t < NL(o); t++) {
        if (!mask_bit(om, t) || mask_bit(im, t)) continue;
        const uint64_t pt = Q(o, t);
        uint64_t *acc = (uint64_t *)calloc(N, 8);
        for (uint64_t j = 0; j < NL(a); j++) {
            if (!mask_bit(im, j)) continue;
            const uint64_t qj = Q(a, j);
            uint64_t prod_j = 1 % qj, prod_t = 1 % pt;
            for (uint64_t k = 0; k < NL(a); k++)
                if (k != j && mask_bit(im, k)) {
                    prod_j = mulm(prod_j, Q(a, k) % qj, qj);
                    prod_t = mulm(prod_t, Q(a, k) % pt, pt);
                }
            const uint64_t dhat = invm(prod_j, qj);
            for (uint64_t e = 0; e < N; e++)
                acc[e] = addm(acc[e], mulm(mulm(a->coeffs[j][e], dhat, qj) % pt, prod_t, pt), pt);
        }
        memcpy(o->coeffs[t], acc, N * 8);
        free(acc);
    }
    o->rns_mask = om;
}

/* ------------------------------------------------------------------ mlwe */
static RNS_MLWE mlwe_new(uint64_t N, uint64_t r, uint64_t mask, incNTT t)
{
    RNS_MLWE m = (RNS_MLWE)calloc(1, sizeof(*m));
    m->a = (RNS_Polynomial *)calloc(r ? r : 1, sizeof(RNS_Polynomial));
    for (uint64_t i = 0; i < r; i++) m->a[i] = (RNS_Polynomial)polynomial_new_RNS_polynomial(N, mask, t);
    m->b = (RNS_Polynomial)polynomial_new_RNS_polynomial(N, mask, t);
    m->r = r;
    return m;
}

void *mlwe_alloc_RNS_sample(uint64_t N, uint64_t r, uint64_t mask, void *ntt) { return mlwe_new(N, r, mask, (incNTT)ntt); }

void free_mlwe_RNS_sample(void *p)
{
    RNS_MLWE m = (RNS_MLWE)p;
    if (!m) return;
    for (uint64_t i = 0; i < m->r; i++) free_RNS_polynomial(m->a[i]);
    free(m->a);
    free_RNS_polynomial(m->b);
    free(m);
}

void *mlwe_alloc_RNS_sample_array(uint64_t size, uint64_t N, uint64_t r, uint64_t mask, void *ntt)
{
    RNS_MLWE *arr = (RNS_MLWE *)malloc((size ? size : 1) * sizeof(RNS_MLWE));
    for (uint64_t i = 0; i < size; i++) arr[i] = mlwe_new(N, r, mask, (incNTT)ntt);
    return arr;
}

void mlwe_copy_RNS_sample(void *out, void *in)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) polynomial_copy_RNS_polynomial(o->a[i], a->a[i]);
    polynomial_copy_RNS_polynomial(o->b, a->b);
}

void *mlwe_create_copy_array(void *in, uint64_t size)
{
    RNS_MLWE *src = (RNS_MLWE *)in;
    RNS_MLWE *arr = (RNS_MLWE *)mlwe_alloc_RNS_sample_array(size, src[0]->b->ntt->N, src[0]->r, src[0]->b->rns_mask,
                                                            src[0]->b->ntt);
    for (uint64_t i = 0; i < size; i++) mlwe_copy_RNS_sample(arr[i], src[i]);
    return arr;
}

void *mlwe_new_RNS_key_from_array(uint64_t *array, uint64_t N, uint64_t r, uint64_t l, void *ntt, double sigma)
{
    RNS_MLWE_Key k = (RNS_MLWE_Key)calloc(1, sizeof(*k));
    k->N = N;
    k->r = r;
    k->l = l;
    k->sigma = sigma;
    k->s = (IntPolynomial *)calloc(r ? r : 1, sizeof(IntPolynomial));
    k->s_RNS = (RNS_Polynomial *)calloc(r ? r : 1, sizeof(RNS_Polynomial));
    for (uint64_t i = 0; i < r; i++) {
        k->s[i] = (IntPolynomial)calloc(1, sizeof(struct _IntPolynomial));
        k->s[i]->coeffs = (uint64_t *)malloc(N * 8);
        k->s[i]->N = N;
        memcpy(k->s[i]->coeffs, array + i * N, N * 8);
        k->s_RNS[i] = (RNS_Polynomial)polynomial_new_RNS_polynomial(N, l >= 64 ? ~0ULL : (1ULL << l) - 1, ntt);
        int_array_to_RNS(k->s_RNS[i], k->s[i]->coeffs);
    }
    return k;
}

void free_mlwe_RNS_key(void *key)
{
    RNS_MLWE_Key k = (RNS_MLWE_Key)key;
    if (!k) return;
    for (uint64_t i = 0; i < k->r; i++) {
        free(k->s[i]->coeffs);
        free(k->s[i]);
        free_RNS_polynomial(k->s_RNS[i]);
    }
    free(k->s);
    free(k->s_RNS);
    free(k);
}

void mlwe_RNSc_to_RNS(void *out, void *in)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) polynomial_RNSc_to_RNS(o->a[i], a->a[i]);
    polynomial_RNSc_to_RNS(o->b, a->b);
}

void mlwe_RNS_to_RNSc(void *out, void *in)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) polynomial_RNS_to_RNSc(o->a[i], a->a[i]);
    polynomial_RNS_to_RNSc(o->b, a->b);
}

static void zero_all(RNS_Polynomial p)
{
    for (uint64_t i = 0; i < NL(p); i++) memset(p->coeffs[i], 0, p->ntt->N * 8);
}

void mlwe_RNS_trivial_sample_of_zero(void *out)
{
    RNS_MLWE o = (RNS_MLWE)out;
    for (uint64_t i = 0; i < o->r; i++) zero_all(o->a[i]);
    zero_all(o->b);
}

void *mlwe_new_RNS_trivial_sample_of_zero(uint64_t N, uint64_t r, uint64_t mask, void *ntt)
{
    RNS_MLWE m = mlwe_new(N, r, mask, (incNTT)ntt);
    mlwe_RNS_trivial_sample_of_zero(m);
    return m;
}

void mlwe_RNS_phase(void *out, void *in, void *key)
{
    RNS_MLWE c = (RNS_MLWE)in;
    RNS_MLWE_Key k = (RNS_MLWE_Key)key;
    product((RNS_Polynomial)out, c->a[0], k->s_RNS[0], 0);
    for (uint64_t i = 1; i < c->r; i++) product((RNS_Polynomial)out, c->a[i], k->s_RNS[i], 1);
    polynomial_sub_RNS_polynomial(out, c->b, out);
}

static void mul_by_poly(void *out, void *in, void *poly, int mode)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) product(o->a[i], a->a[i], (RNS_Polynomial)poly, mode);
    product(o->b, a->b, (RNS_Polynomial)poly, mode);
}
void mlwe_RNS_mul_by_poly(void *o, void *a, void *p) { mul_by_poly(o, a, p, 0); }
void mlwe_RNS_mul_addto_by_poly(void *o, void *a, void *p) { mul_by_poly(o, a, p, 1); }
void mlwe_RNS_mul_subto_by_poly(void *o, void *a, void *p) { mul_by_poly(o, a, p, 2); }

void mlwe_scale_RNS_mlwe_RNS(void *c, uint64_t *s)
{
    RNS_MLWE m = (RNS_MLWE)c;
    for (uint64_t i = 0; i < m->r; i++) scale(m->a[i], m->a[i], s, 0);
    scale(m->b, m->b, s, 0);
}

void mlwe_add_RNSc_sample(void *out, void *in1, void *in2)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in1, b = (RNS_MLWE)in2;
    for (uint64_t i = 0; i < o->r; i++) binop(o->a[i], a->a[i], b->a[i], 0);
    binop(o->b, a->b, b->b, 0);
}

void mlwe_sub_RNSc_sample(void *out, void *in1, void *in2)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in1, b = (RNS_MLWE)in2;
    for (uint64_t i = 0; i < o->r; i++) binop(o->a[i], a->a[i], b->a[i], 1);
    binop(o->b, a->b, b->b, 1);
}

/* out = in * X^a (minus1: in * (X^a - 1)), split 1 (rns_polynomial.c:1048-1180) */
static void xai(RNS_Polynomial o, RNS_Polynomial in, uint64_t a, int minus1)
{
    const uint64_t N = o->ntt->N;
    a &= 2 * N - 1;
    o->rns_mask = in->rns_mask;
    if (a == 0) {
        if (minus1) zero_all(o);
        else polynomial_copy_RNS_polynomial(o, in);
        return;
    }
    for (uint64_t i = 0; i < NL(o); i++) {
        if (!ACTIVE(o, i)) continue;
        const uint64_t q = Q(o, i);
        for (uint64_t x = 0; x < N; x++) {
            const uint64_t src = (x + 2 * N - a) % (2 * N);
            uint64_t v = src < N ? in->coeffs[i][src] : negm(in->coeffs[i][src - N], q);
            o->coeffs[i][x] = minus1 ? subm(v, in->coeffs[i][x], q) : v;
        }
    }
}

void mlwe_RNSc_mul_by_xai(void *out, void *in, uint64_t a)
{
    RNS_MLWE o = (RNS_MLWE)out, s = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) xai(o->a[i], s->a[i], a, 0);
    xai(o->b, s->b, a, 0);
}

void mlwe_RNSc_mul_by_xai_minus1(void *out, void *in, uint64_t a)
{
    RNS_MLWE o = (RNS_MLWE)out, s = (RNS_MLWE)in;
    for (uint64_t i = 0; i < o->r; i++) xai(o->a[i], s->a[i], a, 1);
    xai(o->b, s->b, a, 1);
}

void mlwe_add_RNSc_polynomial(void *o, void *a, void *p) { binop(((RNS_MLWE)o)->b, ((RNS_MLWE)a)->b, p, 0); }
void mlwe_sub_RNSc_polynomial(void *o, void *a, void *p) { binop(((RNS_MLWE)o)->b, ((RNS_MLWE)a)->b, p, 1); }
void mlwe_RNS_add_polynomial(void *o, void *a, void *p) { binop(((RNS_MLWE)o)->b, ((RNS_MLWE)a)->b, p, 0); }
void mlwe_RNS_sub_polynomial(void *o, void *a, void *p) { binop(((RNS_MLWE)o)->b, ((RNS_MLWE)a)->b, p, 1); }

void mlwe_round_division_RNSc(void *out, uint64_t m)
{
    RNS_MLWE o = (RNS_MLWE)out;
    if (!m) return;
    for (uint64_t i = 0; i < o->r; i++) divide(o->a[i], m, 1);
    divide(o->b, m, 1);
}

/* gadget product over RNS digits (gadget.c:5-36) */
static void gadget(RNS_MLWE out, RNS_MLWE *ksk, RNS_Polynomial poly, int mode)
{
    RNS_Polynomial tmp = (RNS_Polynomial)polynomial_new_RNS_polynomial(ksk[0]->b->ntt->N, ksk[0]->b->rns_mask,
                                                                       ksk[0]->b->ntt);
    uint64_t k = 0;
    for (uint64_t j = 0; j < out->b->ntt->l; j++) {
        if (!ACTIVE(poly, j)) continue;
        polynomial_RNSc_mod_reduce_lifted(tmp, poly, j);
        polynomial_RNSc_to_RNS(tmp, tmp);
        mul_by_poly(out, ksk[k++], tmp, mode);
    }
    free_RNS_polynomial(tmp);
}

static void set_mask(RNS_MLWE m, uint64_t mask)
{
    for (uint64_t i = 0; i < m->r; i++) m->a[i]->rns_mask = mask;
    m->b->rns_mask = mask;
}

/* mlwe.c:557-598 */
void mlwe_RNSc_GHS_hybrid_keyswitch(void *out, void *in, void *ksk, uint64_t lvl)
{
    (void)lvl;
    RNS_MLWE o = (RNS_MLWE)out, c = (RNS_MLWE)in;
    RNS_MLWE **K = (RNS_MLWE **)ksk;
    uint64_t first = 0;
    while (first < c->r && !K[first]) first++;
    const uint64_t ext = K[first][0]->b->rns_mask;
    const uint64_t dmask = ext & ~c->b->rns_mask;
    set_mask(o, ext);
    mlwe_RNS_trivial_sample_of_zero(o);
    for (uint64_t i = 0; i < c->r; i++)
        if (K[i]) gadget(o, K[i], c->a[i], 2);
    mlwe_RNS_to_RNSc(o, o);
    mlwe_round_division_RNSc(o, dmask);
    uint64_t keep = 0;
    for (uint64_t i = 0; i < c->r; i++)
        if (!K[i]) {
            binop(o->a[keep], o->a[keep], c->a[i], 0);
            keep++;
        }
    binop(o->b, o->b, c->b, 0);
}

void mlwe_automorphism_RNSc_GHS(void *out, void *in, uint64_t gen, void *ksk, uint64_t lvl)
{
    RNS_MLWE o = (RNS_MLWE)out, c = (RNS_MLWE)in;
    RNS_MLWE t = mlwe_new(o->a[0]->ntt->N, o->r, o->a[0]->rns_mask, o->a[0]->ntt);
    for (uint64_t i = 0; i < o->r; i++) polynomial_RNSc_permute(t->a[i], c->a[i], gen);
    polynomial_RNSc_permute(t->b, c->b, gen);
    mlwe_RNSc_GHS_hybrid_keyswitch(o, t, ksk, lvl);
    free_mlwe_RNS_sample(t);
}

uint64_t mlwe_extended_rank(uint64_t r) { return r * (r + 3) / 2; }

/* mlwe.c:665-709 */
static void tensor(RNS_Polynomial *out, RNS_MLWE a, RNS_MLWE b)
{
    const uint64_t r = a->r, R = mlwe_extended_rank(r);
    uint64_t k = 0;
    for (uint64_t i = 0; i < r; i++)
        for (uint64_t j = i; j < r; j++, k++) {
            product(out[k], a->a[i], b->a[j], 0);
            if (i != j) product(out[k], a->a[j], b->a[i], 1);
        }
    for (uint64_t i = 0; i < r; i++, k++) {
        product(out[k], a->a[i], b->b, 0);
        product(out[k], a->b, b->a[i], 1);
    }
    product(out[R], a->b, b->b, 0);
}

void mlwe_tensor_product(void *out, void *in1, void *in2) { tensor((RNS_Polynomial *)out, in1, in2); }

/* mlwe.c:711-760 */
void mlwe_multiply(void *out, void *in1, void *in2, void *ksk)
{
    RNS_MLWE o = (RNS_MLWE)out, a = (RNS_MLWE)in1, b = (RNS_MLWE)in2;
    const uint64_t R = mlwe_extended_rank(a->r);
    RNS_MLWE ext = ksk ? mlwe_new(a->b->ntt->N, R, a->b->rns_mask, a->b->ntt) : o;
    RNS_Polynomial *tp = (RNS_Polynomial *)malloc((R + 1) * sizeof(RNS_Polynomial));
    for (uint64_t j = 0; j < R; j++) tp[j] = ext->a[j];
    tp[R] = ext->b;
    tensor(tp, a, b);
    free(tp);
    if (!ksk) return;
    mlwe_RNS_to_RNSc(ext, ext);
    mlwe_RNSc_GHS_hybrid_keyswitch(o, ext, ksk, 0);
    mlwe_RNSc_to_RNS(o, o);
    free_mlwe_RNS_sample(ext);
}

/* mgsw.c:6-72 */
void mgsw_external_product(void *out, void *mgsw, void *in, uint64_t ell, uint64_t special_primes)
{
    RNS_MLWE o = (RNS_MLWE)out, c = (RNS_MLWE)in;
    RNS_MLWE *G = (RNS_MLWE *)mgsw;
    set_mask(o, G[0]->b->rns_mask);
    mlwe_RNS_trivial_sample_of_zero(o);
    for (uint64_t j = 0; j < c->r; j++) gadget(o, &G[j * ell], c->a[j], 1);
    gadget(o, &G[c->r * ell], c->b, 1);
    if (special_primes) {
        mlwe_RNS_to_RNSc(o, o);
        uint64_t dm = 0, cnt = 0;
        for (int idx = 63; idx >= 0 && cnt < special_primes; idx--)
            if (mask_bit(o->b->rns_mask, (uint64_t)idx)) {
                dm |= 1ULL << idx;
                cnt++;
            }
        mlwe_round_division_RNSc(o, dm);
        mlwe_RNSc_to_RNS(o, o);
    }
}

void mgsw_CMUX(void *out, void *in1, void *in2, void *mgsw, uint64_t ell, uint64_t special_primes)
{
    RNS_MLWE a = (RNS_MLWE)in1, o = (RNS_MLWE)out;
    RNS_MLWE d = mlwe_new(a->b->ntt->N, a->r, a->b->rns_mask, a->b->ntt);
    mlwe_sub_RNSc_sample(d, in2, in1);
    mgsw_external_product(out, mgsw, d, ell, special_primes);
    RNS_MLWE an = mlwe_new(a->b->ntt->N, a->r, a->b->rns_mask, a->b->ntt);
    mlwe_copy_RNS_sample(an, a);
    mlwe_RNSc_to_RNS(an, an);
    for (uint64_t i = 0; i < o->r; i++) binop(o->a[i], o->a[i], an->a[i], 0);
    binop(o->b, o->b, an->b, 0);
    free_mlwe_RNS_sample(d);
    free_mlwe_RNS_sample(an);
}

/* mlwe.c:40-68 */
void *lwe_alloc_sample(uint64_t n, uint64_t l, void *ntt)
{
    LWE c = (LWE)calloc(1, sizeof(*c));
    c->a = (uint64_t **)malloc((l ? l : 1) * sizeof(uint64_t *));
    for (uint64_t i = 0; i < l; i++) c->a[i] = (uint64_t *)calloc(n ? n : 1, 8);
    c->b = (uint64_t *)calloc(l ? l : 1, 8);
    c->n = n;
    c->l = l;
    c->ntt = (incNTT)ntt;
    return c;
}

void free_lwe_sample(void *p)
{
    LWE c = (LWE)p;
    if (!c) return;
    for (uint64_t i = 0; i < c->l; i++) free(c->a[i]);
    free(c->a);
    free(c->b);
    free(c);
}

void *lwe_alloc_key(uint64_t n, uint64_t l, void *ntt)
{
    LWE_Key k = (LWE_Key)calloc(1, sizeof(*k));
    k->s = (uint64_t **)malloc((l ? l : 1) * sizeof(uint64_t *));
    for (uint64_t i = 0; i < l; i++) k->s[i] = (uint64_t *)calloc(n ? n : 1, 8);
    k->n = n;
    k->l = l;
    k->ntt = (incNTT)ntt;
    return k;
}

void *mlwe_extract_LWE(void *in, uint64_t idx)
{
    RNS_MLWE c = (RNS_MLWE)in;
    const uint64_t N = c->a[0]->ntt->N, r = c->r;
    uint64_t l = 0;
    for (uint64_t i = 0; i < 64; i++) l += mask_bit(c->a[0]->rns_mask, i);
    LWE res = (LWE)lwe_alloc_sample(r * N, l, c->a[0]->ntt);
    uint64_t j = 0;
    for (uint64_t g = 0; g < NL(c->a[0]); g++) {
        if (!ACTIVE(c->a[0], g)) continue;
        const uint64_t q = Q(c->a[0], g);
        for (uint64_t k = 0; k < r; k++)
            for (uint64_t i = 0; i < N; i++)
                res->a[j][k * N + i] = i <= idx ? c->a[k]->coeffs[g][idx - i] : negm(c->a[k]->coeffs[g][N + idx - i], q);
        res->b[j] = c->b->coeffs[g][idx];
        j++;
    }
    return res;
}

/* lwe.c:141-156 */
void lwe_phase(uint64_t *out, void *pc, void *pk)
{
    LWE c = (LWE)pc;
    LWE_Key k = (LWE_Key)pk;
    for (uint64_t i = 0; i < k->l; i++) {
        const uint64_t q = k->ntt->ntt[i]->q;
        uint64_t sum = 0;
        for (uint64_t j = 0; j < k->n; j++) sum = addm(sum, mulm(c->a[i][j], k->s[i][j], q), q);
        out[i] = subm(c->b[i], sum, q);
    }
}

void lwe_subto(void *out, void *in)
{
    LWE o = (LWE)out, a = (LWE)in;
    for (uint64_t i = 0; i < o->l; i++) {
        const uint64_t q = o->ntt->ntt[i]->q;
        for (uint64_t j = 0; j < o->n; j++) o->a[i][j] = subm(o->a[i][j], a->a[i][j], q);
        o->b[i] = subm(o->b[i], a->b[i], q);
    }
}

void *lwe_new_trivial_sample(uint64_t *m, uint64_t n, uint64_t l, void *ntt)
{
    LWE c = (LWE)lwe_alloc_sample(n, l, ntt);
    for (uint64_t i = 0; i < l; i++) c->b[i] = m ? m[i] : 0;
    return c;
}

/* ------------------------------------------------------------ complex FFT (CKKS encoding) */
/* Scalar restatement of modules/arith/c/src/complex.c (the reference's portable build,
 * complex.c:360-440): split real/imaginary layout, twiddles ws[0][m + i] / ws[1][m + i],
 * every product and sum rounded separately (build with -ffp-contract=off). */
#include <math.h>

static uint32_t brv20(uint32_t x, uint32_t prec) /* complex.c:13-24 */
{
    uint32_t r = 0;
    for (int b = 0; b < 20; ++b) r |= ((x >> b) & 1u) << (19 - b);
    return r >> (20 - prec);
}

void bit_reverse_array(double *v, uint64_t N, uint32_t prec) /* complex.c:26-39 */
{
    double *tmp = (double *)malloc(N * sizeof(double));
    for (int h = 0; h < 2; ++h) {
        for (uint64_t i = 0; i < N; i++) tmp[brv20((uint32_t)i, prec)] = v[h * N + i];
        memcpy(v + h * N, tmp, N * sizeof(double));
    }
    free(tmp);
}

void complex_poly_scale_double(double *v, double scale, uint64_t N) /* complex.c:366-370 */
{
    for (uint64_t i = 0; i < 2 * N; i++) v[i] *= scale;
}

static void *load_rous(double *re, double *im, uint64_t size) /* complex.c:371-387 */
{
    double **w = (double **)malloc(2 * sizeof(double *));
    w[0] = (double *)malloc(size * sizeof(double));
    w[1] = (double *)malloc(size * sizeof(double));
    memcpy(w[0], re, size * sizeof(double));
    memcpy(w[1], im, size * sizeof(double));
    return w;
}
void *load_rous_CT(double *re, double *im, uint64_t size) { return load_rous(re, im, size); }
void *load_rous_GS(double *re, double *im, uint64_t size) { return load_rous(re, im, size); }

void CT_NR(double *x, void *pws, uint64_t n) /* complex.c:389-412 */
{
    double **ws = (double **)pws;
    double *re = x, *im = x + n;
    for (uint64_t t = n, m = 1; m < n; m <<= 1) {
        t >>= 1;
        for (uint64_t i = 0; i < m; i++) {
            const double wr = ws[0][m + i], wi = ws[1][m + i];
            for (uint64_t j = 2 * i * t; j < 2 * i * t + t; j++) {
                const double vi = re[j + t] * wi + wr * im[j + t];
                const double vr = re[j + t] * wr - im[j + t] * wi;
                re[j + t] = re[j] - vr;
                im[j + t] = im[j] - vi;
                re[j] += vr;
                im[j] += vi;
            }
        }
    }
}

void GS_RN(double *x, void *pws, uint64_t n) /* complex.c:414-440 */
{
    double **ws = (double **)pws;
    double *re = x, *im = x + n;
    for (uint64_t t = 1, m = n; m > 1; t <<= 1, m >>= 1) {
        const uint64_t h = m >> 1;
        for (uint64_t i = 0; i < h; i++) {
            const double wr = ws[0][h + i], wi = ws[1][h + i];
            for (uint64_t j = 2 * i * t; j < 2 * i * t + t; j++) {
                const double vr = re[j] - re[j + t], vi = im[j] - im[j + t];
                re[j] += re[j + t];
                im[j] += im[j + t];
                im[j + t] = vr * wi + wr * vi;
                re[j + t] = vr * wr - vi * wi;
            }
        }
    }
}

void complex_poly_round_to_RNS(void *out, double *in, uint64_t N) /* complex.c:41-52 */
{
    (void)N;
    RNS_Polynomial o = (RNS_Polynomial)out;
    const uint64_t n = o->ntt->N;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) tmp[i] = (uint64_t)(int64_t)llrint(in[i]);
    int_array_to_RNS(o, tmp);
    free(tmp);
}

/* complex.c:458-476 (one thread) */
void complex_polys_ifft_scale_round_to_RNS_batch(void **rows_in, void **outs_rns, uint64_t count,
                                                 uint64_t n_complex, uint32_t log_prec, void *gs_ws,
                                                 double temp_delta)
{
    const double scale = temp_delta / (double)n_complex;
    for (uint64_t i = 0; i < count; i++) {
        double *row = (double *)rows_in[i];
        bit_reverse_array(row, n_complex, log_prec);
        GS_RN(row, gs_ws, n_complex);
        complex_poly_scale_double(row, scale, n_complex);
        complex_poly_round_to_RNS(outs_rns[i], row, n_complex);
    }
}
