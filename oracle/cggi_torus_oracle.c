/*
 * CPU oracle for the 32-bit-torus CGGI bootstrap with FP64 FFT external products.
 * TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's CPU leg
 * use it as the checker; nothing in the product links or calls it.
 *
 * The reference has no torus/FFT CGGI (its CGGI16 uses an RNS gadget with NTT
 * external products, modules/mlwe/c/src/mgsw.c:6-72, and its LWE key switch is a
 * stub, modules/mlwe/c/src/lwe.c:170-176), so this variant's parity is UNPINNED
 * against the reference.  This file restates the published TFHE bootstrap
 * (Chillotti, Gama, Georgieva, Izabachene, "TFHE: Fast Fully Homomorphic Encryption
 * over the Torus", J. Cryptology 33, 2020: GGSW external product, CMUX blind
 * rotation, sample extraction, base-2^b LWE key switching) with EXACT integer
 * arithmetic mod 2^32: every polynomial product is a schoolbook negacyclic
 * convolution, so the GPU's FFT products can be checked against the exact result and
 * its bootstraps against exact phases.  The blind rotation follows the reference's
 * CGGI16 orchestration (modules/fhe/python/src/vfhe/fhe/cggi16.py:46-128: rotation
 * amounts with a half-box offset, CMUX(acc, acc X^a_i), extraction at coefficient 0).
 *
 * Conventions (shared with vfhe_b200/csrc/cggi_fft.cu):
 *   torus values are uint32 (Z / 2^32); a GLWE sample (a, b) of rank 1 has phase
 *   b - a S mod X^N + 1; an LWE (a[0..n), b) has phase b - <a, s>.
 *   gadget: base 2^g, `levels` levels, signed digits in [-2^(g-1), 2^(g-1)) of the
 *   value rounded to its top g*levels bits; level l (0 = most significant) has weight
 *   2^(32 - g (l + 1)).
 *   GGSW row order: (component c, level l) at row c * levels + l, each row a GLWE
 *   (a, b) of 2N torus values; row (c, l) carries mu * 2^(32 - g (l+1)) on component c.
 *   key switch: base 2^kb, kt levels, KSK[j][l] = LWE_s(S_j 2^(32 - kb (l+1))), rows
 *   of n + 1 values (a, then b); signed digits as for the gadget.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* signed digits of v rounded to its top base_log * levels bits; digit[0] most significant */
void tor_decompose(int32_t *digits, uint32_t v, int base_log, int levels)
{
    const int total = base_log * levels;
    uint64_t r = ((uint64_t)v + (1ULL << (31 - total))) >> (32 - total); /* round to `total` bits */
    r &= (total >= 32) ? 0xFFFFFFFFULL : ((1ULL << total) - 1);
    const int64_t half = 1LL << (base_log - 1), full = 1LL << base_log;
    for (int l = levels - 1; l >= 0; --l)
    {
        int64_t d = (int64_t)(r & (uint64_t)(full - 1));
        r >>= base_log;
        if (d >= half)
        {
            d -= full;
            r += 1;
        }
        digits[l] = (int32_t)d;
    }
}

/* out += d * p mod (X^N + 1, 2^32): d small signed integers, p torus values */
void tor_negacyclic_mac(uint32_t *out, const int32_t *d, const uint32_t *p, int N)
{
    for (int i = 0; i < N; ++i)
    {
        const uint32_t di = (uint32_t)d[i];
        if (!di)
            continue;
        for (int j = 0; j < N; ++j)
        {
            const uint32_t t = di * p[j];
            if (i + j < N)
                out[i + j] += t;
            else
                out[i + j - N] -= t;
        }
    }
}

/* out[2N] = ExtProd(ggsw, c) for a rank-1 GLWE c[2N] = (a, b) */
void tor_external_product(uint32_t *out, const uint32_t *c, const uint32_t *ggsw, int N, int base_log, int levels)
{
    int32_t *dig = (int32_t *)malloc(sizeof(int32_t) * levels * 2 * N);
    int32_t tmp[32];
    for (int comp = 0; comp < 2; ++comp)
        for (int k = 0; k < N; ++k)
        {
            tor_decompose(tmp, c[comp * N + k], base_log, levels);
            for (int l = 0; l < levels; ++l)
                dig[(comp * levels + l) * N + k] = tmp[l];
        }
    memset(out, 0, sizeof(uint32_t) * 2 * N);
    for (int row = 0; row < 2 * levels; ++row)
        for (int oc = 0; oc < 2; ++oc)
            tor_negacyclic_mac(out + oc * N, dig + row * N, ggsw + ((size_t)row * 2 + oc) * N, N);
    free(dig);
}

/* r = p * X^e mod X^N + 1, 0 <= e < 2N */
static void rot(uint32_t *r, const uint32_t *p, int N, int e)
{
    for (int j = 0; j < N; ++j)
    {
        int k = j + e;
        uint32_t v = p[j];
        k %= 2 * N;
        if (k >= N)
        {
            k -= N;
            v = (uint32_t)(0u - v);
        }
        r[k] = v;
    }
}

/* round(v 2N / 2^32) mod 2N */
static int modswitch(uint32_t v, int N)
{
    const int logN2 = __builtin_ctz((unsigned)(2 * N));
    return (int)((((uint64_t)v + (1ULL << (31 - logN2))) >> (32 - logN2)) & (uint64_t)(2 * N - 1));
}

/*
 * Blind rotation and extraction of one LWE (a[0..n), b) through the test vector tv[N]
 * (the b component of a trivial GLWE): acc = (0, tv X^-rot_b), rot_b = modswitch(b +
 * 2^32 / (4 base)); acc = CMUX(s_i, acc, acc X^modswitch(a_i)) for every i (bsk: n GGSW
 * of 2*levels rows x 2N); extracted LWE out[0..N) mask, out[N] body.
 */
void tor_bootstrap(uint32_t *out, const uint32_t *a, uint32_t b, const uint32_t *tv, const uint32_t *bsk, int n, int N,
                   int base_log, int levels, uint32_t torus_base)
{
    uint32_t *acc = (uint32_t *)calloc(2 * N, sizeof(uint32_t));
    uint32_t *r = (uint32_t *)malloc(sizeof(uint32_t) * 2 * N);
    uint32_t *e = (uint32_t *)malloc(sizeof(uint32_t) * 2 * N);
    const uint32_t offset = (uint32_t)((1ULL << 32) / (4ULL * torus_base));
    const int rb = modswitch(b + offset, N);
    rot(acc + N, tv, N, (2 * N - rb) % (2 * N));
    const size_t gg = (size_t)2 * levels * 2 * N;
    for (int i = 0; i < n; ++i)
    {
        const int ai = modswitch(a[i], N);
        if (!ai)
            continue; /* CMUX of equal inputs: acc unchanged (the product of zero is zero) */
        rot(r, acc, N, ai);
        rot(r + N, acc + N, N, ai);
        for (int k = 0; k < 2 * N; ++k)
            r[k] -= acc[k];
        tor_external_product(e, r, bsk + gg * i, N, base_log, levels);
        for (int k = 0; k < 2 * N; ++k)
            acc[k] += e[k];
    }
    out[0] = acc[0];
    for (int j = 1; j < N; ++j)
        out[j] = (uint32_t)(0u - acc[N - j]);
    out[N] = acc[N];
    free(acc);
    free(r);
    free(e);
}

/* key switch in[0..N) mask, in[N] body (key S, dimension N) to out[0..n), out[n] (key s) */
void tor_keyswitch(uint32_t *out, const uint32_t *in, const uint32_t *ksk, int N, int n, int base_log, int levels)
{
    int32_t d[32];
    memset(out, 0, sizeof(uint32_t) * (n + 1));
    out[n] = in[N];
    for (int j = 0; j < N; ++j)
    {
        tor_decompose(d, in[j], base_log, levels);
        for (int l = 0; l < levels; ++l)
        {
            if (!d[l])
                continue;
            const uint32_t *row = ksk + ((size_t)j * levels + l) * (n + 1);
            const uint32_t dl = (uint32_t)d[l];
            for (int k = 0; k <= n; ++k)
                out[k] -= dl * row[k];
        }
    }
}

/* b - <a, s> for an LWE of dimension n and a binary (or small) secret */
uint32_t tor_lwe_phase(const uint32_t *a, uint32_t b, const int32_t *s, int n)
{
    uint32_t acc = b;
    for (int i = 0; i < n; ++i)
        acc -= a[i] * (uint32_t)s[i];
    return acc;
}
