/*
 * NOT BLAKE3.  Compile-only stand-in for the BLAKE3 header that the vfhe
 * reference sources include (the BLAKE3 submodule is not vendored in the
 * reference checkout this build reads).
 *
 * It exists only so that the reference's own C sources compile into the
 * oracle/_ref libraries used as a correctness checker.  None of the functions
 * that hash (polynomial_RNS_get_hash, field_hash_element,
 * field_sample_random_element) are on the checked path, and the portable
 * engine's random-byte expansion is never relied on by any test: every key,
 * ciphertext and noise vector is generated by numpy from a seed and injected.
 *
 * The "hash" below is a splitmix64 absorb/squeeze.  It is deterministic and
 * nothing more: do not use its output where a cryptographic hash is expected.
 */
#ifndef VFHE_ORACLE_BLAKE3_STANDIN_H
#define VFHE_ORACLE_BLAKE3_STANDIN_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define BLAKE3_OUT_LEN 32
#define BLAKE3_KEY_LEN 32

typedef struct
{
    uint64_t state;
    uint64_t absorbed;
} blake3_hasher;

static inline uint64_t standin_mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static inline void blake3_hasher_init(blake3_hasher *h)
{
    h->state = 0x243f6a8885a308d3ULL;
    h->absorbed = 0;
}

static inline void blake3_hasher_update(blake3_hasher *h, const void *in, size_t len)
{
    const uint8_t *p = (const uint8_t *)in;
    for (size_t i = 0; i < len; i++)
    {
        h->state = standin_mix64(h->state ^ ((uint64_t)p[i] << ((i & 7) * 8)));
    }
    h->absorbed += len;
}

static inline void blake3_hasher_init_derive_key(blake3_hasher *h, const char *context)
{
    blake3_hasher_init(h);
    blake3_hasher_update(h, context, strlen(context));
}

static inline void blake3_hasher_finalize(const blake3_hasher *h, uint8_t *out, size_t out_len)
{
    uint64_t s = h->state ^ h->absorbed;
    for (size_t i = 0; i < out_len; i += 8)
    {
        s = standin_mix64(s);
        size_t n = out_len - i < 8 ? out_len - i : 8;
        memcpy(out + i, &s, n);
    }
}

#endif
