// Randomness of the cuda engine: the ChaCha20 stream cipher as a counter-based
// generator (D. J. Bernstein, "ChaCha, a variant of Salsa20", 2008; the block function
// of RFC 8439 section 2.3 with the original layout: a 64-bit block counter in state
// words 12-13 and a 64-bit nonce in words 14-15).  Block number c of a key is 64 bytes
// that any thread can compute on its own, so every sampling kernel draws its bits
// from the blocks it owns without shared state: the host reserves a range of block
// counters per call (prng_advance) and thread j of the call uses block base + j.
//
// The reference draws its randomness from AES-CTR or a BLAKE3 XOF keyed by RDRAND or
// /dev/urandom (modules/misc/c/src/prng.c:91-137); streams are not comparable across
// engines, only distributions (uniform residues, rounded Gaussians, ternary keys).
#pragma once
#include <stdint.h>

#include "modarith.cuh"

namespace vc {

struct PrngKey {
    uint32_t w[8];
};

VC_HD uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

VC_HD void chacha_quarter(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
    a += b;
    d = rotl32(d ^ a, 16);
    c += d;
    b = rotl32(b ^ c, 12);
    a += b;
    d = rotl32(d ^ a, 8);
    c += d;
    b = rotl32(b ^ c, 7);
}

// Block `counter` of the keystream for (key, nonce): 16 little-endian words.
VC_HD void chacha20_block(const PrngKey& key, uint64_t counter, uint64_t nonce, uint32_t (&out)[16]) {
    uint32_t s[16];
    s[0] = 0x61707865u;  // "expand 32-byte k"
    s[1] = 0x3320646eu;
    s[2] = 0x79622d32u;
    s[3] = 0x6b206574u;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int i = 0; i < 8; ++i) s[4 + i] = key.w[i];
    s[12] = (uint32_t)counter;
    s[13] = (uint32_t)(counter >> 32);
    s[14] = (uint32_t)nonce;
    s[15] = (uint32_t)(nonce >> 32);
    uint32_t x[16];
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int i = 0; i < 16; ++i) x[i] = s[i];
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {  // 20 rounds: column round + diagonal round
        chacha_quarter(x[0], x[4], x[8], x[12]);
        chacha_quarter(x[1], x[5], x[9], x[13]);
        chacha_quarter(x[2], x[6], x[10], x[14]);
        chacha_quarter(x[3], x[7], x[11], x[15]);
        chacha_quarter(x[0], x[5], x[10], x[15]);
        chacha_quarter(x[1], x[6], x[11], x[12]);
        chacha_quarter(x[2], x[7], x[8], x[13]);
        chacha_quarter(x[3], x[4], x[9], x[14]);
    }
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

// 64-bit word i (0..7) of a block.
VC_HD uint64_t block_u64(const uint32_t (&b)[16], int i) { return (uint64_t)b[2 * i] | ((uint64_t)b[2 * i + 1] << 32); }

// floor(r q / 2^128) for the 128-bit r = hi 2^64 + lo: a residue in [0, q) whose
// distance from uniform is below q / 2^128.
VC_HD uint64_t uniform_mod(uint64_t lo, uint64_t hi, uint64_t q) {
    const unsigned __int128 t = (unsigned __int128)hi * q + (uint64_t)(((unsigned __int128)lo * q) >> 64);
    return (uint64_t)(t >> 64);
}

// Lemire's multiply-shift with rejection ("Fast random integer generation in an
// interval", ACM TOMACS 29(1), 2019): for a uniform 64-bit r and m = r q, hi(m) is
// exactly uniform on [0, q) once the draws with lo(m) < 2^64 mod q (`thresh`) are
// rejected; a draw is rejected with probability below q / 2^64.  Returns acceptance.
VC_HD bool uniform_mod64(uint64_t r, uint64_t q, uint64_t thresh, uint64_t& out) {
    const unsigned __int128 m = (unsigned __int128)r * q;
    out = (uint64_t)(m >> 64);
    return (uint64_t)m >= thresh;
}

// Uniform double in (0, 1] and [0, 1) from 53 bits of a 64-bit word.
VC_HD double unit_open_low(uint64_t r) { return ((double)(r >> 11) + 1.0) * (1.0 / 9007199254740992.0); }
VC_HD double unit_closed_low(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Nonces that keep the engine's samplers on separate streams of the same key.
enum PrngStream : uint64_t {
    kStreamUniform = 1,
    kStreamGaussian = 2,
    kStreamInteger = 3,
    kStreamTernary = 4,
    kStreamUniformRedraw = 5,  // replacements for rejected uniform_mod64 draws
};

}  // namespace vc
