"""The engine's generator is ChaCha20 (RFC 8439 block function, 64-bit counter and
nonce in state words 12..15).  A plain restatement of the block function here is
pinned to the golden blocks of tests/golden/chacha20_blocks.json (made by the
`cryptography` package); the GPU tests hold the device generator to the same blocks."""

from __future__ import annotations

import json
import random
from pathlib import Path

GOLDEN = Path(__file__).parent / "golden" / "chacha20_blocks.json"
M32 = 0xFFFFFFFF


def _rotl(x: int, r: int) -> int:
    return ((x << r) | (x >> (32 - r))) & M32


def _quarter(s: list[int], a: int, b: int, c: int, d: int) -> None:
    s[a] = (s[a] + s[b]) & M32
    s[d] = _rotl(s[d] ^ s[a], 16)
    s[c] = (s[c] + s[d]) & M32
    s[b] = _rotl(s[b] ^ s[c], 12)
    s[a] = (s[a] + s[b]) & M32
    s[d] = _rotl(s[d] ^ s[a], 8)
    s[c] = (s[c] + s[d]) & M32
    s[b] = _rotl(s[b] ^ s[c], 7)


def chacha20_block(key_words: list[int], counter: int, nonce: int) -> list[int]:
    init = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574, *key_words,
            counter & M32, counter >> 32, nonce & M32, nonce >> 32]
    s = list(init)
    for _ in range(10):
        _quarter(s, 0, 4, 8, 12)
        _quarter(s, 1, 5, 9, 13)
        _quarter(s, 2, 6, 10, 14)
        _quarter(s, 3, 7, 11, 15)
        _quarter(s, 0, 5, 10, 15)
        _quarter(s, 1, 6, 11, 12)
        _quarter(s, 2, 7, 8, 13)
        _quarter(s, 3, 4, 9, 14)
    return [(x + y) & M32 for x, y in zip(s, init)]


def golden_cases() -> list[dict]:
    return json.loads(GOLDEN.read_text())["cases"]


def test_block_function_matches_golden():
    for case in golden_cases():
        for j, blk in enumerate(case["blocks"]):
            assert chacha20_block(case["key_words"], case["counter"] + j, case["nonce"]) == blk


def test_uniform_mod_is_floor_of_scaled_128_bit_draw():
    # the device maps 128 random bits r to floor(r q / 2^128) as the top 64 bits of
    # hi q + floor(lo q / 2^64): check that limb arithmetic against exact integers
    rng = random.Random(5)
    for _ in range(2000):
        q = rng.randrange(2**40, 2**50) | 1
        lo, hi = rng.getrandbits(64), rng.getrandbits(64)
        t = hi * q + ((lo * q) >> 64)
        assert t >> 64 == (((hi << 64) | lo) * q) >> 128
