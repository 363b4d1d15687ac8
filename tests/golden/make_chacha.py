"""Golden ChaCha20 keystream blocks for the engine's generator (tests/golden/chacha20_blocks.json).

Generated with the `cryptography` package's ChaCha20 (an independent implementation of
RFC 8439's block function), whose 16-byte nonce argument is state words 12..15: the
64-bit block counter then the 64-bit nonce, the layout the engine uses.

    python tests/golden/make_chacha.py
"""

from __future__ import annotations

import json
import struct
from pathlib import Path

from cryptography.hazmat.primitives.ciphers import Cipher, algorithms

CASES = [
    # (key bytes, first block counter, nonce, blocks)
    (bytes(range(32)), 0, 0, 2),
    (bytes(range(32)), 1, 0x4A000000_09000000, 1),
    (bytes([0xFF] * 32), 12345, 5, 3),
    (bytes((7 * i + 3) % 256 for i in range(32)), 0x1_0000_0010, 2, 2),
]


def blocks(key: bytes, counter: int, nonce: int, n: int) -> list[list[int]]:
    out = []
    for j in range(n):
        c = Cipher(algorithms.ChaCha20(key, struct.pack("<QQ", counter + j, nonce)), mode=None).encryptor()
        out.append(list(struct.unpack("<16I", c.update(bytes(64)))))
    return out


def main() -> None:
    cases = [{"key_words": list(struct.unpack("<8I", key)), "counter": ctr, "nonce": nonce,
              "blocks": blocks(key, ctr, nonce, n)} for key, ctr, nonce, n in CASES]
    path = Path(__file__).with_name("chacha20_blocks.json")
    path.write_text(json.dumps({"generator": "cryptography ChaCha20 (RFC 8439 block function)", "cases": cases},
                               indent=1))
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
