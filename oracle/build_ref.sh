#!/usr/bin/env bash
# Compile the reference vfhe C library, from its own sources where they lie,
# into oracle/_ref/ (git-ignored; the .so files travel with the repo snapshot).
#
# One shared library per reference engine:
#   oracle/_ref/libvfhe_ref_portable.so    scalar unsigned __int128 engine
#   oracle/_ref/libvfhe_ref_avx512ifma.so  AVX-512 IFMA engine (built only if the
#                                          compiler accepts the ISA flags)
#
# This mirrors the reference's per-engine flags (tools/_engines.py:91-126,
# meson.build:18,130-205) without running its meson build: gcc on the module
# sources, gnu11, -O2.  The reference's BLAKE3 submodule is empty in the
# checkout, so oracle/blake3_standin/blake3.h (NOT BLAKE3) is put on the include
# path; no checked function hashes.
#
# Used only as a correctness checker and as the CPU baseline; nothing in the
# product links it.
set -euo pipefail

REF="${VFHE_REFERENCE_ROOT:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"

if [ ! -d "$REF/modules" ]; then
    echo "build_ref: reference sources not found at $REF; keeping prebuilt oracle/_ref" >&2
    exit 0
fi

M="$REF/modules"
SRCS=$(ls "$M"/arith/c/src/*.c "$M"/misc/c/src/*.c "$M"/mlwe/c/src/*.c "$M"/fhe/c/src/*.c)
INC="-I$M/arith/c/include -I$M/arith/c/src -I$M/misc/c/include -I$M/mlwe/c/include -I$HERE/blake3_standin"
COMMON="-O2 -std=gnu11 -fPIC -shared -w -pthread"

build_engine() {
    local name="$1"; shift
    local flags="$*"
    local lib="$OUT/libvfhe_ref_${name}.so"
    local tmp
    tmp="$(mktemp -d)"
    local objs=()
    for s in $SRCS; do
        local o="$tmp/$(basename "$s" .c).o"
        gcc $COMMON -c $INC -DVFHE_ENGINE_NAME="\"$name\"" $flags "$s" -o "$o"
        objs+=("$o")
    done
    gcc -shared -pthread -o "$lib" "${objs[@]}" -lm
    rm -rf "$tmp"
    echo "built $lib"
}

build_engine portable -DPORTABLE_BUILD
if echo 'int main(void){return 0;}' | gcc -mavx512f -mavx512ifma -x c - -o /dev/null 2>/dev/null; then
    build_engine avx512ifma -mavx512f -mavx512ifma -mavx512dq -mavx512vl -mavx2 -maes -mrdrnd
fi
