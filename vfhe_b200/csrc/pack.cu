// Compact wire format for residue rows (ciphertexts in transit between host and GPU).
//
// A row of N residues of a b-bit prime (b = bit length of q, residues < q < 2^b) is
// stored as N b-bit fields in a little-endian bit stream: residue x occupies bits
// [x b, x b + b) of the row, bit k of the stream being bit (k mod 64) of 64-bit word
// k / 64.  N b must be a multiple of 64, so every row is whole words.  An item (one
// ciphertext [2][L][N]) is its rows one after another; items follow each other.
// For the CKKS benchmark's primes (one 50-bit, eight 40-bit) a ciphertext shrinks from
// 72 to 46.25 bytes per coefficient: the host-device copies that bound the end-to-end
// rate shrink with it.
//
// The reference has no serialisation (its ciphertexts live in host memory), so this
// format has no counterpart there.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "abi_common.cuh"

namespace vc {

namespace {

constexpr int kMaxPackRows = 128;

struct PackLayout {
    uint32_t bits[kMaxPackRows];
    uint64_t word_off[kMaxPackRows];  // first 64-bit word of row r inside an item
    uint64_t item_words;
    int rows;
};

// one thread per residue: up to two words, shifted and masked
__global__ void k_unpack(uint64_t* __restrict__ out, const uint64_t* __restrict__ in, long long N,
                         const __grid_constant__ PackLayout lay) {
    const long long item = blockIdx.y / lay.rows;
    const int r = blockIdx.y - (int)(item * lay.rows);
    const uint32_t b = lay.bits[r];
    const uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    const uint64_t* row = in + item * lay.item_words + lay.word_off[r];
    const uint64_t row_words = ((uint64_t)N * b) / 64;
    uint64_t* o = out + ((uint64_t)item * lay.rows + r) * N;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
         x += (long long)gridDim.x * blockDim.x) {
        const uint64_t bit = (uint64_t)x * b;
        const uint64_t w = bit >> 6;
        const uint32_t s = (uint32_t)(bit & 63);
        uint64_t v = row[w] >> s;
        if (s + b > 64 && w + 1 < row_words) v |= row[w + 1] << (64 - s);
        o[x] = v & mask;
    }
}

// one thread per output word: the residues overlapping it, shifted into place
__global__ void k_pack(uint64_t* __restrict__ out, const uint64_t* __restrict__ in, long long N,
                       const __grid_constant__ PackLayout lay) {
    const long long item = blockIdx.y / lay.rows;
    const int r = blockIdx.y - (int)(item * lay.rows);
    const uint32_t b = lay.bits[r];
    const uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    uint64_t* row = out + item * lay.item_words + lay.word_off[r];
    const uint64_t row_words = ((uint64_t)N * b) / 64;
    const uint64_t* src = in + ((uint64_t)item * lay.rows + r) * N;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < row_words;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t lo = w * 64, hi = lo + 64;  // bit range of this word
        uint64_t x = lo / b;
        uint64_t acc = 0;
        for (; x < (uint64_t)N && x * b < hi; ++x) {
            const uint64_t v = src[x] & mask;
            const uint64_t start = x * b;
            if (start >= lo) acc |= v << (start - lo);
            else acc |= v >> (lo - start);
        }
        row[w] = acc;
    }
}

bool make_layout(PackLayout& lay, uint64_t N, const uint32_t* bits, uint32_t rows, const char* where) {
    if (!bits || rows == 0 || rows > (uint32_t)kMaxPackRows || N == 0) {
        set_error(where, "need 1..128 rows per item, their bit widths and N > 0");
        return false;
    }
    memset(&lay, 0, sizeof lay);
    uint64_t off = 0;
    for (uint32_t r = 0; r < rows; ++r) {
        if (bits[r] == 0 || bits[r] > 64 || (N * bits[r]) % 64 != 0) {
            set_error(where, "bit widths must be 1..64 with N * bits a multiple of 64");
            return false;
        }
        lay.bits[r] = bits[r];
        lay.word_off[r] = off;
        off += N * bits[r] / 64;
    }
    lay.item_words = off;
    lay.rows = (int)rows;
    return true;
}

// Host form of k_pack for one row: N residues (masked to b bits) into N b / 64 words,
// least significant bits first (the same stream k_pack writes).
void pack_row_host(uint64_t* w, const uint64_t* src, uint64_t N, uint32_t b) {
    const uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    uint64_t acc = 0;
    uint32_t nb = 0;  // bits of acc in use, always < 64 here
    for (uint64_t x = 0; x < N; ++x) {
        const uint64_t v = src[x] & mask;
        acc |= v << nb;
        nb += b;
        if (nb >= 64) {
            *w++ = acc;
            nb -= 64;
            acc = nb ? v >> (b - nb) : 0;  // the bits of v that did not fit
        }
    }
}

// Host form of k_unpack for one row.
void unpack_row_host(uint64_t* dst, const uint64_t* w, uint64_t N, uint32_t b) {
    const uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    uint64_t cur = 0;
    uint32_t avail = 0;  // unread low bits of cur
    for (uint64_t x = 0; x < N; ++x) {
        uint64_t v;
        if (avail >= b) {
            v = cur & mask;
            cur = b >= 64 ? 0 : cur >> b;
            avail -= b;
        } else {
            const uint64_t nxt = *w++;
            v = (cur | (nxt << avail)) & mask;
            const uint32_t used = b - avail;
            cur = used >= 64 ? 0 : nxt >> used;
            avail = 64 - used;
        }
        dst[x] = v;
    }
}

// The same two transforms for one field width B fixed at compile time.  A row falls into
// periods of G = 64 / gcd(64, B) residues that fill W = B G / 64 words exactly (N B being
// a multiple of 64 makes N a multiple of G).  Within a period every word is an OR of the
// at most ceil(64 / B) + 1 residues that overlap it, at constant shifts, and every
// residue comes from at most two words, so neither direction carries a bit counter from
// one residue to the next.  Same bits as pack_row_host / unpack_row_host.
template <int B, int J, int POS>
inline uint64_t fixed_tail_bits(const uint64_t* v) {
    if constexpr (POS >= 64) {
        return 0;
    } else {
        return (v[J] << POS) | fixed_tail_bits<B, J + 1, POS + B>(v);
    }
}
template <int B, int K>
inline uint64_t fixed_word(const uint64_t* v) {
    constexpr int i0 = 64 * K / B, s0 = 64 * K % B;  // first residue overlapping word K
    return (v[i0] >> s0) | fixed_tail_bits<B, i0 + 1, B - s0>(v);
}
template <int B, int... K>
inline void fixed_pack_period(uint64_t* o, const uint64_t* v, std::integer_sequence<int, K...>) {
    ((o[K] = fixed_word<B, K>(v)), ...);
}
template <int B, int X>
inline uint64_t fixed_value(const uint64_t* w) {
    constexpr uint64_t mask = B >= 64 ? ~0ULL : ((1ULL << B) - 1);
    constexpr int k0 = X * B / 64, off = X * B % 64;
    if constexpr (off + B <= 64) {
        return (w[k0] >> off) & mask;
    } else {
        return ((w[k0] >> off) | (w[k0 + 1] << (64 - off))) & mask;
    }
}
template <int B, int... X>
inline void fixed_unpack_period(uint64_t* d, const uint64_t* w, std::integer_sequence<int, X...>) {
    ((d[X] = fixed_value<B, X>(w)), ...);
}
template <int B>
struct FixedPeriod {
    static constexpr int G = 64 / std::gcd(64, B);
    static constexpr int W = B * G / 64;
};
template <int B>
void pack_row_fixed(uint64_t* w, const uint64_t* src, uint64_t N) {
    constexpr int G = FixedPeriod<B>::G, W = FixedPeriod<B>::W;
    constexpr uint64_t mask = B >= 64 ? ~0ULL : ((1ULL << B) - 1);
    const uint64_t periods = N / G;
    for (uint64_t p = 0; p < periods; ++p) {
        uint64_t v[G];
        for (int j = 0; j < G; ++j) v[j] = src[p * G + j] & mask;
        fixed_pack_period<B>(w + p * W, v, std::make_integer_sequence<int, W>{});
    }
    if (periods * G < N) pack_row_host(w + periods * W, src + periods * G, N - periods * G, B);
}
template <int B>
void unpack_row_fixed(uint64_t* dst, const uint64_t* w, uint64_t N) {
    constexpr int G = FixedPeriod<B>::G, W = FixedPeriod<B>::W;
    const uint64_t periods = N / G;
    for (uint64_t p = 0; p < periods; ++p)
        fixed_unpack_period<B>(dst + p * G, w + p * W, std::make_integer_sequence<int, G>{});
    if (periods * G < N) unpack_row_host(dst + periods * G, w + periods * W, N - periods * G, B);
}

// Fixed-width forms for the widths of the engine's primes; other widths use the loops above.
constexpr int kFixedLo = 24, kFixedHi = 62;
using PackRowFn = void (*)(uint64_t*, const uint64_t*, uint64_t);
template <int... I>
constexpr std::array<PackRowFn, sizeof...(I)> fixed_pack_table(std::integer_sequence<int, I...>) {
    return {{&pack_row_fixed<kFixedLo + I>...}};
}
template <int... I>
constexpr std::array<PackRowFn, sizeof...(I)> fixed_unpack_table(std::integer_sequence<int, I...>) {
    return {{&unpack_row_fixed<kFixedLo + I>...}};
}
constexpr auto kPackFixed = fixed_pack_table(std::make_integer_sequence<int, kFixedHi - kFixedLo + 1>{});
constexpr auto kUnpackFixed = fixed_unpack_table(std::make_integer_sequence<int, kFixedHi - kFixedLo + 1>{});

void pack_row_best(uint64_t* w, const uint64_t* src, uint64_t N, uint32_t b) {
    if (b >= (uint32_t)kFixedLo && b <= (uint32_t)kFixedHi) return kPackFixed[b - kFixedLo](w, src, N);
    pack_row_host(w, src, N, b);
}
void unpack_row_best(uint64_t* dst, const uint64_t* w, uint64_t N, uint32_t b) {
    if (b >= (uint32_t)kFixedLo && b <= (uint32_t)kFixedHi) return kUnpackFixed[b - kFixedLo](dst, w, N);
    unpack_row_host(dst, w, N, b);
}

// Run fn(item, row) over every (item, row) of a layout on nthreads host threads, each
// taking a contiguous share.
template <class F>
void host_rows_parallel(const PackLayout& lay, uint64_t items, uint32_t nthreads, F fn) {
    const uint64_t units = items * (uint64_t)lay.rows;
    uint64_t nt = nthreads ? nthreads : std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<uint64_t>(nt, units);
    auto work = [&](uint64_t t) {
        for (uint64_t u = units * t / nt; u < units * (t + 1) / nt; ++u) fn(u / lay.rows, (int)(u % lay.rows));
    };
    std::vector<std::thread> pool;
    for (uint64_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

dim3 pack_grid(uint64_t per_row, uint64_t rows_total) {
    note_launch();
    uint64_t blocks = (per_row + 255) / 256;
    if (blocks > 64) blocks = 64;
    if (blocks < 1) blocks = 1;
    return dim3((unsigned)blocks, (unsigned)rows_total, 1);
}

}  // namespace

}  // namespace vc

using namespace vc;

extern "C" {

uint64_t vfhe_cuda_packed_bytes(uint64_t N, const uint32_t* bits, uint32_t rows_per_item, uint64_t items) {
    PackLayout lay;
    if (!make_layout(lay, N, bits, rows_per_item, "vfhe_cuda_packed_bytes")) return 0;
    return 8 * lay.item_words * items;
}

int vfhe_cuda_pack_rows(void* d_packed, const uint64_t* d_rows, uint64_t N, const uint32_t* bits,
                        uint32_t rows_per_item, uint64_t items, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_pack_rows";
    PackLayout lay;
    if (!make_layout(lay, N, bits, rows_per_item, where)) return 1;
    if (!d_packed || !d_rows || items == 0 || items * rows_per_item > 65535) {
        set_error(where, "null buffers or items * rows_per_item outside 1..65535");
        return 1;
    }
    uint64_t maxw = 0;
    for (uint32_t r = 0; r < rows_per_item; ++r) maxw = std::max<uint64_t>(maxw, N * bits[r] / 64);
    k_pack<<<pack_grid(maxw, items * rows_per_item), 256, 0, (cudaStream_t)stream>>>(
        (uint64_t*)d_packed, d_rows, (long long)N, lay);
    return check_cuda(cudaGetLastError(), where) ? 0 : 1;
}

int vfhe_cuda_unpack_rows(uint64_t* d_rows, const void* d_packed, uint64_t N, const uint32_t* bits,
                          uint32_t rows_per_item, uint64_t items, void* stream) {
    if (!ensure_ready()) return 1;
    const char* where = "vfhe_cuda_unpack_rows";
    PackLayout lay;
    if (!make_layout(lay, N, bits, rows_per_item, where)) return 1;
    if (!d_packed || !d_rows || items == 0 || items * rows_per_item > 65535) {
        set_error(where, "null buffers or items * rows_per_item outside 1..65535");
        return 1;
    }
    k_unpack<<<pack_grid(N, items * rows_per_item), 256, 0, (cudaStream_t)stream>>>(
        d_rows, (const uint64_t*)d_packed, (long long)N, lay);
    return check_cuda(cudaGetLastError(), where) ? 0 : 1;
}

int vfhe_cuda_pack_rows_host(void* h_packed, const uint64_t* h_rows, uint64_t N, const uint32_t* bits,
                             uint32_t rows_per_item, uint64_t items, uint32_t nthreads) {
    const char* where = "vfhe_cuda_pack_rows_host";
    PackLayout lay;
    if (!make_layout(lay, N, bits, rows_per_item, where)) return 1;
    if (!h_packed || !h_rows || items == 0) {
        set_error(where, "null buffers or no items");
        return 1;
    }
    uint64_t* out = (uint64_t*)h_packed;
    host_rows_parallel(lay, items, nthreads, [&](uint64_t item, int r) {
        pack_row_best(out + item * lay.item_words + lay.word_off[r], h_rows + (item * lay.rows + r) * N, N,
                      lay.bits[r]);
    });
    return 0;
}

int vfhe_cuda_unpack_rows_host(uint64_t* h_rows, const void* h_packed, uint64_t N, const uint32_t* bits,
                               uint32_t rows_per_item, uint64_t items, uint32_t nthreads) {
    const char* where = "vfhe_cuda_unpack_rows_host";
    PackLayout lay;
    if (!make_layout(lay, N, bits, rows_per_item, where)) return 1;
    if (!h_packed || !h_rows || items == 0) {
        set_error(where, "null buffers or no items");
        return 1;
    }
    const uint64_t* in = (const uint64_t*)h_packed;
    host_rows_parallel(lay, items, nthreads, [&](uint64_t item, int r) {
        unpack_row_best(h_rows + (item * lay.rows + r) * N, in + item * lay.item_words + lay.word_off[r], N,
                        lay.bits[r]);
    });
    return 0;
}

}  // extern "C"
