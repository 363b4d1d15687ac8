// Evaluation-key files: raw residue rows behind a versioned header.
//
// The reference keeps its keys in process memory only (it has no serialisation), so a
// serving host must regenerate relinearisation, Galois and bootstrapping keys on every
// start.  This format lets a host save keys made once (on the GPU or elsewhere) and
// load them back bit for bit.  Layout, all little-endian:
//
//   offset  size  field
//        0     8  magic "VFHEKEY\0"
//        8     4  format version (1)
//       12     4  kind (vfhe_cuda.h: VFHE_KEY_*)
//       16     4  element bytes (8: RNS residues, 4: torus values)
//       20     4  number of dimensions (1..8)
//       24    64  dims[8] (uint64; unused ones 0)
//       88     4  number of moduli (0..64)
//       92     4  reserved (0)
//       96    32  aux[4] (uint64, kind-specific: Galois element, level, N, ...)
//      128   512  moduli[64] (uint64; the primes of the limb axis, in order)
//      640     8  payload bytes
//      648     8  FNV-1a-64 of the payload, over 64-bit little-endian words
//      656     -  payload: the key tensor in row-major order
//
// The functions take host buffers only, so they need no GPU; callers copy device keys
// in and out around them.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "abi_common.cuh"

namespace {

constexpr char kMagic[8] = {'V', 'F', 'H', 'E', 'K', 'E', 'Y', '\0'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeaderBytes = 656;

uint64_t fnv1a_words(const uint8_t* p, uint64_t bytes) {
    uint64_t h = 0xcbf29ce484222325ULL;
    uint64_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        memcpy(&w, p + i, 8);
        h = (h ^ w) * 0x100000001b3ULL;
    }
    if (i < bytes) {
        uint64_t w = 0;
        memcpy(&w, p + i, bytes - i);
        h = (h ^ w) * 0x100000001b3ULL;
    }
    return h;
}

bool shape_bytes(const VfheKeyHeader* h, uint64_t* out) {
    if (h->ndims == 0 || h->ndims > 8 || (h->elem_bytes != 4 && h->elem_bytes != 8) || h->nmoduli > 64) return false;
    uint64_t n = h->elem_bytes;
    for (uint32_t d = 0; d < h->ndims; ++d) {
        if (h->dims[d] == 0 || n > (UINT64_MAX / h->dims[d])) return false;
        n *= h->dims[d];
    }
    for (uint32_t d = h->ndims; d < 8; ++d)
        if (h->dims[d] != 0) return false;
    *out = n;
    return true;
}

void put_u32(uint8_t* p, uint32_t v) { memcpy(p, &v, 4); }
void put_u64(uint8_t* p, uint64_t v) { memcpy(p, &v, 8); }
uint32_t get_u32(const uint8_t* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}
uint64_t get_u64(const uint8_t* p) {
    uint64_t v;
    memcpy(&v, p, 8);
    return v;
}

// Parse and validate a header block; on success *payload and *checksum are set.
bool parse_header(const uint8_t* b, VfheKeyHeader* h, uint64_t* payload, uint64_t* checksum, const char* where) {
    if (memcmp(b, kMagic, 8) != 0) {
        vc::set_error(where, "not a vfhe key file (bad magic)");
        return false;
    }
    if (get_u32(b + 8) != kVersion) {
        vc::set_error(where, "unsupported key file version");
        return false;
    }
    memset(h, 0, sizeof *h);
    h->kind = get_u32(b + 12);
    h->elem_bytes = get_u32(b + 16);
    h->ndims = get_u32(b + 20);
    for (int d = 0; d < 8; ++d) h->dims[d] = get_u64(b + 24 + 8 * d);
    h->nmoduli = get_u32(b + 88);
    for (int k = 0; k < 4; ++k) h->aux[k] = get_u64(b + 96 + 8 * k);
    for (int k = 0; k < 64; ++k) h->moduli[k] = get_u64(b + 128 + 8 * k);
    uint64_t want = 0;
    if (!shape_bytes(h, &want) || get_u64(b + 640) != want) {
        vc::set_error(where, "key file header is inconsistent (shape, element size or payload size)");
        return false;
    }
    *payload = want;
    *checksum = get_u64(b + 648);
    return true;
}

}  // namespace

extern "C" {

uint64_t vfhe_cuda_keyfile_payload_bytes(const VfheKeyHeader* hdr) {
    uint64_t n = 0;
    return hdr && shape_bytes(hdr, &n) ? n : 0;
}

int vfhe_cuda_keyfile_write(const char* path, const VfheKeyHeader* hdr, const void* host_data) {
    static const char* const where = "vfhe_cuda_keyfile_write";
    uint64_t bytes = 0;
    if (!path || !hdr || !host_data || !shape_bytes(hdr, &bytes)) {
        vc::set_error(where, "bad path, header (1..8 dims, 4- or 8-byte elements, <= 64 moduli) or data");
        return 1;
    }
    uint8_t b[kHeaderBytes];
    memset(b, 0, sizeof b);
    memcpy(b, kMagic, 8);
    put_u32(b + 8, kVersion);
    put_u32(b + 12, hdr->kind);
    put_u32(b + 16, hdr->elem_bytes);
    put_u32(b + 20, hdr->ndims);
    for (int d = 0; d < 8; ++d) put_u64(b + 24 + 8 * d, hdr->dims[d]);
    put_u32(b + 88, hdr->nmoduli);
    for (int k = 0; k < 4; ++k) put_u64(b + 96 + 8 * k, hdr->aux[k]);
    for (uint32_t k = 0; k < hdr->nmoduli; ++k) put_u64(b + 128 + 8 * k, hdr->moduli[k]);
    put_u64(b + 640, bytes);
    put_u64(b + 648, fnv1a_words((const uint8_t*)host_data, bytes));
    FILE* f = fopen(path, "wb");
    if (!f) {
        vc::set_error(where, "cannot open the file for writing");
        return 1;
    }
    const bool ok = fwrite(b, 1, sizeof b, f) == sizeof b && fwrite(host_data, 1, bytes, f) == bytes;
    const bool closed = fclose(f) == 0;
    if (!ok || !closed) {
        vc::set_error(where, "write failed");
        return 1;
    }
    return 0;
}

int vfhe_cuda_keyfile_read_header(const char* path, VfheKeyHeader* hdr) {
    static const char* const where = "vfhe_cuda_keyfile_read_header";
    if (!path || !hdr) {
        vc::set_error(where, "null path or header");
        return 1;
    }
    FILE* f = fopen(path, "rb");
    if (!f) {
        vc::set_error(where, "cannot open the file");
        return 1;
    }
    uint8_t b[kHeaderBytes];
    const bool got = fread(b, 1, sizeof b, f) == sizeof b;
    fclose(f);
    uint64_t payload = 0, sum = 0;
    if (!got) {
        vc::set_error(where, "file shorter than a key file header");
        return 1;
    }
    return parse_header(b, hdr, &payload, &sum, where) ? 0 : 1;
}

int vfhe_cuda_keyfile_read(const char* path, VfheKeyHeader* hdr, void* host_data, uint64_t capacity_bytes) {
    static const char* const where = "vfhe_cuda_keyfile_read";
    if (!path || !hdr || !host_data) {
        vc::set_error(where, "null path, header or buffer");
        return 1;
    }
    FILE* f = fopen(path, "rb");
    if (!f) {
        vc::set_error(where, "cannot open the file");
        return 1;
    }
    uint8_t b[kHeaderBytes];
    uint64_t payload = 0, sum = 0;
    if (fread(b, 1, sizeof b, f) != sizeof b) {
        fclose(f);
        vc::set_error(where, "file shorter than a key file header");
        return 1;
    }
    if (!parse_header(b, hdr, &payload, &sum, where)) {
        fclose(f);
        return 1;
    }
    if (payload > capacity_bytes) {
        fclose(f);
        vc::set_error(where, "buffer smaller than the key");
        return 1;
    }
    const bool got = fread(host_data, 1, payload, f) == payload;
    const bool trailing = fgetc(f) != EOF;
    fclose(f);
    if (!got || trailing) {
        vc::set_error(where, "payload size does not match the header (truncated or trailing bytes)");
        return 1;
    }
    if (fnv1a_words((const uint8_t*)host_data, payload) != sum) {
        vc::set_error(where, "payload checksum mismatch (corrupted key file)");
        return 1;
    }
    return 0;
}

}  // extern "C"
