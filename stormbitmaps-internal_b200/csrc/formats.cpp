// formats.cpp -- the reference's on-disk corpus format, read straight into the
// containers of this library.
//
// STORMBIN (written by the reference's tools/gt2bin.py, gnomad2bin.py,
// msprime2bin.py, sets2bin.py; read by bench/bench_allpairs.cpp:44-72 and
// bench/bench_threshold.cpp:65-83), little-endian:
//   "STORMBIN", u32 version (1), u32 n_rows, u32 n_bits, u32 pad
//   per row: u32 count, then count u32 positions, strictly ascending, < n_bits
// The header's n_rows may be 0 (the writers patch it at the end); rows are
// read until the end of the file. Like the reference's loaders, empty rows
// are skipped and every stride-th row (counting all rows, empty ones too) is
// kept, up to max_rows.
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "storm.h"
#include "storm_rows.h"

namespace {

struct StormbinHeader {
    uint32_t version = 0, n_rows = 0, n_bits = 0, pad = 0;
};

// Calls add(positions, n) for each kept row; returns rows kept or a status.
int64_t read_stormbin(const char* path, uint32_t max_rows, uint32_t stride, StormbinHeader* hdr_out,
                      const std::function<int(const uint32_t*, uint32_t)>& add) {
    if (path == NULL) return STORM_B200_EVALUES;
    FILE* f = std::fopen(path, "rb");
    if (!f) return STORM_B200_EARG;
    char magic[8];
    StormbinHeader h;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "STORMBIN", 8) != 0 ||
        std::fread(&h, sizeof(h), 1, f) != 1 || h.version != 1) {
        std::fclose(f);
        return STORM_B200_EVALUES;
    }
    if (hdr_out) *hdr_out = h;
    if (stride == 0) stride = 1;
    std::vector<uint32_t> pos;
    int64_t kept = 0;
    uint64_t seen = 0;
    while (max_rows == 0 || kept < (int64_t)max_rows) {
        uint32_t n = 0;
        if (std::fread(&n, 4, 1, f) != 1) break;
        pos.resize(n);
        if (n && std::fread(pos.data(), 4, n, f) != n) {
            std::fclose(f);
            return STORM_B200_EVALUES;   // truncated row
        }
        if (seen++ % stride != 0 || n == 0) continue;
        for (uint32_t k = 0; k < n; ++k)
            if (pos[k] >= h.n_bits || (k && pos[k] <= pos[k - 1])) {
                std::fclose(f);
                return STORM_B200_EVALUES;
            }
        const int rc = add(pos.data(), n);
        if (rc < 0) {
            std::fclose(f);
            return rc;
        }
        ++kept;
    }
    std::fclose(f);
    return kept;
}

// STORMPACK (written by the reference's tools/pack.cpp:100-145; one stored
// representation per row), little-endian:
//   "STRMPACK", u32 version (1), u32 n_rows, u32 n_bits (<= 65536), u32 flags
//   u32 offset[n_rows], u32 length[n_rows]   (bytes, into the payload)
//   u8 tag[n_rows]                           0 bitmap, 1 u16 array, 2 u16 runs
//                                            (start, length), 3 full, 4 empty
//   zero padding to a multiple of 8 bytes, then the payload.
// Every row is kept, empty ones included (the file stores them).
int64_t read_stormpack(const char* path, uint32_t* n_bits_out,
                       const std::function<int(const uint32_t*, uint32_t)>& add) {
    if (path == NULL) return STORM_B200_EVALUES;
    FILE* f = std::fopen(path, "rb");
    if (!f) return STORM_B200_EARG;
    std::vector<uint8_t> file;
    {
        uint8_t buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) file.insert(file.end(), buf, buf + got);
        std::fclose(f);
    }
    uint32_t hdr[4];
    if (file.size() < 24 || std::memcmp(file.data(), "STRMPACK", 8) != 0) return STORM_B200_EVALUES;
    std::memcpy(hdr, file.data() + 8, 16);
    const uint32_t version = hdr[0], n = hdr[1], nb = hdr[2];
    if (version != 1 || nb > 65536) return STORM_B200_EVALUES;
    uint64_t head = 24 + 9ull * n;
    head = (head + 7) & ~7ull;
    if (file.size() < head) return STORM_B200_EVALUES;
    const uint8_t* offs = file.data() + 24;
    const uint8_t* lens = offs + 4ull * n;
    const uint8_t* tags = lens + 4ull * n;
    const uint8_t* blob = file.data() + head;
    const uint64_t blob_len = file.size() - head;
    const uint32_t nw = (nb + 63) / 64;
    if (n_bits_out) *n_bits_out = nb;
    std::vector<uint32_t> pos;
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t off, len;
        std::memcpy(&off, offs + 4ull * r, 4);
        std::memcpy(&len, lens + 4ull * r, 4);
        if ((uint64_t)off + len > blob_len) return STORM_B200_EVALUES;
        const uint8_t* p = blob + off;
        pos.clear();
        switch (tags[r]) {
            case 0: {   // bitmap
                if (len < 8ull * nw) return STORM_B200_EVALUES;
                for (uint32_t w = 0; w < nw; ++w) {
                    uint64_t x;
                    std::memcpy(&x, p + 8ull * w, 8);
                    for (; x; x &= x - 1) pos.push_back(w * 64 + (uint32_t)__builtin_ctzll(x));
                }
                break;
            }
            case 1:     // u16 array
                for (uint32_t k = 0; 2 * k + 1 < len; ++k) {
                    uint16_t v;
                    std::memcpy(&v, p + 2ull * k, 2);
                    pos.push_back(v);
                }
                break;
            case 2:     // u16 runs
                for (uint32_t k = 0; 4 * k + 3 < len; ++k) {
                    uint16_t st, ln;
                    std::memcpy(&st, p + 4ull * k, 2);
                    std::memcpy(&ln, p + 4ull * k + 2, 2);
                    for (uint32_t e = 0; e < ln; ++e) pos.push_back((uint32_t)st + e);
                }
                break;
            case 3:     // full
                for (uint32_t e = 0; e < nb; ++e) pos.push_back(e);
                break;
            case 4:     // empty
                break;
            default:
                return STORM_B200_EVALUES;
        }
        for (size_t k = 0; k < pos.size(); ++k)
            if (pos[k] >= nb || (k && pos[k] <= pos[k - 1])) return STORM_B200_EVALUES;
        const int rc = add(pos.data(), (uint32_t)pos.size());
        if (rc < 0) return rc;
    }
    return n;
}

}  // namespace

extern "C" {

int64_t STORM_load_stormpack(STORM_t* s, const char* path, uint32_t* n_bits) {
    if (s == NULL) return STORM_B200_ENULL;
    return read_stormpack(path, n_bits, [&](const uint32_t* p, uint32_t n) {
        const int rc = STORM_add(s, p, n);
        return rc < 0 ? rc : 0;
    });
}

int64_t STORM_rows_load_stormpack(const char* path, STORM_rows_t** out) {
    if (out == NULL) return STORM_B200_ENULL;
    *out = NULL;
    STORM_rows_t* r = NULL;
    uint32_t nb = 0;
    const int64_t kept = read_stormpack(path, &nb, [&](const uint32_t* p, uint32_t n) {
        if (r == NULL) r = STORM_rows_new(nb);
        if (r == NULL) return (int)STORM_B200_ENOMEM;
        const int rc = STORM_rows_add(r, p, n);
        return rc < 0 ? rc : 0;
    });
    if (kept < 0) {
        if (r) STORM_rows_free(r);
        return kept;
    }
    if (r == NULL) r = STORM_rows_new(nb);   // a file of zero rows
    *out = r;
    return kept;
}

int64_t STORM_rows_load_stormbin(const char* path, uint32_t max_rows, uint32_t stride, STORM_rows_t** out) {
    if (out == NULL) return STORM_B200_ENULL;
    *out = NULL;
    StormbinHeader h;
    {   // header first: the universe of the rows container
        FILE* f = path ? std::fopen(path, "rb") : NULL;
        if (!f) return path ? STORM_B200_EARG : STORM_B200_EVALUES;
        char magic[8];
        const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "STORMBIN", 8) == 0 &&
                        std::fread(&h, sizeof(h), 1, f) == 1 && h.version == 1;
        std::fclose(f);
        if (!ok) return STORM_B200_EVALUES;
    }
    STORM_rows_t* r = STORM_rows_new(h.n_bits);
    if (r == NULL) return STORM_B200_ENOMEM;
    const int64_t kept = read_stormbin(path, max_rows, stride, NULL,
                                       [&](const uint32_t* p, uint32_t n) { return STORM_rows_add(r, p, n); });
    if (kept < 0) {
        STORM_rows_free(r);
        return kept;
    }
    *out = r;
    return kept;
}

int64_t STORM_load_stormbin(STORM_t* s, const char* path, uint32_t max_rows, uint32_t stride, uint32_t* n_bits) {
    if (s == NULL) return STORM_B200_ENULL;
    StormbinHeader h;
    const int64_t kept = read_stormbin(path, max_rows, stride, &h, [&](const uint32_t* p, uint32_t n) {
        const int rc = STORM_add(s, p, n);
        return rc < 0 ? rc : 0;
    });
    if (kept >= 0 && n_bits) *n_bits = h.n_bits;
    return kept;
}

}  // extern "C"
