/*
 * pq_oracle.cpp -- CPU restatement of the reference's Parquet page decoding.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for libvrgpu's page decoder
 * and its timed CPU baseline. Nothing in the product path may call it.
 *
 * Restates, from the reference (vecruntime, Java):
 *   RleBitPackingReader.readInts / readRunHeader / unpackGroup / readUleb128
 *       parquet/src/main/java/io/vecruntime/parquet/codec/RleBitPackingReader.java:138-185, 331-391
 *   ParquetFraming (run headers, value bytes, widths)  ParquetFraming.java:60-115
 *   ParquetPageDecoder.decode for flat pages (levels -> validity, present
 *       slots, RLE_DICTIONARY ids / PLAIN fixed values)  ParquetPageDecoder.java:214-311, 415-433
 *   ParquetPageDecoder.decodeDictionary, BYTE_ARRAY     ParquetPageDecoder.java:452-497
 * One difference, shared with the GPU decoder it checks: an RLE_DICTIONARY
 * page yields its ids, not the dictionary values they resolve to (the
 * aggregate resolves them through the batch dictionary), and a null slot
 * holds 0. Reads past a stream's end are errors here (the reference reads
 * whatever bytes follow in the page).
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

thread_local std::string g_pq_err;

int pq_fail(const std::string& why) {
    g_pq_err = why;
    return VR_ERR_INVALID;
}

// The reader's state over [pos, end) of `buf` (RleBitPackingReader's fields).
struct Rle {
    const uint8_t* buf;
    int64_t pos, end;
    int width, value_bytes;
    uint32_t mask;
    uint32_t rle_value = 0;
    int64_t rle_left = 0, packed_left = 0;
};

bool uleb(Rle& r, uint32_t& v) {
    v = 0;
    for (int shift = 0;; shift += 7) {
        if (r.pos >= r.end || shift > 28) return false;
        const uint8_t b = r.buf[r.pos++];
        v |= (uint32_t)(b & 0x7F) << shift;
        if (!(b & 0x80)) return true;
    }
}

// RleBitPackingReader.readRunHeader: low bit 1 = groups of 8 bit-packed
// values, 0 = a count of one repeated little-endian value.
bool run_header(Rle& r) {
    uint32_t h;
    if (!uleb(r, h)) return false;
    const int64_t count = h >> 1;
    if (h & 1) {
        r.packed_left = count * 8;
    } else {
        r.rle_left = count;
        if (r.pos + r.value_bytes > r.end) return false;
        uint32_t v = 0;
        for (int i = 0; i < r.value_bytes; ++i) v |= (uint32_t)r.buf[r.pos++] << (8 * i);
        r.rle_value = v;
    }
    return true;
}

// One group of 8 values, LSB first (unpackGroup / refillPackedGroup).
bool unpack8(Rle& r, uint32_t* dst) {
    if (r.pos + r.width > r.end) return false;
    uint64_t buf = 0;
    int bits = 0;
    for (int i = 0; i < 8; ++i) {
        while (bits < r.width) {
            buf |= (uint64_t)r.buf[r.pos++] << bits;
            bits += 8;
        }
        dst[i] = (uint32_t)(buf & r.mask);
        buf >>= r.width;
        bits -= r.width;
    }
    return true;
}

// RleBitPackingReader.readInts(dst, 0, n) from a fresh reader.
int rle_decode(const uint8_t* buf, int64_t len, int width, int64_t n, uint32_t* out) {
    if (width < 0 || width > 32) return pq_fail("bit width out of range: " + std::to_string(width));
    if (width == 0) {
        for (int64_t i = 0; i < n; ++i) out[i] = 0;
        return VR_OK;
    }
    Rle r{buf, 0, len, width, (width + 7) / 8, width == 32 ? 0xFFFFFFFFu : ((1u << width) - 1)};
    int64_t o = 0;
    uint32_t group[8];
    while (o < n) {
        if (r.rle_left == 0 && r.packed_left == 0) {
            if (!run_header(r)) return pq_fail("RLE/bit-packed stream ended inside a run header");
            continue;
        }
        if (r.rle_left > 0) {
            const int64_t take = std::min(n - o, r.rle_left);
            for (int64_t i = 0; i < take; ++i) out[o + i] = r.rle_value;
            o += take;
            r.rle_left -= take;
        } else {
            if (!unpack8(r, group)) return pq_fail("RLE/bit-packed stream ended inside a bit-packed run");
            const int64_t take = std::min<int64_t>(std::min<int64_t>(8, r.packed_left), n - o);
            for (int64_t i = 0; i < take; ++i) out[o + i] = group[i];
            o += take;
            r.packed_left -= 8;  // a group cut short is the end of the read
        }
    }
    return VR_OK;
}

uint32_t ld_u32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

int bit_width_of(int max_value) {
    int w = 0;
    while (w < 32 && (max_value >> w) != 0) ++w;
    return w;
}

}  // namespace

extern "C" {

const char* orc_pq_last_error(void) { return g_pq_err.c_str(); }

int orc_rle_decode(const uint8_t* buf, int64_t len, int32_t bit_width, int64_t n, uint32_t* out) {
    return rle_decode(buf, len, bit_width, n, out);
}

int orc_pq_decode_page(const uint8_t* page, const vr_pq_page* d, void* out_data, uint8_t* out_validity,
                       int64_t* present_count) {
    const int64_t n = d->num_values;
    if (n < 0 || d->length < 0) return pq_fail("negative page size");
    const int vb = d->encoding == VR_PQ_RLE_DICTIONARY ? 4 : d->value_bytes;
    if (vb != 4 && vb != 8) return pq_fail("value bytes must be 4 or 8");
    std::vector<uint8_t> present(n, 1);
    int64_t values_start = 0, npresent = n;
    if (d->max_def_level > 0) {
        int64_t lstart, llen;
        if (d->v2) {
            lstart = 0;
            llen = d->levels_length;
        } else {
            if (d->length < 4) return pq_fail("v1 page shorter than its level length prefix");
            lstart = 4;
            llen = (int32_t)ld_u32(page);
        }
        if (llen < 0 || lstart + llen > d->length) return pq_fail("definition levels past the end of the page");
        values_start = lstart + llen;
        std::vector<uint32_t> lv(n);
        int rc = rle_decode(page + lstart, llen, bit_width_of(d->max_def_level), n, lv.data());
        if (rc) return rc;
        npresent = 0;
        for (int64_t i = 0; i < n; ++i) {
            present[i] = lv[i] == (uint32_t)d->max_def_level;
            npresent += present[i];
        }
    }
    std::vector<uint8_t> vals(npresent * vb);
    if (d->encoding == VR_PQ_RLE_DICTIONARY) {
        if (values_start >= d->length) return pq_fail("dictionary page without its id bit width");
        const int w = page[values_start];
        const int64_t s = values_start + 1;
        std::vector<uint32_t> ids(npresent);
        int rc = rle_decode(page + s, d->length - s, w, npresent, ids.data());
        if (rc) return rc;
        std::memcpy(vals.data(), ids.data(), npresent * 4);
    } else {
        if (values_start + npresent * vb > d->length) return pq_fail("PLAIN values past the end of the page");
        std::memcpy(vals.data(), page + values_start, npresent * vb);
    }
    uint8_t* out = static_cast<uint8_t*>(out_data);
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (present[i])
            std::memcpy(out + i * vb, vals.data() + (k++) * vb, vb);
        else
            std::memset(out + i * vb, 0, vb);
        if (out_validity) {
            if (present[i])
                out_validity[i >> 3] |= (uint8_t)(1u << (i & 7));
            else
                out_validity[i >> 3] &= (uint8_t)~(1u << (i & 7));
        }
    }
    if (present_count) *present_count = npresent;
    return VR_OK;
}

int orc_pq_plain_dictionary(const uint8_t* page, int64_t length, int32_t num_values, int32_t* offsets,
                            uint8_t* data, int64_t* data_bytes) {
    if (num_values < 0) return pq_fail("dictionary page: negative value count");
    int64_t src = 0, total = 0;
    for (int32_t i = 0; i < num_values; ++i) {
        if (src + 4 > length) return pq_fail("dictionary page: length prefix past the end of the page");
        const int32_t len = (int32_t)ld_u32(page + src);
        src += 4;
        if (len < 0 || len > length - src) return pq_fail("dictionary page: an entry past the end of the page");
        if (offsets) offsets[i] = (int32_t)total;
        if (data) std::memcpy(data + total, page + src, len);
        total += len;
        src += len;
    }
    if (offsets) offsets[num_values] = (int32_t)total;
    if (data_bytes) *data_bytes = total;
    return VR_OK;
}

// A column chunk's pages decoded on `threads` host threads, pages taken in
// turn from a shared counter, each into its own output as the reference's
// decoder produces one VectorBuffers per page: page k's slots at
// out_data + slot_base[k] values, its validity bitmap at
// out_validity + valid_base[k] bytes. The timed CPU baseline. Returns the
// first error; *seconds = wall time of the decode.
int orc_pq_decode_pages_threads(int32_t num_pages, const uint8_t* const* pages, const vr_pq_page* descs,
                                const int64_t* slot_base, const int64_t* valid_base, void* out_data,
                                uint8_t* out_validity, int32_t threads, double* seconds) {
    std::atomic<int32_t> next{0};
    std::atomic<int> err{VR_OK};
    const int vb = num_pages && descs[0].encoding == VR_PQ_RLE_DICTIONARY ? 4 : (num_pages ? descs[0].value_bytes : 4);
    auto work = [&]() {
        for (int32_t k; (k = next.fetch_add(1)) < num_pages;) {
            int64_t present = 0;
            const int rc = orc_pq_decode_page(pages[k], &descs[k], static_cast<uint8_t*>(out_data) + slot_base[k] * vb,
                                              out_validity + valid_base[k], &present);
            if (rc) {
                int expect = VR_OK;
                err.compare_exchange_strong(expect, rc);
                return;
            }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return err.load();
}

}  // extern "C"
