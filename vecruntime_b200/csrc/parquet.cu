// Parquet data pages -> Arrow columns on the device: the scan side of the
// aggregate (vr_pq_* in vrgpu.h). A column chunk's decompressed pages sit in
// device memory; one call decodes a run of them into one column:
//
//   1. k_pq_walk    one warp per (page, stream): the RLE / bit-packed hybrid
//                   run headers of the definition levels and of the
//                   dictionary ids, walked in order (each header's position
//                   depends on the previous run), into a run table;
//   2. k_pq_expand  one warp per run entry: levels become the bits of a
//                   present bitmap (level == max_def_level), ids go to a
//                   compact per-page array;
//   3. a CUB exclusive scan of the bitmap words' popcounts: a slot's rank
//                   among the present slots is its word's prefix plus the
//                   present bits below it;
//   4. k_pq_gather  four slots per thread: each slot's id or PLAIN value
//                   (the rank-th present value of its page), 0 at a null
//                   slot, and the validity bitmap.
//
// Reference: ParquetPageDecoder.decode (parquet/src/main/java/io/vecruntime/
// parquet/codec/ParquetPageDecoder.java:214-311) and RleBitPackingReader
// (RleBitPackingReader.java:117-392), for flat columns. Every read stays
// inside its page: headers and payloads are bounds-checked against their
// stream before they are read, and a malformed stream stops its walk with
// a reason the host reports.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "runtime.h"

namespace vr {
namespace {

// One run of a stream: `begin` = index of its first value in the stream,
// bit 31 set for a bit-packed run; `word` = the repeated value of an RLE run
// or the page byte offset of a bit-packed run's first group. A run's count
// is the next entry's begin minus its own (the walk writes a terminator).
struct RunEntry {
    uint32_t begin;
    uint32_t word;
};
constexpr uint32_t kPacked = 0x80000000u;
// A run longer than this is recorded as several entries (a bit-packed one at
// group boundaries: kChunk is a multiple of 8), so one warp expands at most
// kChunk values and a page of one long RLE run still spreads over warps.
constexpr int64_t kChunk = 4096;

enum PqReason : int32_t {
    PQ_OK = 0,
    PQ_LEVELS_SHORT = 1,    // the level stream ends or is malformed before num_values levels
    PQ_IDS_SHORT = 2,       // the id stream ends or is malformed before the present slots' ids
    PQ_PLAIN_SHORT = 3,     // PLAIN values past the end of the page
    PQ_BAD_WIDTH = 4,       // an id bit width above 32
    PQ_LEVELS_PAST_END = 5, // the levels' byte length runs past the page
    PQ_TOO_MANY_RUNS = 6,   // more runs than the run table's share for the stream
};

// A page as the kernels see it (host-filled; the walk fills the rest).
struct PqDev {
    const uint8_t* data;
    int64_t length;
    int64_t slot_base;       // first slot of the page in the call's column
    int64_t run_base[2];     // first run-table entry of the level / value stream
    int32_t run_cap[2];      // entries the stream may use (terminator included)
    int32_t num_values;
    int32_t max_def;
    int32_t v2;
    int32_t levels_length;
    int32_t encoding;
    int32_t value_bytes;
    // written by k_pq_walk
    int64_t values_start;    // first byte of the values region
    int32_t runs[2];         // runs recorded per stream
    int32_t decoded[2];      // values the runs cover (at most num_values)
    int32_t width[2];        // bit width per stream
    int32_t pad_;
};

// status[0] reason, [1] page (first error wins); [2..3] present count (u64)
__device__ void pq_fail(int32_t* status, int reason, int page) {
    if (atomicCAS(status, 0, reason) == 0) atomicExch(status + 1, page);
}

__device__ uint32_t ld_le(const uint8_t* p, int n) {
    uint32_t v = 0;
    for (int i = 0; i < n; ++i) v |= (uint32_t)__ldg(p + i) << (8 * i);
    return v;
}

__device__ int width_of(int max_value) { return max_value ? 32 - __clz(max_value) : 0; }

// Bytes [pos, pos + 16) of a page as two little-endian words, bytes at or
// past `end` read as 0 (and not loaded): 16 independent loads, one latency.
__device__ void load16(const uint8_t* base, int64_t pos, int64_t end, uint64_t& lo, uint64_t& hi) {
    lo = hi = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const uint64_t b = pos + i < end ? (uint64_t)__ldg(base + pos + i) : 0ull;
        if (i < 8) lo |= b << (8 * i);
        else hi |= b << (8 * (i - 8));
    }
}

// The run whose header would start at page position q, from the 9 bytes at
// q (x: bytes q..q+7, y: bytes q+8..): `step` = bytes to the next header
// (0: no valid run starts here within [q, end)), `nvals` = its values
// (clamped to 2^31 - 1), `word` = the RLE value or the page position of the
// bit-packed payload.
struct RunAt {
    uint32_t step;
    int32_t nvals;
    uint32_t word;
    bool packed;
};
__device__ RunAt run_at(uint64_t x, uint64_t y, int64_t q, int64_t end, int w, int vbytes, uint64_t vmask) {
    RunAt r{0u, 0, 0u, false};
    const int64_t avail = end - q;
    if (avail <= 0) return r;
    uint32_t h = 0;
    int hl = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {  // ULEB128, at most 5 bytes (as the reference reads it)
        const uint32_t b = (uint32_t)(x >> (8 * i)) & 0xFFu;
        h |= (b & 0x7Fu) << (7 * i);
        if (!(b & 0x80u)) {
            hl = i + 1;
            break;
        }
    }
    if (hl == 0 || hl > avail) return r;  // a header cut by the end of the stream
    const int64_t count = h >> 1;
    r.packed = h & 1;
    if (r.packed) {
        const int64_t bytes = count * w;
        if (hl + bytes > avail) return r;  // a bit-packed run past the end
        r.step = (uint32_t)(hl + bytes);
        r.nvals = (int32_t)(count * 8 < 0x7FFFFFFF ? count * 8 : 0x7FFFFFFF);
        r.word = (uint32_t)(q + hl);
    } else {
        if (hl + vbytes > avail) return r;  // an RLE value past the end
        const uint64_t z = (x >> (8 * hl)) | (y << (64 - 8 * hl));  // hl is 1..5
        r.step = (uint32_t)(hl + vbytes);
        r.nvals = (int32_t)(count < 0x7FFFFFFF ? count : 0x7FFFFFFF);
        r.word = (uint32_t)(z & vmask);
    }
    return r;
}

// The walk's state in lane 0: entries written, values covered, no room left.
struct Emit {
    RunEntry* runs;
    int32_t cap;
    int32_t k = 0;
    int64_t got = 0;
    bool full = false;
};

constexpr int kWin = 256;  // bytes a warp decodes at once in dense mode (8 per lane)
struct WinTable {
    uint16_t jump[2][kWin];  // 2^r-hop successor within the window (>= kWin: leaves it)
    uint8_t mark[kWin];      // on the chain from the window's first byte
};

// Inclusive warp prefix sum of a 64-bit value.
__device__ int64_t warp_scan(int64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Walks the run headers of [pos, end) in order until `need` values are
// covered or the stream stops; the whole warp calls it and lane 0 writes the
// run table. A header's position follows from the previous run, so the walk
// is a chain. Two modes, switched by the runs just seen:
//   sparse -- lane 0 reads one header at a time (long bit-packed runs: the
//             next header is far away, one step per run);
//   dense  -- the warp decodes, in parallel, a run at every byte position of
//             the next 256 bytes into shared memory, and lane 0 follows the
//             chain through that table (short runs, e.g. the definition
//             levels of a column with scattered nulls: a table read and a few
//             register operations per run instead of a dependent parse).
// Returns the values covered, or -1 when the run table had no room.
__device__ int64_t walk_stream(const uint8_t* base, int64_t pos, int64_t end, int w, int64_t need,
                               RunEntry* runs, int32_t cap, int32_t& nruns, WinTable& T) {
    const int lane = threadIdx.x & 31;
    Emit E{runs, cap};
    if (w == 0) {  // every value is 0 and no byte is read
        if (lane == 0) {
            if (need > 0 && cap >= 2) {
                runs[0] = RunEntry{0u, 0u};
                E.k = 1;
                E.got = need;
            }
            runs[E.k].begin = (uint32_t)E.got;
            nruns = E.k;
        }
        return __shfl_sync(0xffffffffu, E.got, 0);
    }
    const int vbytes = (w + 7) >> 3;
    const uint64_t vmask = vbytes == 4 ? 0xFFFFFFFFull : ((1ull << (8 * vbytes)) - 1);
    bool dense = false, stop = false;
    int64_t got = 0;
    while (!stop && got < need && pos < end) {  // uniform: lane 0's state is broadcast each step
        // the next 8 KiB of the stream into L2 while lane 0 works through this
        // part (every 128-byte line, two per lane; addresses inside the stream
        // only): each step of the chain then waits on L2, not DRAM
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int64_t a = pos + 128 + 256 * lane + 128 * j;
            if (a < end) asm volatile("prefetch.global.L2 [%0];" ::"l"(base + a));
        }
        if (!dense) {
            // stride speculation: lane 0 reads the run at pos (step S); lane l
            // reads the one that would start at pos + l * S. Writers emit long
            // bit-packed runs of one size, so the guesses hold and one step
            // covers 32 runs; lanes 0..m are right, m being the first lane
            // whose run is not S bytes long (its own start was still right).
            RunAt r{0u, 0, 0u, false};
            uint64_t lo, hi;
            if (lane == 0) {
                load16(base, pos, end, lo, hi);
                r = run_at(lo, hi, pos, end, w, vbytes, vmask);
            }
            const uint32_t S = __shfl_sync(0xffffffffu, r.step, 0);
            if (S == 0) {
                if (lane == 0) stop = true;
            } else {
                const int64_t q = pos + (int64_t)lane * S;
                if (lane > 0 && q < end) {
                    load16(base, q, end, lo, hi);
                    r = run_at(lo, hi, q, end, w, vbytes, vmask);
                }
                const uint32_t same = __ballot_sync(0xffffffffu, r.step == S);
                const int m = ~same ? __ffs(~same) - 1 : 31;
                const bool mine = lane <= m && r.step != 0;
                const int64_t got0 = __shfl_sync(0xffffffffu, E.got, 0);
                const int32_t k0 = __shfl_sync(0xffffffffu, E.k, 0);
                const int64_t vsum = mine ? r.nvals : 0;
                const int64_t vincl = warp_scan(vsum);
                const int64_t b = got0 + vincl - vsum;
                const int64_t cover = mine && b < need ? (r.nvals < need - b ? r.nvals : need - b) : 0;
                const int64_t nent = (cover + kChunk - 1) / kChunk;
                const int64_t eincl = warp_scan(nent);
                const int64_t etotal = __shfl_sync(0xffffffffu, eincl, 31);
                const int64_t vtotal = __shfl_sync(0xffffffffu, vincl, 31);
                const bool full = k0 + etotal + 1 > cap;
                if (!full) {
                    int64_t e = k0 + eincl - nent;
                    for (int64_t off = 0; off < cover; off += kChunk)
                        runs[e++] = RunEntry{(uint32_t)(b + off) | (r.packed ? kPacked : 0u),
                                             r.packed ? r.word + (uint32_t)(off / 8 * w) : r.word};
                }
                const uint32_t stm = __shfl_sync(0xffffffffu, r.step, m);
                if (lane == 0) {
                    if (full) {
                        E.full = true;
                        stop = true;
                    } else {
                        E.k = (int32_t)(k0 + etotal);
                        E.got = got0 + vtotal;
                        if (stm == 0) {
                            stop = true;  // lane m's run is malformed, or the stream ended there
                        } else {
                            pos = pos + (int64_t)m * S + stm;
                            dense = stm < 32;
                        }
                    }
                }
            }
        } else {
            // this lane's 8 positions of the window: their runs stay in
            // registers; only the jump table and the marks are shared
            const int64_t ws = pos;
            uint64_t lo, hi;
            load16(base, ws + 8 * lane, end, lo, hi);
            RunAt R[8];
            uint32_t J[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int sh = 8 * j;
                const uint64_t x = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
                const uint64_t y = sh ? hi >> sh : hi;
                const int q = 8 * lane + j;
                R[j] = run_at(x, y, ws + q, end, w, vbytes, vmask);
                J[j] = R[j].step == 0 ? 0xFFFFu : (q + R[j].step < 0xFFFFu ? q + R[j].step : 0xFFFEu);
                T.jump[0][q] = (uint16_t)J[j];
                T.mark[q] = q == 0;
            }
            __syncwarp();
            // the chain through the window, in parallel: pointer doubling marks
            // every position reachable from byte 0 (a run is at least one byte,
            // so 8 rounds cover the 256 bytes); chain order is position order.
            // Each phase reads all 8 positions before it writes any, so the
            // reads overlap.
            int cur = 0;
            for (int r = 0; r < 8; ++r) {
                uint8_t mk[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) mk[j] = T.mark[8 * lane + j];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (mk[j] && J[j] < kWin) T.mark[J[j]] = 1;
                if (r == 7) break;  // the last round's jumps are not needed
                uint32_t N2[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) N2[j] = J[j] < kWin ? T.jump[cur][J[j]] : J[j];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    J[j] = N2[j];
                    T.jump[cur ^ 1][8 * lane + j] = (uint16_t)N2[j];
                }
                __syncwarp();
                cur ^= 1;
            }
            __syncwarp();
            bool on[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) on[j] = T.mark[8 * lane + j] != 0;
            // this lane's chain runs: values, entries (runs split at kChunk), the last one
            const int64_t got0 = __shfl_sync(0xffffffffu, E.got, 0);
            const int32_t k0 = __shfl_sync(0xffffffffu, E.k, 0);
            int64_t vsum = 0;
            bool bad = false;
            int last = -1;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (!on[j]) continue;
                if (R[j].step == 0) bad = true;  // the chain stops here (malformed, or the stream ended)
                else {
                    vsum += R[j].nvals;
                    last = 8 * lane + j;
                }
            }
            const int64_t vincl = warp_scan(vsum);
            const int64_t begin = got0 + vincl - vsum;  // values before this lane's first chain run
            int64_t nent = 0;
            {
                int64_t b = begin;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (!on[j] || R[j].step == 0) continue;
                    if (b < need) {
                        const int64_t cover = R[j].nvals < need - b ? R[j].nvals : need - b;
                        nent += (cover + kChunk - 1) / kChunk;
                    }
                    b += R[j].nvals;
                }
            }
            const int64_t eincl = warp_scan(nent);
            const int64_t etotal = __shfl_sync(0xffffffffu, eincl, 31);
            const int64_t vtotal = __shfl_sync(0xffffffffu, vincl, 31);
            const bool full = k0 + etotal + 1 > cap;
            if (!full) {
                int64_t e = k0 + eincl - nent;
                int64_t b = begin;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (!on[j] || R[j].step == 0) continue;
                    const int64_t cover = b < need ? (R[j].nvals < need - b ? R[j].nvals : need - b) : 0;
                    for (int64_t off = 0; off < cover; off += kChunk)
                        runs[e++] = RunEntry{(uint32_t)(b + off) | (R[j].packed ? kPacked : 0u),
                                             R[j].packed ? R[j].word + (uint32_t)(off / 8 * w) : R[j].word};
                    b += R[j].nvals;
                }
            }
            // the chain's exit: past its last run in the window
            int qlast = last;
            uint32_t slast = 0;  // the step of this lane's last chain run
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (8 * lane + j == last) slast = R[j].step;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) qlast = max(qlast, __shfl_xor_sync(0xffffffffu, qlast, d));
            const int owner = qlast >= 0 ? qlast >> 3 : 0;
            const uint32_t stl = __shfl_sync(0xffffffffu, slast, owner);
            const bool any_bad = __any_sync(0xffffffffu, bad);
            if (lane == 0) {
                if (full) {
                    E.full = true;
                    stop = true;
                } else {
                    E.k = (int32_t)(k0 + etotal);
                    E.got = got0 + vtotal;
                    stop = any_bad;
                    if (qlast >= 0) {
                        const int64_t exit = qlast + (int64_t)stl;
                        pos = ws + exit;
                        dense = exit < kWin + 64;  // the chain left the window by a long jump: back to sparse
                    } else {
                        stop = true;
                    }
                }
            }
            __syncwarp();
        }
        pos = __shfl_sync(0xffffffffu, pos, 0);
        got = __shfl_sync(0xffffffffu, E.got, 0);
        stop = __shfl_sync(0xffffffffu, stop, 0);
        dense = __shfl_sync(0xffffffffu, dense, 0);
    }
    if (lane == 0) {
        if (E.full) {
            nruns = 0;
        } else {
            runs[E.k].begin = (uint32_t)(E.got < need ? E.got : need);  // terminator: the end of the last run
            nruns = E.k;
        }
    }
    const bool full = __shfl_sync(0xffffffffu, E.full, 0);
    return full ? -1 : (got < need ? got : need);
}

// Slots per entry of the slot -> page table the gather starts its page
// lookup from (entry j: the page holding slot j * kSlotBlock).
constexpr int kSlotBlock = 1024;

__global__ void k_pq_walk(PqDev* __restrict__ pages, RunEntry* __restrict__ runs, int32_t* __restrict__ status,
                          int32_t* __restrict__ page_of_block) {
    __shared__ WinTable tables[2];
    const int p = blockIdx.x;
    const int s = threadIdx.x >> 5;  // warp 0: definition levels, warp 1: values
    const bool lead = (threadIdx.x & 31) == 0;
    WinTable& T = tables[s];
    PqDev& d = pages[p];
    if (s == 0) {  // this page's entries of the slot -> page table
        const int64_t lo = d.slot_base, hi = d.slot_base + d.num_values;
        for (int64_t j = (lo + kSlotBlock - 1) / kSlotBlock + (threadIdx.x & 31); j * kSlotBlock < hi; j += 32)
            page_of_block[j] = p;
    }
    const uint8_t* base = d.data;
    int64_t lstart = 0, llen = 0;
    if (d.max_def > 0) {
        if (d.v2) {
            llen = d.levels_length;
        } else {
            if (d.length < 4) {
                if (s == 0 && lead) pq_fail(status, PQ_LEVELS_PAST_END, p);
                return;
            }
            lstart = 4;
            llen = (int32_t)ld_le(base, 4);
        }
        if (llen < 0 || lstart + llen > d.length) {
            if (s == 0 && lead) pq_fail(status, PQ_LEVELS_PAST_END, p);
            return;
        }
    }
    const int64_t vstart = lstart + llen;
    int32_t nr = 0;
    if (s == 0) {
        if (lead) d.values_start = vstart;
        if (d.max_def == 0) {
            if (lead) {
                d.runs[0] = 0;
                d.decoded[0] = d.num_values;
            }
            return;
        }
        const int w = width_of(d.max_def);
        const int64_t got = walk_stream(base, lstart, lstart + llen, w, d.num_values, runs + d.run_base[0],
                                        d.run_cap[0], nr, T);
        if (lead) {
            d.width[0] = w;
            d.runs[0] = nr;
            d.decoded[0] = got < 0 ? 0 : (int32_t)got;
            if (got < 0) pq_fail(status, PQ_TOO_MANY_RUNS, p);
            else if (got < d.num_values) pq_fail(status, PQ_LEVELS_SHORT, p);
        }
        return;
    }
    if (d.encoding != VR_PQ_RLE_DICTIONARY) {  // PLAIN: the values region is the values
        if (lead) {
            d.runs[1] = 0;
            const int64_t avail = (d.length - vstart) / d.value_bytes;
            d.decoded[1] = (int32_t)(avail < d.num_values ? (avail < 0 ? 0 : avail) : d.num_values);
        }
        return;
    }
    if (vstart >= d.length) {  // no id bit width byte
        if (lead) {
            d.runs[1] = 0;
            d.decoded[1] = 0;
        }
        return;
    }
    const int w = __ldg(base + vstart);
    if (w > 32) {
        if (lead) {
            d.runs[1] = 0;
            d.decoded[1] = 0;
            pq_fail(status, PQ_BAD_WIDTH, p);
        }
        return;
    }
    const int64_t got = walk_stream(base, vstart + 1, d.length, w, d.num_values, runs + d.run_base[1], d.run_cap[1],
                                    nr, T);
    if (lead) {
        d.width[1] = w;
        d.runs[1] = nr;
        d.decoded[1] = got < 0 ? 0 : (int32_t)got;
        if (got < 0) pq_fail(status, PQ_TOO_MANY_RUNS, p);
    }
}

// A level run entry's present slots (level == max_def) as bits of the call's
// bitmap (zeroed before): an RLE run sets whole words with plain stores (no
// other run touches a word its slots cover) and its end words with atomic
// ORs; a bit-packed run's groups of 8 levels become 8 bits each, ORed into
// the one or two words they land in.
__device__ void levels_to_bits(const PqDev& d, const RunEntry& e, int64_t slot0, int64_t cnt, bool packed, int w,
                               uint32_t* bits, int lane) {
    if (!packed) {
        if (e.word != (uint32_t)d.max_def) return;
        const int64_t first = slot0 >> 5, last = (slot0 + cnt - 1) >> 5;
        for (int64_t wd = first + lane; wd <= last; wd += 32) {
            uint32_t m = 0xFFFFFFFFu;
            if (wd == first) m &= 0xFFFFFFFFu << (slot0 & 31);
            if (wd == last) m &= 0xFFFFFFFFu >> (31 - ((slot0 + cnt - 1) & 31));
            if (m == 0xFFFFFFFFu) bits[wd] = m;
            else atomicOr(&bits[wd], m);
        }
        return;
    }
    const uint8_t* payload = d.data + e.word;
    const uint64_t mask = w == 32 ? 0xFFFFFFFFull : ((1ull << w) - 1);
    const int64_t ng = (cnt + 7) >> 3;
    for (int64_t g = lane; g < ng; g += 32) {
        const uint8_t* src = payload + g * w;
        uint64_t acc = 0;
        int nbits = 0, nb = 0;
        uint32_t b8 = 0;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            while (nbits < w) {
                acc |= (uint64_t)__ldg(src + nb) << nbits;
                ++nb;
                nbits += 8;
            }
            if (8 * g + v < cnt && (uint32_t)(acc & mask) == (uint32_t)d.max_def) b8 |= 1u << v;
            acc >>= w;
            nbits -= w;
        }
        if (!b8) continue;
        const int64_t s0 = slot0 + 8 * g;
        const int off = (int)(s0 & 31);
        atomicOr(&bits[s0 >> 5], b8 << off);
        if (off > 24) atomicOr(&bits[(s0 >> 5) + 1], b8 >> (32 - off));
    }
}

// One warp per run entry, lanes over its values (an RLE run) or its groups
// of 8 (a bit-packed run). present: a byte per slot;
// bits: the call's present bitmap; compact: a page's ids at slot_base +
// value index (the gather moves them to their slots).
__global__ void k_pq_expand(const PqDev* __restrict__ pages, int page0, const RunEntry* __restrict__ runs,
                            uint32_t* __restrict__ bits, int32_t* __restrict__ compact) {
    __shared__ uint32_t stage[8][256];  // 256 threads per block: one 256-value stage per warp
    const int lane = threadIdx.x & 31;
    uint32_t* sb = stage[threadIdx.x >> 5];
    // blocks (x, page, stream): the page's stream's runs over gridDim.x blocks of 8 warps
    const int64_t warp = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int64_t nwarps = (int64_t)gridDim.x * 8;
    const int p = page0 + (int)blockIdx.y;
    const int s = (int)blockIdx.z;
    const PqDev& d = pages[p];
    {
        {
            const int nr = d.runs[s];
            if (s == 1 && d.encoding != VR_PQ_RLE_DICTIONARY) return;
            const RunEntry* R = runs + d.run_base[s];
            const int w = d.width[s];
            for (int64_t k = warp; k < nr; k += nwarps) {
                const RunEntry e = R[k];
                const int64_t b0 = e.begin & ~kPacked;
                const int64_t cnt = (int64_t)(R[k + 1].begin & ~kPacked) - b0;
                const bool packed = (e.begin & kPacked) != 0;
                const int64_t slot0 = d.slot_base + b0;
                if (s == 0) {  // levels: the present slots' bits of the call's bitmap
                    levels_to_bits(d, e, slot0, cnt, packed, w, bits, lane);
                    continue;
                }
                auto put = [&](int64_t i, uint32_t v) { compact[slot0 + i] = (int32_t)v; };
                if (!packed) {
                    for (int64_t i = lane; i < cnt; i += 32) put(i, e.word);
                    continue;
                }
                // bit-packed: each lane unpacks one group of 8 (its w bytes,
                // LSB first) into the warp's stage, then the warp stores the
                // 256 values in order (coalesced)
                const uint8_t* payload = d.data + e.word;
                const uint64_t m = w == 32 ? 0xFFFFFFFFull : ((1ull << w) - 1);
                const int64_t ng = (cnt + 7) >> 3;
                for (int64_t g0 = 0; g0 < ng; g0 += 32) {
                    const int64_t g = g0 + lane;
                    if (g < ng) {
                        const uint8_t* src = payload + g * w;
                        uint64_t acc = 0;
                        int bits = 0, nb = 0;
#pragma unroll
                        for (int v = 0; v < 8; ++v) {
                            while (bits < w) {
                                acc |= (uint64_t)__ldg(src + nb) << bits;
                                ++nb;
                                bits += 8;
                            }
                            sb[8 * lane + v] = (uint32_t)(acc & m);
                            acc >>= w;
                            bits -= w;
                        }
                    }
                    __syncwarp();
                    const int64_t here = cnt - 8 * g0 < 256 ? cnt - 8 * g0 : 256;
                    for (int t = lane; t < here; t += 32) put(8 * g0 + t, sb[t]);
                    __syncwarp();
                }
            }
        }
    }
}

struct PopCount {
    __device__ uint32_t operator()(uint32_t x) const { return (uint32_t)__popc(x); }
};

// The page of slot i: the last page whose slot_base <= i, found from the
// table entry of i's slot block by stepping forward over the pages that
// start inside the block.
__device__ int page_at(const PqDev* pages, int num_pages, const int32_t* page_of_block, int64_t i) {
    int p = page_of_block[i / kSlotBlock];
    while (p + 1 < num_pages && pages[p + 1].slot_base <= i) ++p;
    return p;
}

// Four consecutive slots per thread in a grid-stride loop (a block covers
// 1,024 slots per step): the 4 slots share one bitmap word, so a thread
// loads the word and its prefix once, finds each slot's rank with a
// popcount, reads the 4 values (consecutive ranks of one page, or the
// page's PLAIN values) and stores them with one 16-byte store where the
// column is aligned. Lanes 8k..8k+7 of a warp cover one 32-slot validity
// word, combined by shuffles. The present count is summed per block and
// added once per block.
__global__ void k_pq_gather(const PqDev* __restrict__ pages, int num_pages, int64_t n,
                            const uint32_t* __restrict__ bits, const uint32_t* __restrict__ wpre,
                            const int32_t* __restrict__ compact, uint8_t* __restrict__ out, int vb,
                            uint8_t* __restrict__ validity, int32_t* __restrict__ status,
                            const int32_t* __restrict__ page_of_block) {
    __shared__ unsigned long long block_present;
    if (threadIdx.x == 0) block_present = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const bool aligned = ((uintptr_t)out & 15) == 0;
    unsigned long long mine = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * 4;
    for (int64_t first = (int64_t)blockIdx.x * blockDim.x * 4; first < n; first += stride) {
        const int64_t i0 = first + 4 * (int64_t)threadIdx.x;
        uint32_t nib = 0;
        if (i0 < n) {
            const uint32_t wbits = bits[i0 >> 5];
            const uint32_t wp = wpre[i0 >> 5];
            int p = page_at(pages, num_pages, page_of_block, i0);
            uint64_t v[4] = {0, 0, 0, 0};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t i = i0 + j;
                if (i >= n) break;
                while (p + 1 < num_pages && pages[p + 1].slot_base <= i) ++p;
                const PqDev& d = pages[p];
                const bool levels = d.max_def > 0;
                bool valid = true;
                int64_t r = i - d.slot_base;
                if (levels) {
                    // a slot's rank among the call's present slots: its word's
                    // prefix plus the present bits below it in the word
                    const int64_t sb = d.slot_base;
                    const int64_t rank0 = (int64_t)wpre[sb >> 5] + __popc(bits[sb >> 5] & ((1u << (sb & 31)) - 1u));
                    valid = ((wbits >> (i & 31)) & 1u) != 0;
                    r = (int64_t)wp + __popc(wbits & ((1u << (i & 31)) - 1u)) - rank0;
                }
                if (!valid) continue;
                nib |= 1u << j;
                if (r >= d.decoded[1]) {
                    pq_fail(status, d.encoding == VR_PQ_RLE_DICTIONARY ? PQ_IDS_SHORT : PQ_PLAIN_SHORT, p);
                } else if (d.encoding == VR_PQ_RLE_DICTIONARY) {
                    v[j] = (uint32_t)compact[d.slot_base + r];
                } else {
                    const uint8_t* src = d.data + d.values_start + r * vb;
                    uint64_t x = 0;
                    for (int b = 0; b < vb; ++b) x |= (uint64_t)__ldg(src + b) << (8 * b);
                    v[j] = x;
                }
            }
            if (aligned && i0 + 4 <= n) {
                if (vb == 4) {
                    *reinterpret_cast<uint4*>(out + i0 * 4) =
                        make_uint4((uint32_t)v[0], (uint32_t)v[1], (uint32_t)v[2], (uint32_t)v[3]);
                } else {
                    uint4* o = reinterpret_cast<uint4*>(out + i0 * 8);
                    o[0] = make_uint4((uint32_t)v[0], (uint32_t)(v[0] >> 32), (uint32_t)v[1], (uint32_t)(v[1] >> 32));
                    o[1] = make_uint4((uint32_t)v[2], (uint32_t)(v[2] >> 32), (uint32_t)v[3], (uint32_t)(v[3] >> 32));
                }
            } else {
                for (int j = 0; j < 4 && i0 + j < n; ++j)
                    for (int b = 0; b < vb; ++b) out[(i0 + j) * vb + b] = (uint8_t)(v[j] >> (8 * b));
            }
        }
        // the 32-slot validity word of lanes 8k..8k+7
        uint32_t wv = nib << (4 * (lane & 7));
        wv |= __shfl_xor_sync(0xffffffffu, wv, 1);
        wv |= __shfl_xor_sync(0xffffffffu, wv, 2);
        wv |= __shfl_xor_sync(0xffffffffu, wv, 4);
        if ((lane & 7) == 0 && i0 < n) {
            if (validity) {
                const int64_t nbytes = (n + 7) >> 3;
                for (int j = 0; j < 4 && (i0 >> 3) + j < nbytes; ++j) validity[(i0 >> 3) + j] = (uint8_t)(wv >> (8 * j));
            }
            mine += __popc(wv);
        }
    }
    for (int d = 16; d > 0; d >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, d);
    if (lane == 0 && mine) atomicAdd(&block_present, mine);
    __syncthreads();
    if (threadIdx.x == 0 && block_present)
        atomicAdd(reinterpret_cast<unsigned long long*>(status + 2), block_present);
}

const char* reason_text(int r) {
    switch (r) {
        case PQ_LEVELS_SHORT: return "the definition-level stream ends or is malformed before the page's slots";
        case PQ_IDS_SHORT: return "the dictionary-id stream ends or is malformed before the page's present slots";
        case PQ_PLAIN_SHORT: return "PLAIN values past the end of the page";
        case PQ_BAD_WIDTH: return "a dictionary-id bit width above 32";
        case PQ_LEVELS_PAST_END: return "the definition levels run past the end of the page";
        case PQ_TOO_MANY_RUNS: return "more runs than the stream's bytes allow";
        default: return "malformed page";
    }
}

}  // namespace
}  // namespace vr

using namespace vr;

struct vr_pq_decoder {
    int device = 0;
    cudaStream_t own = nullptr;
    int64_t max_values = 0, max_bytes = 0;
    PqDev* pages_dev = nullptr;
    PqDev* pages_host = nullptr;  // pinned
    int pages_cap = 0;
    RunEntry* runs = nullptr;
    int64_t runs_cap = 0;
    uint32_t* bits = nullptr;  // the call's present slots, one bit per slot
    uint32_t* wpre = nullptr;  // per bitmap word: present slots in the words before it
    int32_t* page_of_block = nullptr;  // slot block -> page, one entry per kSlotBlock slots
    int32_t* compact = nullptr;
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    int32_t* status_dev = nullptr;
    int32_t* status_host = nullptr;  // pinned: reason, page, present (u64)
    cudaEvent_t done = nullptr;
    bool pending = false;
    int last_pages = 0;
};

namespace {

int pq_err(int code, const std::string& msg) {
    vr::set_thread_error(msg);
    return code;
}

int cuda_err(cudaError_t e, const char* what) {
    return pq_err(VR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Run-table entries a stream of a page may need: at most one per two bytes
// of the page (a run is a header and at least one byte of value or
// payload), plus the entries long runs split into, plus the terminator.
int64_t stream_cap(const vr_pq_page& pg) {
    const int64_t n = pg.num_values;
    return std::min<int64_t>(n, pg.length / 2 + n / kChunk + 2) + 2;
}

void free_all(vr_pq_decoder* d) {
    cudaFree(d->pages_dev);
    cudaFreeHost(d->pages_host);
    cudaFree(d->runs);
    cudaFree(d->bits);
    cudaFree(d->wpre);
    cudaFree(d->page_of_block);
    cudaFree(d->compact);
    cudaFree(d->scan_tmp);
    cudaFree(d->status_dev);
    cudaFreeHost(d->status_host);
    if (d->done) cudaEventDestroy(d->done);
    if (d->own) cudaStreamDestroy(d->own);
}

}  // namespace

extern "C" {

int vr_pq_create(int32_t device, int64_t max_values, int64_t max_bytes, vr_pq_decoder** out) {
    if (!out || max_values < 0 || max_bytes < 0 || max_values >= ((int64_t)1 << 31))
        return pq_err(VR_ERR_INVALID, "vr_pq_create: bad argument (max_values must be below 2^31)");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_err(e, "vr_pq_create");
    auto* d = new vr_pq_decoder;
    d->device = device;
    d->max_values = max_values;
    d->max_bytes = max_bytes;
    const size_t n = (size_t)std::max<int64_t>(max_values, 1);
    bool ok = cudaStreamCreateWithFlags(&d->own, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&d->done, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&d->bits, (n / 32 + 2) * 4) == cudaSuccess &&
              cudaMalloc(&d->wpre, (n / 32 + 2) * 4) == cudaSuccess &&
              cudaMalloc(&d->page_of_block, (n / kSlotBlock + 2) * 4) == cudaSuccess &&
              cudaMalloc(&d->compact, n * 4) == cudaSuccess && cudaMalloc(&d->status_dev, 16) == cudaSuccess &&
              cudaMallocHost(&d->status_host, 16) == cudaSuccess;
    if (ok) {
        auto it = thrust::make_transform_iterator(static_cast<const uint32_t*>(d->bits), PopCount());
        ok = cub::DeviceScan::ExclusiveSum(nullptr, d->scan_bytes, it, d->wpre, (int)(n / 32 + 2)) == cudaSuccess &&
             cudaMalloc(&d->scan_tmp, std::max<size_t>(d->scan_bytes, 16)) == cudaSuccess;
    }
    if (!ok) {
        free_all(d);
        delete d;
        cudaGetLastError();
        return pq_err(VR_ERR_OOM, "vr_pq_create: device allocation refused");
    }
    std::memset(d->status_host, 0, 16);
    *out = d;
    return VR_OK;
}

int vr_pq_decode(vr_pq_decoder* d, int32_t num_pages, const vr_pq_page* pages, void* out_data,
                 uint8_t* out_validity, void* stream) {
    if (!d || num_pages < 0 || (num_pages > 0 && (!pages || !out_data)))
        return pq_err(VR_ERR_INVALID, "vr_pq_decode: null argument");
    cudaSetDevice(d->device);
    if (d->pending) {  // the pinned descriptors and status belong to the last call until it is done
        cudaError_t e = cudaEventSynchronize(d->done);
        if (e != cudaSuccess) return cuda_err(e, "vr_pq_decode");
    }
    int64_t slots = 0, bytes = 0, runs = 0;
    bool levels = false;
    const int enc = num_pages ? pages[0].encoding : 0;
    const int vb = enc == VR_PQ_RLE_DICTIONARY ? 4 : (num_pages ? pages[0].value_bytes : 4);
    for (int i = 0; i < num_pages; ++i) {
        const vr_pq_page& pg = pages[i];
        const std::string where = "vr_pq_decode: page " + std::to_string(i) + ": ";
        if (!pg.data || pg.length < 0 || pg.num_values < 0 || pg.max_def_level < 0 || pg.levels_length < 0)
            return pq_err(VR_ERR_INVALID, where + "bad descriptor");
        if (pg.encoding != VR_PQ_PLAIN && pg.encoding != VR_PQ_RLE_DICTIONARY)
            return pq_err(VR_ERR_UNSUPPORTED, where + "encoding other than PLAIN or RLE_DICTIONARY");
        if (pg.encoding != enc)
            return pq_err(VR_ERR_INVALID, where + "every page of one call must have the same encoding");
        if (enc == VR_PQ_PLAIN && pg.value_bytes != vb)
            return pq_err(VR_ERR_INVALID, where + "PLAIN pages of one call must have one value width");
        if (vb != 4 && vb != 8) return pq_err(VR_ERR_UNSUPPORTED, where + "PLAIN values of 4 or 8 bytes only");
        if (pg.length >= ((int64_t)1 << 32)) return pq_err(VR_ERR_UNSUPPORTED, where + "a page of 4 GiB or more");
        levels |= pg.max_def_level > 0;
        slots += pg.num_values;
        bytes += pg.length;
        runs += 2 * stream_cap(pg);
    }
    if (slots > d->max_values || bytes > d->max_bytes)
        return pq_err(VR_ERR_INVALID, "vr_pq_decode: more slots or page bytes than the decoder was created for");
    if (levels && !out_validity)
        return pq_err(VR_ERR_INVALID, "vr_pq_decode: pages with definition levels need a validity buffer");
    cudaStream_t st = stream ? (cudaStream_t)stream : d->own;
    // grow the descriptor and run tables (rare: once per larger call)
    if (num_pages > d->pages_cap) {
        cudaStreamSynchronize(st);
        cudaFree(d->pages_dev);
        cudaFreeHost(d->pages_host);
        d->pages_dev = nullptr;
        d->pages_host = nullptr;
        const int cap = std::max(num_pages, 2 * d->pages_cap);
        if (cudaMalloc(&d->pages_dev, sizeof(PqDev) * cap) != cudaSuccess ||
            cudaMallocHost(&d->pages_host, sizeof(PqDev) * cap) != cudaSuccess) {
            d->pages_cap = 0;
            cudaGetLastError();
            return pq_err(VR_ERR_OOM, "vr_pq_decode: descriptor allocation refused");
        }
        d->pages_cap = cap;
    }
    if (runs > d->runs_cap) {
        cudaStreamSynchronize(st);
        cudaFree(d->runs);
        d->runs = nullptr;
        const int64_t cap = std::max(runs, d->runs_cap + d->runs_cap / 2);
        if (cudaMalloc(&d->runs, sizeof(RunEntry) * cap) != cudaSuccess) {
            d->runs_cap = 0;
            cudaGetLastError();
            return pq_err(VR_ERR_OOM, "vr_pq_decode: run table allocation refused");
        }
        d->runs_cap = cap;
    }
    int64_t slot = 0, rb = 0;
    for (int i = 0; i < num_pages; ++i) {
        const vr_pq_page& pg = pages[i];
        PqDev& h = d->pages_host[i];
        std::memset(&h, 0, sizeof(h));
        h.data = pg.data;
        h.length = pg.length;
        h.slot_base = slot;
        h.num_values = pg.num_values;
        h.max_def = pg.max_def_level;
        h.v2 = pg.v2;
        h.levels_length = pg.levels_length;
        h.encoding = pg.encoding;
        h.value_bytes = vb;
        const int64_t cap = stream_cap(pg);
        for (int s = 0; s < 2; ++s) {
            h.run_base[s] = rb;
            h.run_cap[s] = (int32_t)cap;
            rb += cap;
        }
        slot += pg.num_values;
    }
    d->pending = false;
    d->last_pages = num_pages;
    std::memset(d->status_host, 0, 16);
    cudaError_t e = cudaMemsetAsync(d->status_dev, 0, 16, st);
    if (num_pages > 0 && e == cudaSuccess)
        e = cudaMemcpyAsync(d->pages_dev, d->pages_host, sizeof(PqDev) * num_pages, cudaMemcpyHostToDevice, st);
    if (slots > 0 && e == cudaSuccess) {
        const int64_t words = (slots + 31) / 32;
        if (levels) e = cudaMemsetAsync(d->bits, 0, (size_t)words * 4, st);
        if (e == cudaSuccess) {
            k_pq_walk<<<num_pages, 64, 0, st>>>(d->pages_dev, d->runs, d->status_dev, d->page_of_block);
            // blocks per (page, stream): enough warps for the largest page's
            // runs, ~1 warp per 1,024 slots, 1 to 64 blocks of 8 warps
            int64_t most = 1;
            for (int i = 0; i < num_pages; ++i) most = std::max<int64_t>(most, pages[i].num_values);
            const unsigned bx = (unsigned)std::min<int64_t>(64, std::max<int64_t>(1, (most + 8191) / 8192));
            for (int p0 = 0; p0 < num_pages && e == cudaSuccess; p0 += 65535) {
                const unsigned np = (unsigned)std::min(65535, num_pages - p0);
                k_pq_expand<<<dim3(bx, np, 2), 256, 0, st>>>(d->pages_dev, p0, d->runs, d->bits, d->compact);
                e = cudaGetLastError();
            }
        }
        if (levels && e == cudaSuccess) {
            auto it = thrust::make_transform_iterator(static_cast<const uint32_t*>(d->bits), PopCount());
            size_t tb = d->scan_bytes;
            e = cub::DeviceScan::ExclusiveSum(d->scan_tmp, tb, it, d->wpre, (int)words, st);
        }
        if (e == cudaSuccess) {
            const int64_t blocks = std::min<int64_t>((slots + 255) / 256, 148 * 16);
            k_pq_gather<<<(unsigned)blocks, 256, 0, st>>>(d->pages_dev, num_pages, slots, d->bits, d->wpre,
                                                          d->compact, static_cast<uint8_t*>(out_data), vb,
                                                          out_validity, d->status_dev, d->page_of_block);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d->status_host, d->status_dev, 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(d->done, st);
    if (e != cudaSuccess) return cuda_err(e, "vr_pq_decode");
    d->pending = true;
    return VR_OK;
}

int vr_pq_sync(vr_pq_decoder* d, int64_t* present) {
    if (!d) return pq_err(VR_ERR_INVALID, "vr_pq_sync: null decoder");
    cudaSetDevice(d->device);
    if (d->pending) {
        cudaError_t e = cudaEventSynchronize(d->done);
        if (e != cudaSuccess) return cuda_err(e, "vr_pq_sync");
        d->pending = false;
    }
    const int reason = d->status_host[0];
    if (present) {
        uint64_t n;
        std::memcpy(&n, d->status_host + 2, 8);
        *present = (int64_t)n;
    }
    if (reason)
        return pq_err(VR_ERR_INVALID, "page " + std::to_string(d->status_host[1]) + ": " + reason_text(reason));
    return VR_OK;
}

void vr_pq_destroy(vr_pq_decoder* d) {
    if (!d) return;
    cudaSetDevice(d->device);
    if (d->pending) cudaEventSynchronize(d->done);
    free_all(d);
    delete d;
}

int vr_pq_plain_dictionary(const uint8_t* page, int64_t length, int32_t num_values, int32_t* offsets,
                           uint8_t* data, int64_t* data_bytes) {
    if ((!page && length > 0) || length < 0 || num_values < 0 || !data_bytes)
        return pq_err(VR_ERR_INVALID, "vr_pq_plain_dictionary: bad argument");
    int64_t at = 0, total = 0;
    for (int32_t i = 0; i < num_values; ++i) {
        if (length - at < 4) return pq_err(VR_ERR_INVALID, "dictionary page: entry " + std::to_string(i) +
                                                               "'s length past the end of the page");
        int32_t len;
        std::memcpy(&len, page + at, 4);
        at += 4;
        if (len < 0 || len > length - at)
            return pq_err(VR_ERR_INVALID, "dictionary page: entry " + std::to_string(i) + " past the end of the page");
        if (offsets) offsets[i] = (int32_t)total;
        if (data) std::memcpy(data + total, page + at, (size_t)len);
        at += len;
        total += len;
        if (total >= ((int64_t)1 << 31)) return pq_err(VR_ERR_UNSUPPORTED, "dictionary page: 2 GiB of strings or more");
    }
    if (offsets) offsets[num_values] = (int32_t)total;
    *data_bytes = total;
    return VR_OK;
}

}  // extern "C"
