// Device-side views shared by the join engine's kernels.
//
// A column lives in HBM as its 8 KiB contest pages, copied verbatim and back
// to back (page p at pages + p * 8192). Nothing is decoded ahead of time: the
// kernels read values straight out of the pages, helped by three small index
// arrays built once per column (k_pages.cu):
//   hdr[p]           page p's header (row count, non-null count), so row
//                    lookups never touch the page for it
//   row_start[p]     first row of page p (exclusive prefix of contained rows)
//   page_of_blk[b]   page holding row b * 1024 (shortcut for the page search)
//   dense_base[c]    non-null values before 64-row chunk c of a page, with
//                    chunk_base[p] the first chunk of page p
// This replaces the reference's per-thread readers (TableScan.cpp:82-239:
// exponential page search, popcount to the non-null index, pdep/pext).
#pragma once

#include <cstdint>

#include <vector_types.h>

#if defined(__CUDACC__)
#define BJ_HD __host__ __device__ __forceinline__
#else
#define BJ_HD inline
#endif

namespace bj {

constexpr uint32_t kPageSize = 8192;
constexpr uint32_t kBlkShift = 10;  // rows per page_of_blk entry = 1024
constexpr int kMaxProbes = 16;      // children probed by one pipeline
constexpr int kMaxSlots = 32;       // payload slots carried by one hash table
constexpr uint64_t kNullBits = ~0ull;

enum ColType : int32_t { kInt32 = 0, kInt64 = 1, kFp64 = 2, kVarchar = 3 };

// Device error codes, written (first one wins) to the context's error word.
enum DevError : uint32_t {
    kErrNone = 0,
    kErrPageHeader = 1,   // a page header contradicts the page format
    kErrRowRange = 2,     // a row id beyond the column
    kErrCapacity = 3,     // an output buffer would overflow
    kErrLongString = 4,   // a long-string page run is malformed
    kErrTimeout = 5,      // a bounded wait (mbarrier) ran out
};

struct DevColumn {
    const uint8_t* pages;
    const uint32_t* hdr;          // npages: each page's first 4 bytes (row count | non-null count << 16)
    const uint32_t* row_start;    // npages + 1
    const uint32_t* page_of_blk;  // (nrows >> kBlkShift) + 1
    const uint32_t* dense_base;   // per 64-row chunk
    const uint32_t* chunk_base;   // npages + 1
    uint32_t npages;
    uint32_t nrows;
    int32_t type;
    uint32_t flags;  // kColNulls | kColLongStrings | kColHostPages
    // Rows per page when every page but the last holds exactly rpp rows and
    // the last at most rpp (pages written full, as the contest's writers do):
    // row r is then on page r / rpp. 0 otherwise.
    uint32_t rpp;
    // ceil(2^64 / rpp) for rpp >= 2 (set with set_rpp): r / rpp is the high
    // 64 bits of rpp_m * r for every 32-bit r (Lemire, Kaser and Kurz,
    // "Faster remainder by direct computation", 2019), a few multiplies
    // instead of a division in every lookup of a row.
    uint64_t rpp_m;
};

// Sets a column's rows per page and the multiplier that divides by it.
inline void set_rpp(DevColumn& c, uint32_t rpp) {
    c.rpp = rpp;
    c.rpp_m = rpp >= 2 ? ~uint64_t(0) / rpp + 1 : 0;
}
constexpr uint32_t kColNulls = 1;        // some page has NULLs
constexpr uint32_t kColLongStrings = 2;  // long-string page runs present
constexpr uint32_t kColHostPages = 4;    // pages are read in place from (pinned) host memory
constexpr uint32_t kColRaggedPages = 8;  // page row counts are not uniform (rpp = 0)

// String handle carried in a value slot: page index << 16 | value index in the
// page; a long string (its own page run) uses value index 0xffff.
BJ_HD uint64_t make_str_handle(uint32_t page, uint32_t dense) {
    return (uint64_t(page) << 16) | dense;
}
BJ_HD uint32_t str_handle_page(uint64_t h) { return uint32_t(h >> 16); }
BJ_HD uint32_t str_handle_dense(uint64_t h) { return uint32_t(h & 0xffff); }

#if defined(__CUDACC__)
__device__ __forceinline__ uint16_t ld16(const uint8_t* p) { return *reinterpret_cast<const uint16_t*>(p); }

// Page holding `row` (row < nrows).
__device__ __forceinline__ uint32_t locate_page(const DevColumn& c, uint32_t row) {
    uint32_t lo = c.page_of_blk[row >> kBlkShift];
    uint32_t hi = c.page_of_blk[(row >> kBlkShift) + 1];  // page of the next block start (or npages - 1)
    // Binary search for the last page p in [lo, hi] with row_start[p] <= row.
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (c.row_start[mid] <= row)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Loads the bitmap bits [64k, 64k+64) of a page whose bitmap starts at `bm`
// (bytes may be unaligned; bits beyond the page's rows are garbage).
__device__ __forceinline__ uint64_t load_bits64(const uint8_t* bm, uint32_t k, uint32_t nbytes) {
    uint64_t w = 0;
    uint32_t b0 = k * 8;
#pragma unroll
    for (int i = 0; i < 8; i++)
        if (b0 + i < nbytes) w |= uint64_t(bm[b0 + i]) << (8 * i);
    return w;
}

// Reads the value of `row` as a 64-bit slot. Returns false for NULL.
// INT32 is zero-extended, INT64/FP64 are raw bits, VARCHAR yields a handle.
// row / c.rpp for c.rpp != 0: floor(rpp_m * row / 2^64) from 32-bit halves
// (rpp_m = hi 2^32 + lo: hi row + umulhi(lo, row) carries the same high word).
__device__ __forceinline__ uint32_t page_of_row(const DevColumn& c, uint32_t row) {
    if (c.rpp == 1) return row;
    const uint32_t lo = uint32_t(c.rpp_m), hi = uint32_t(c.rpp_m >> 32);
    return uint32_t((uint64_t(hi) * row + __umulhi(lo, row)) >> 32);
}

__device__ __forceinline__ bool col_get(const DevColumn& c, uint32_t row, uint64_t& v) {
    uint32_t p, i;
    if (c.rpp) {
        p = page_of_row(c, row);
        i = row - p * c.rpp;
    } else {
        p = locate_page(c, row);
        i = row - c.row_start[p];
    }
    const uint8_t* pg = c.pages + size_t(p) * kPageSize;
    if (!(c.flags & (kColNulls | kColLongStrings))) {
        // No NULLs and no long strings anywhere: the value index is the row's
        // index in its page, and the header need not be read.
        switch (c.type) {
        case kInt32: v = *reinterpret_cast<const uint32_t*>(pg + 4 + 4 * i); break;
        case kInt64:
        case kFp64: v = *reinterpret_cast<const uint64_t*>(pg + 8 + 8 * size_t(i)); break;
        default: v = make_str_handle(p, i); break;
        }
        return true;
    }
    const uint32_t h = c.hdr[p];  // header from the device-side cache (pages may be in host memory)
    uint32_t nrows = h & 0xffff;
    if (c.type == kVarchar && nrows >= 0xfffe) {
        v = make_str_handle(p, 0xffff);
        return true;
    }
    uint32_t nn = h >> 16;
    uint32_t dense = i;
    if (nn != nrows) {
        uint32_t nbytes = (nrows + 7) >> 3;
        const uint8_t* bm = pg + kPageSize - nbytes;
        if (!((bm[i >> 3] >> (i & 7)) & 1)) return false;
        uint64_t w = load_bits64(bm, i >> 6, nbytes);
        dense = c.dense_base[c.chunk_base[p] + (i >> 6)] + __popcll(w & ((1ull << (i & 63)) - 1));
    }
    switch (c.type) {
    case kInt32: v = *reinterpret_cast<const uint32_t*>(pg + 4 + 4 * dense); break;
    case kInt64:
    case kFp64: v = *reinterpret_cast<const uint64_t*>(pg + 8 + 8 * size_t(dense)); break;
    default: v = make_str_handle(p, dense); break;
    }
    return true;
}

#endif  // __CUDACC__

// The reference's key hash (engine/op/Hashtable.hpp:35-39): the 32-bit key
// times the 64-bit Fibonacci constant; buckets take the high bits.
BJ_HD uint64_t key_hash(uint32_t key) {
    return uint64_t(key) * 0x9E3779B97F4A7C15ull;
}

// 64-bit mixer for whole-tuple hashing in eager aggregation (the murmur3
// fmix64 finaliser).
BJ_HD uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Hash of a join-key slot of either width. An INT32 key (zero-extended in
// its slot) hashes as the reference's does; an INT64 key, which has no
// reference counterpart (the reference reads every join key as 32 bits,
// engine/op/TableScan.cpp:328), is mixed with the murmur3 finaliser first and
// then multiplied like a 32-bit key, so its high bits reach the bucket bits.
BJ_HD uint64_t key_hash_any(uint64_t key, int32_t type) {
    return type == kInt32 ? key_hash(uint32_t(key)) : mix64(key) * 0x9E3779B97F4A7C15ull;
}

// Blocked bloom filter: one 32-bit word per key with up to four bits set.
// The word is the top log2w bits (at most 15, so a filter is at most 128 KiB
// and fits in shared memory) of the high half hh of the key hash. The bits
// are two rotations of fixed two-bit patterns, P1 rotated by hh mod 32 and
// P2 by (hh >> 5) mod 32: 1024 masks of three or four bits, each made by one
// funnel shift per pattern, with no mask table. (The reference uses a 16-bit
// word per bucket and a 2048-entry mask table, engine/infra/JoinFilter.hpp:
// 9-23; a bloom only removes probes, never results.)
constexpr uint32_t kBloomMaxLog2 = 15;
constexpr uint32_t kBloomP1 = (1u << 0) | (1u << 11);
constexpr uint32_t kBloomP2 = (1u << 0) | (1u << 19);
BJ_HD uint32_t rotl32(uint32_t x, uint32_t s) {
    s &= 31;
    return s ? (x << s) | (x >> (32 - s)) : x;
}
BJ_HD uint32_t bloom_bits_hi(uint32_t hh) { return rotl32(kBloomP1, hh) | rotl32(kBloomP2, hh >> 5); }
BJ_HD uint32_t bloom_word_hi(uint32_t hh, uint32_t log2_words) { return log2_words ? hh >> (32 - log2_words) : 0u; }
// High 32 bits of key_hash(key) (all the bloom filter uses), in two multiplies.
#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t key_hash_hi(uint32_t key) {
    return __umulhi(key, 0x7F4A7C15u) + key * 0x9E3779B9u;
}
// bloom_bits_hi given hh and hh >> 5 (or any value with the same low five
// bits): a funnel shift of a pattern with itself is a rotation by the shift
// amount mod 32.
__device__ __forceinline__ uint32_t bloom_bits_fast(uint32_t hh, uint32_t hh5) {
    return __funnelshift_l(kBloomP1, kBloomP1, hh) | __funnelshift_l(kBloomP2, kBloomP2, hh5);
}
#else
inline uint32_t key_hash_hi(uint32_t key) { return uint32_t(key_hash(key) >> 32); }
#endif

// A built hash table: entries grouped by bucket (CSR), keys 32-bit, a
// multiplicity per entry (eager aggregation folds identical tuples into one
// entry, engine/op/Hashtable.cpp:236-248), `width` 64-bit payload slots per
// entry with a NULL mask.
struct HTView {
    // nbuckets + 1: x = position of the bucket's first entry (the last x is
    // the entry count), y = that entry's key when the bucket is not empty,
    // so one 8-byte load answers a probe of a bucket with a single key.
    const uint2* buckets;
    const uint32_t* keys;        // nentries
    const uint64_t* mult;        // nentries
    const uint64_t* pay;         // nentries * width
    const uint32_t* pnull;       // nentries (bit j: slot j is NULL)
    const uint32_t* bloom;       // 1 << bloom_log2 words, or null (always null for INT64 keys)
    const uint32_t* keys_hi;     // INT64 keys: high halves (keys holds the low ones); null for INT32
    uint32_t shift;              // bucket = key_hash >> shift
    uint32_t bloom_log2;
    uint32_t nentries;
    uint32_t width;
};

// Bucket of key slot k in a table keyed on 64-bit (wide) or 32-bit keys.
BJ_HD uint32_t bucket_of(uint64_t k, bool wide, uint32_t shift) {
    return uint32_t((wide ? key_hash_any(k, kInt64) : key_hash(uint32_t(k))) >> shift);
}

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t ht_bucket(const HTView& ht, uint64_t k) {
    return bucket_of(k, ht.keys_hi != nullptr, ht.shift);
}
// Entry e's key equals key slot k.
__device__ __forceinline__ bool ht_key_eq(const HTView& ht, uint32_t e, uint64_t k) {
    return ht.keys[e] == uint32_t(k) && (!ht.keys_hi || ht.keys_hi[e] == uint32_t(k >> 32));
}
// Entry e's key as a value slot.
__device__ __forceinline__ uint64_t ht_key(const HTView& ht, uint32_t e) {
    return uint64_t(ht.keys[e]) | (ht.keys_hi ? uint64_t(ht.keys_hi[e]) << 32 : 0ull);
}

__device__ __forceinline__ bool bloom_may_contain(const uint32_t* bloom, uint32_t log2w, uint32_t key) {
    const uint32_t hh = key_hash_hi(key);
    const uint32_t bits = bloom_bits_fast(hh, hh >> 5);
    return (bloom[bloom_word_hi(hh, log2w)] & bits) == bits;
}

__device__ __forceinline__ void record_error(uint32_t* err, uint32_t code) {
    if (err) atomicCAS(err, 0u, code);
}

#endif  // __CUDACC__

} // namespace bj
