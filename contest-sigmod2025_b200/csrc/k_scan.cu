// K2 + K3 + K5 fused: the scan-side probe stage of a pipeline.
//
// The reference scans a base table morsel by morsel (TableScan::produceImpl,
// engine/op/TableScan.cpp:616-741): per 64-row step it loads the null bitmap,
// evaluates the restrictions (NOT NULL, bloom join filter, Hashtable.hpp:81-85)
// and hands survivors to the probe (HashtableProbe::operator(), :228-241).
//
// Here warps stream the pages of the probe key column without block-level
// barriers:
//  * a page is read as two work units of 4 KiB, given to warps round-robin:
//    eight 128-bit loads per lane, plus the page header and first row, are
//    issued before any is used (every load stays inside the 8 KiB page;
//    value v sits in 16-byte word (v+1)/4 because values start at byte 4);
//  * a unit without NULLs gives each lane 32 values. The bloom test
//    of a value is four multiplies, one shared-memory load of the filter word,
//    two funnel shifts and a logic op (bloom_bits_fast), spread over the
//    multiply and integer pipes; the lane's survivors form a 32-bit mask, so
//    a unit costs one vote and at most one warp prefix sum;
//  * a page with NULLs is read in blocks of 1024 rows, 32 per lane: the null
//    bitmap word of a lane's rows gives their validity, and the page index's
//    dense base of their 64-row chunk plus a popcount the value index of
//    each (units split a page's rows the same way);
//  * the hash table's bloom filter (up to 128 KiB) is staged once per CTA in
//    shared memory; one CTA of 32 warps runs per SM;
//  * bloom survivors are recorded as (key, row) in a per-warp buffer in
//    shared memory (the key read again from the page just loaded, a cache
//    hit); the buffer is probed 128 entries at a time, four independent
//    bucket lookups per lane, so the latency of the probes is paid once per
//    batch instead of once per hit. Without a bloom filter (a probe that is
//    not selective) every lane probes its own rows directly, four at a time;
//  * matches become items (row, entry, mult). With unique build keys a row
//    has at most one match: items are appended with one atomicAdd per batch
//    and the buffer carries over from unit to unit (mode 2). Otherwise a
//    counting pass writes per-unit counts (mode 0) and an emitting pass
//    writes at the units' offsets (mode 1); the buffer is emptied at the end
//    of every unit.
#include "launch.h"

#include <algorithm>
#include <cstdlib>

namespace bj {
namespace {

constexpr int kWarpsPerCta = 32;
constexpr int kCtaThreads = kWarpsPerCta * 32;
constexpr int kPerLane = 4;                          // buffered candidates per lane
constexpr int kBatch = 32 * kPerLane;                // buffer entries per warp
constexpr int kStepWords = 8;                        // 16-byte words per lane per step
constexpr uint32_t kWordsPerStep = 32 * kStepWords;  // 256 words = 4 KiB: one work unit
constexpr uint32_t kUnitsPerPage = kPageSize / (16 * kWordsPerStep);
constexpr size_t kBloomSmemMax = size_t(4) << kBloomMaxLog2;  // 128 KiB

struct ScanArgs {
    DevColumn key;             // probe key column (pages of the scanned table)
    HTView ht;
    uint32_t mode;             // 0 count per unit, 1 emit at unit offsets, 2 emit with atomics (unique keys)
    uint32_t use_bloom;        // stage ht.bloom in shared memory and test it
    uint32_t prefetch;         // 1-2: a warp prefetches the unit that many units ahead into L2; 3: the next into L1
    // Multipliers for the bloom test, given at run time so that the shifts
    // they stand for (hh >> (32 - log2w), hh >> 5) run on the multiply pipe
    // as __umulhi instead of competing with the shifts on the integer pipe.
    uint32_t word_mul;         // 1 << ht.bloom_log2
    uint32_t field_mul;        // 1 << 27
    uint32_t* page_counts;     // mode 0 output: matches per work unit (scan_probe_units(npages))
    const uint32_t* page_off;  // mode 1 input: exclusive scan of page_counts (units + 1)
    uint32_t* cursor;          // mode 2 global item counter
    uint32_t* out_rows;
    uint32_t* out_ents;
    uint64_t* out_mult;        // may be null when every entry has multiplicity 1
    uint32_t capacity;         // items the outputs can hold
    uint32_t* err;
    uint32_t row_base;         // row of the first page when rows follow from key.rpp (a window of a column)
    // Split form (scan_probe_split): the filter kernel appends every bloom
    // survivor (key, row) here instead of probing it; the probe kernel then
    // probes them all.
    uint32_t* cand_key;
    uint32_t* cand_row;
    uint32_t* cand_count;      // zero before the filter kernel
    uint32_t cand_cap;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// L2 policy for the scanned pages: normal priority, given explicitly (the
// loads with a cache-policy operand came out at 61 registers instead of 64,
// and ran 1-2% faster in same-box A/B runs on the snowflake). Evict-first
// was measured too: slower with a bloom filter (the survivors' keys are read
// again from the pages just loaded) and no better without one (join2).
__device__ __forceinline__ uint64_t stream_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// 16-byte read-only load under an L2 policy.
__device__ __forceinline__ uint4 ld_stream(const uint4* p, uint64_t pol) {
    uint4 v;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(pol));
    return v;
}

// Brings the line holding p into L2; nothing waits for it.
__device__ __forceinline__ void prefetch_line_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
__device__ __forceinline__ void prefetch_line_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Warp-wide exclusive prefix sum; `total` receives the sum.
__device__ __forceinline__ uint32_t warp_excl(uint32_t v, uint32_t& total) {
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane_id() >= uint32_t(o)) inc += u;
    }
    total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}

struct WarpState {
    uint32_t* bkey;     // candidate buffer: key
    uint32_t* brow;     // row of the scanned table
    uint32_t n;         // entries buffered (warp-uniform)
    uint32_t page_cnt;  // matches counted / written for the current unit (modes 0 and 1)
};

// Probes up to kPerLane candidates per lane (candidate i present when bit i
// of `has` is set) and counts (mode 0) or writes their matches. In modes 0
// and 1 every candidate belongs to work unit `unit`.
__device__ __forceinline__ void probe_batch(const ScanArgs& a, WarpState& w, const uint32_t (&key)[kPerLane],
                                            const uint32_t (&row)[kPerLane], uint32_t has, uint32_t unit) {
    const uint32_t lane = lane_id();
    // One load per candidate gives its bucket's range and first key; only
    // buckets with more entries (few: about one key per bucket) loop.
    uint32_t lo[kPerLane], hi[kPerLane], k0[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; i++) {
        lo[i] = hi[i] = 0;
        k0[i] = ~key[i];
        if ((has >> i) & 1) {
            const uint32_t b = uint32_t(key_hash(key[i]) >> a.ht.shift);
            const uint2 b0 = a.ht.buckets[b];
            lo[i] = b0.x;
            hi[i] = a.ht.buckets[b + 1].x;
            k0[i] = b0.y;
        }
    }
#pragma unroll
    for (int i = 0; i < kPerLane; i++)
        if (lo[i] >= hi[i]) k0[i] = ~key[i];
    uint32_t cnt = 0;
    uint32_t cj[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; i++) {
        uint32_t c = k0[i] == key[i] ? 1u : 0u, first = c ? lo[i] : hi[i];
        // Mode 2 (unique build keys): nothing after the first match.
        for (uint32_t e = lo[i] + 1; e < hi[i] && !(a.mode == 2 && c); e++)
            if (a.ht.keys[e] == key[i]) {
                first = c ? first : e;
                c++;
            }
        lo[i] = first;
        cj[i] = c;
        cnt += c;
    }
    uint32_t total;
    const uint32_t off = warp_excl(cnt, total);
    if (a.mode != 0 && total) {
        uint32_t base;
        if (a.mode == 2) {
            uint32_t b = 0;
            if (lane == 31) b = atomicAdd(a.cursor, total);
            base = __shfl_sync(0xffffffffu, b, 31);
        } else {
            base = a.page_off[unit] + w.page_cnt;
        }
        uint32_t o = base + off;
        auto emit = [&](uint32_t r, uint32_t e) {
            if (o < a.capacity) {
                a.out_rows[o] = r;
                a.out_ents[o] = e;
                if (a.out_mult) a.out_mult[o] = a.ht.mult[e];
            } else {
                record_error(a.err, kErrCapacity);
            }
            o++;
        };
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            if (!cj[i]) continue;
            emit(row[i], lo[i]);  // the first match, found above
            uint32_t left = cj[i] - 1;
            for (uint32_t e = lo[i] + 1; left; e++) {
                if (a.ht.keys[e] != key[i]) continue;
                left--;
                emit(row[i], e);
            }
        }
    }
    w.page_cnt += total;
}

// Probes every buffered candidate.
__device__ __forceinline__ void flush(const ScanArgs& a, WarpState& w, uint32_t unit) {
    if (w.n == 0) return;
    __syncwarp();
    const uint32_t lane = lane_id();
    uint32_t key[kPerLane], row[kPerLane], has = 0;
#pragma unroll
    for (int i = 0; i < kPerLane; i++) {
        const uint32_t h = lane + 32 * i;
        key[i] = row[i] = 0;
        if (h < w.n) {
            key[i] = w.bkey[h];
            row[i] = w.brow[h];
            has |= 1u << i;
        }
    }
    probe_batch(a, w, key, row, has, unit);
    w.n = 0;
    __syncwarp();
}

// Probes the candidates flagged in `take` (up to 32 per lane) directly, every
// lane taking kPerLane of its own per round: for dense candidates (no bloom
// filter) this keeps all lanes busy, where buffering would fill the buffer
// from a few lanes at a time. map(c, key, row) gives candidate c.
template <typename Map>
__device__ __forceinline__ void probe_bits(const ScanArgs& a, WarpState& w, uint32_t take, uint32_t unit, Map&& map) {
    uint32_t t = take;
    while (__any_sync(0xffffffffu, t != 0)) {
        uint32_t key[kPerLane], row[kPerLane], has = 0;
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            key[i] = row[i] = 0;
            if (t) {
                const uint32_t c = __ffs(t) - 1;
                t &= t - 1;
                map(c, key[i], row[i]);
                has |= 1u << i;
            }
        }
        probe_batch(a, w, key, row, has, unit);
    }
}

// Buffers the candidates flagged in `take` (up to 32 per lane): map(c, key,
// row) gives candidate c's key and row. Candidates are numbered across the
// warp in lane order; when they do not fit, the buffer is filled, probed and
// refilled until all are in.
template <typename Map>
__device__ __forceinline__ void push_bits(const ScanArgs& a, WarpState& w, uint32_t take, uint32_t p, Map&& map) {
    if (!__any_sync(0xffffffffu, take != 0)) return;
    uint32_t total;
    const uint32_t cnt = __popc(take);
    const uint32_t off = warp_excl(cnt, total);
    for (uint32_t done = 0;;) {
        const uint32_t room = kBatch - w.n;
        // This lane's candidates are numbered [off, off + cnt); only those in
        // the window [done, done + room) go into the buffer this round.
        if (off + cnt > done && off < done + room) {
            uint32_t t = take, j = off;
            for (; j < done; j++) t &= t - 1;  // skip the ones already buffered
            for (; t && j < done + room; j++) {
                const uint32_t c = __ffs(t) - 1;
                t &= t - 1;
                uint32_t key, row;
                map(c, key, row);
                w.bkey[w.n + j - done] = key;
                w.brow[w.n + j - done] = row;
            }
        }
        const uint32_t took = min(room, total - done);
        w.n += took;
        done += took;
        if (done >= total) break;
        flush(a, w, p);
    }
}

// Split form: appends the candidates flagged in `take` to the global
// candidate list, one atomic per warp (candidates numbered in lane order).
template <typename Map>
__device__ __forceinline__ void append_bits(const ScanArgs& a, uint32_t take, Map&& map) {
    if (!__any_sync(0xffffffffu, take != 0)) return;
    uint32_t total;
    const uint32_t off = warp_excl(__popc(take), total);
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(a.cand_count, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    uint32_t o = base + off;
    for (uint32_t t = take; t; t &= t - 1, o++) {
        uint32_t key, row;
        map(__ffs(t) - 1, key, row);
        if (o < a.cand_cap) {
            a.cand_key[o] = key;
            a.cand_row[o] = row;
        } else {
            record_error(a.err, kErrCapacity);
        }
    }
}

// Candidates of one step of a page without NULLs: bit c of `take` is value
// vi0 + 128 (c / 4) + c % 4 of the page of unit p (values at vals, first row
// row0); the key is read again from the page, which this warp has just loaded.
template <bool kFilter>
__device__ __forceinline__ void push_step(const ScanArgs& a, WarpState& w, uint32_t take, int vi0,
                                          const uint32_t* vals, uint32_t row0, uint32_t p, bool dense) {
    auto cand = [&](uint32_t c, uint32_t& key, uint32_t& row) {
        const uint32_t vi = uint32_t(vi0 + 128 * int(c >> 2) + int(c & 3));
        key = __ldg(vals + vi);
        row = row0 + vi;
    };
    if (kFilter)
        append_bits(a, take, cand);
    else if (dense)
        probe_bits(a, w, take, p, cand);
    else
        push_bits(a, w, take, p, cand);
}

__device__ __forceinline__ bool bloom_pass(const ScanArgs& a, const uint32_t* bloom, uint32_t key) {
    const uint32_t hh = key_hash_hi(key);
    const uint32_t m = bloom_bits_fast(hh, __umulhi(hh, a.field_mul));
    return (~bloom[__umulhi(hh, a.word_mul)] & m) == 0;
}

// Values of one step of a page without NULLs that pass the bloom (or all of
// them without one), as bit 4u + k for value k of word u.
__device__ __forceinline__ uint32_t step_take(const ScanArgs& a, const uint4 (&q)[kStepWords], const uint32_t* bloom,
                                              bool use_bloom) {
    if (!use_bloom) return 0xffffffffu;
    uint32_t take = 0;
#pragma unroll
    for (int u = 0; u < kStepWords; u++) {
        const uint32_t v[4] = {q[u].x, q[u].y, q[u].z, q[u].w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (bloom_pass(a, bloom, v[k])) take |= 1u << (4 * u + k);
    }
    return take;
}

// Valid-value mask of a step for a lane whose first value is vi0 (bit 4u + k
// is value vi0 + 128u + k, valid when 0 <= value < n).
__device__ __forceinline__ uint32_t step_valid(int vi0, uint32_t n) {
    const int avail = int(n) - vi0;  // values from vi0 to n - 1
    if (avail <= 0) return 0;
    const uint32_t t = min(uint32_t(avail), 32u * 32u);
    const uint32_t full = t >> 7;             // words with all four values valid
    const uint32_t part = min(t & 127u, 4u);  // valid values of word `full`
    const uint32_t lowfull = full >= 8 ? 0xffffffffu : (1u << (4 * full)) - 1;
    const uint32_t partial = full >= 8 ? 0u : ((1u << part) - 1) << (4 * full);
    uint32_t valid = lowfull | partial;
    if (vi0 < 0) valid &= ~1u;  // the page header
    return valid;
}

// Rows [r_begin, r_end) of page p, which has NULLs, in blocks of 1024 rows:
// lane l takes 32 rows (one 32-bit bitmap word); the page index's dense base
// of their 64-row chunk, plus the popcount of the chunk's lower word for an
// upper half, gives the value index of the first valid row. Without a bloom
// every valid row is a candidate and no value is read before the probe.
template <bool kFilter>
__device__ __forceinline__ void scan_rows_nulls(const ScanArgs& a, WarpState& w, const uint32_t* bloom,
                                                bool use_bloom, uint32_t unit, uint32_t p, uint32_t n,
                                                uint32_t row0, uint32_t r_begin, uint32_t r_end) {
    const uint32_t lane = lane_id();
    if (!a.key.chunk_base || !a.key.dense_base) {
        // A column run without a page index (its layout speculated to have
        // no NULLs): the speculation was wrong and the call runs again.
        if (lane == 0) record_error(a.err, kErrPageHeader);
        return;
    }
    const uint8_t* pg = a.key.pages + size_t(p) * kPageSize;
    const uint32_t* vals = reinterpret_cast<const uint32_t*>(pg + 4);
    const uint32_t nbytes = (n + 7) >> 3;
    const uint8_t* bm = pg + kPageSize - nbytes;
    const uint32_t cb = __ldg(a.key.chunk_base + p);
    for (uint32_t blk = r_begin; blk < r_end; blk += 1024) {
        const uint32_t r = blk + 32 * lane;  // this lane's first row
        uint32_t wb = 0;
        if (r < r_end) {
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const uint32_t byte = (r >> 3) + b;
                if (byte < nbytes) wb |= uint32_t(bm[byte]) << (8 * b);
            }
            if (r_end - r < 32) wb &= (1u << (r_end - r)) - 1;
        }
        // Lanes pair up into 64-row chunks (blocks start at a multiple of 64).
        const uint32_t lower = __shfl_up_sync(0xffffffffu, wb, 1);
        uint32_t d0 = 0;
        if (r < r_end) d0 = __ldg(a.key.dense_base + cb + (r >> 6)) + ((lane & 1) ? __popc(lower) : 0u);
        // An INT32 page holds at most 2047 values; a larger dense index only
        // comes from a malformed page (reported by the page index) and is not read.
        if (d0 + __popc(wb) > 2047) wb = 0;
        uint32_t take = wb;
        if (use_bloom && wb) {
            take = 0;
            uint32_t t = wb, d = d0;
            while (t) {
                const uint32_t j = __ffs(t) - 1;
                t &= t - 1;
                if (bloom_pass(a, bloom, __ldg(vals + d))) take |= 1u << j;
                d++;
            }
        }
        auto cand = [&](uint32_t c, uint32_t& key, uint32_t& row) {
            key = __ldg(vals + d0 + __popc(wb & ((1u << c) - 1)));
            row = row0 + r + c;
        };
        if (kFilter)
            append_bits(a, take, cand);
        else if (use_bloom)
            push_bits(a, w, take, unit, cand);
        else
            probe_bits(a, w, take, unit, cand);
    }
}

// kFilter: the filter kernel of the split form (no probes; survivors go to
// the candidate list). Otherwise the fused scan-side probe.
template <bool kFilter>
__global__ void __launch_bounds__(kCtaThreads, 1) k_scan_probe(ScanArgs a) {
    extern __shared__ uint4 bloom4[];
    __shared__ uint32_t bkey[kFilter ? 1 : kWarpsPerCta][kFilter ? 1 : kBatch];
    __shared__ uint32_t brow[kFilter ? 1 : kWarpsPerCta][kFilter ? 1 : kBatch];
    const uint32_t* bloom = reinterpret_cast<const uint32_t*>(bloom4);
    const bool use_bloom = a.use_bloom != 0;
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint32_t total_warps = gridDim.x * kWarpsPerCta;
    const uint32_t nunits = kUnitsPerPage * a.key.npages;
    const uint32_t first = blockIdx.x * kWarpsPerCta + warp;

    // Work unit u is part u % kUnitsPerPage (4 KiB, 256 words) of page
    // u / kUnitsPerPage; the warp's
    // units are first, first + total_warps, ... (half pages balance the
    // warps better than whole pages: 10.6 units per warp against 5.3 pages
    // on the 50M-row fact). A unit's loads are all issued before any is
    // used, and every load stays inside its 8 KiB page.
    const uint64_t pol = stream_policy();
    auto load_unit = [&](uint32_t u, uint4 (&q)[kStepWords], uint32_t& hdr, uint32_t& row0) {
        const uint4* pw = reinterpret_cast<const uint4*>(a.key.pages + size_t(u / kUnitsPerPage) * kPageSize);
#pragma unroll
        for (int i = 0; i < kStepWords; i++) q[i] = ld_stream(pw + (u % kUnitsPerPage) * kWordsPerStep + lane + 32 * i, pol);
        hdr = lane == 0 ? __ldg(reinterpret_cast<const uint32_t*>(pw)) : 0;
        row0 = lane == 0 ? (a.key.rpp ? a.row_base + (u / kUnitsPerPage) * a.key.rpp
                                      : __ldg(a.key.row_start + u / kUnitsPerPage))
                         : 0;
    };
    uint4 q[kStepWords];
    uint32_t hdr_l = 0, row0_l = 0;

    if (use_bloom) {
        // Asynchronous 16-byte copies (no registers, all in flight at once):
        // a load-then-store loop pays an L2 round trip per iteration, about
        // a fifth of the kernel's time for a 128 KiB filter.
        const uint4* src = reinterpret_cast<const uint4*>(a.ht.bloom);
        const uint32_t n4 = (1u << a.ht.bloom_log2) / 4;
        for (uint32_t i = threadIdx.x; i < n4; i += kCtaThreads) {
            const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(bloom4 + i));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src + i) : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();

    WarpState w{bkey[kFilter ? 0 : warp], brow[kFilter ? 0 : warp], 0, 0};
    for (uint32_t u = first; u < nunits; u += total_warps) {
        const uint32_t p = u / kUnitsPerPage, part = u % kUnitsPerPage;
        load_unit(u, q, hdr_l, row0_l);
        if (a.prefetch) {
            // One 128-byte line per lane of the unit a.prefetch units ahead
            // (mode 3: the next unit, into L1).
            const uint32_t ahead = a.prefetch == 3 ? 1u : a.prefetch;
            const uint64_t un = uint64_t(u) + uint64_t(ahead) * total_warps;
            if (un < nunits) {
                const uint8_t* line = a.key.pages + size_t(un / kUnitsPerPage) * kPageSize +
                                      (un % kUnitsPerPage) * (16 * kWordsPerStep) + (lane * 128) % (16 * kWordsPerStep);
                if (a.prefetch == 3)
                    prefetch_line_l1(line);
                else
                    prefetch_line_l2(line);
            }
        }
        const uint32_t hdr = __shfl_sync(0xffffffffu, hdr_l, 0);
        const uint32_t row0 = __shfl_sync(0xffffffffu, row0_l, 0);
        const uint32_t n = hdr & 0xffff, nn = hdr >> 16;
        const uint32_t* vals = reinterpret_cast<const uint32_t*>(a.key.pages + size_t(p) * kPageSize) + 1;
        w.page_cnt = 0;
        if (nn == n) {
            const int vi0 = 4 * int(lane) - 1 + int(part * 4 * kWordsPerStep);
            if (vi0 - int(lane) * 4 < int(n))  // some value of the unit is below n
                push_step<kFilter>(a, w, step_take(a, q, bloom, use_bloom) & step_valid(vi0, n), vi0, vals, row0,
                                   u, !use_bloom);
        } else {
            // A page with NULLs: unit k takes rows [1024 k, 1024 (k + 1)), the
            // last unit every row from there on.
            const uint32_t r_begin = part * 1024;
            const uint32_t r_end = part + 1 == kUnitsPerPage ? n : min(n, r_begin + 1024);
            if (r_begin < r_end) scan_rows_nulls<kFilter>(a, w, bloom, use_bloom, u, p, n, row0, r_begin, r_end);
        }
        if (!kFilter && a.mode != 2) {
            flush(a, w, u);
            if (a.mode == 0 && lane == 0) a.page_counts[u] = w.page_cnt;
        }
    }
    if (!kFilter && a.mode == 2) flush(a, w, 0);
}

// The probe kernel of the split form: every candidate of the list, 128 per
// warp (four per lane), probed against the table and appended as items
// (mode 2: unique build keys).
__global__ void __launch_bounds__(256) k_probe_candidates(ScanArgs a) {
    const uint32_t n = min(*a.cand_count, a.cand_cap);
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    WarpState w{nullptr, nullptr, 0, 0};
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kBatch; base < n;
         base += warps * kBatch) {
        uint32_t key[kPerLane], row[kPerLane], has = 0;
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            const uint32_t h = base + lane + 32 * i;
            key[i] = row[i] = 0;
            if (h < n) {
                key[i] = a.cand_key[h];
                row[i] = a.cand_row[h];
                has |= 1u << i;
            }
        }
        probe_batch(a, w, key, row, has, 0);
    }
}

template <bool kFilter>
void launch_scan(const ScanArgs& a, size_t bloom_bytes, int num_sms, cudaStream_t st) {
    // Once per process and form (thread-safe static initialisation; server
    // workers launch from several threads).
    static const bool configured = [] {
        cudaFuncSetAttribute(k_scan_probe<kFilter>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBloomSmemMax));
        return true;
    }();
    (void)configured;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan_probe<kFilter>, kCtaThreads, bloom_bytes);
    per_sm = std::max(1, per_sm);
    const uint64_t ctas =
        std::min<uint64_t>((uint64_t(kUnitsPerPage) * a.key.npages + kWarpsPerCta - 1) / kWarpsPerCta,
                           uint64_t(num_sms) * per_sm);
    k_scan_probe<kFilter><<<unsigned(ctas), kCtaThreads, bloom_bytes, st>>>(a);
}

} // namespace

size_t scan_probe_bloom_limit() { return kBloomSmemMax; }
uint32_t scan_probe_units(uint32_t npages) { return kUnitsPerPage * npages; }

int scan_probe(const DevColumn& key, const HTView& ht, int mode, bool bloom_smem, uint32_t* page_counts,
               const uint32_t* page_off, uint32_t* cursor, uint32_t* out_rows, uint32_t* out_ents, uint64_t* out_mult,
               uint32_t capacity, uint32_t* err, int num_sms, cudaStream_t st, uint32_t row_base) {
    if (!key.npages) return 0;
    size_t bloom_bytes = bloom_smem && ht.bloom ? (sizeof(uint32_t) << ht.bloom_log2) : 0;
    if (bloom_bytes > kBloomSmemMax) bloom_bytes = 0;
    // Prefetch of the work unit this many units ahead of each warp's current
    // one into L2, or (3) of the next one into L1 (tuning knob
    // B200JOIN_SCAN_PREFETCH = 0-3; device-memory pages only).
    static const uint32_t ahead = [] {
        const char* e = std::getenv("B200JOIN_SCAN_PREFETCH");
        return e ? uint32_t(std::min(3, std::max(0, std::atoi(e)))) : 0u;
    }();
    const uint32_t prefetch = (key.flags & kColHostPages) ? 0u : ahead;
    ScanArgs a{key,      ht,       uint32_t(mode), bloom_bytes ? 1u : 0u, prefetch,
               ht.bloom_log2 ? (1u << ht.bloom_log2) : 0u, 1u << 27,
               page_counts, page_off, cursor, out_rows, out_ents, out_mult, capacity, err, row_base,
               nullptr, nullptr, nullptr, 0};
    launch_scan<false>(a, bloom_bytes, num_sms, st);
    return 1;
}

int scan_probe_split(const DevColumn& key, const HTView& ht, uint32_t* cursor, uint32_t* out_rows, uint32_t* out_ents,
                     uint64_t* out_mult, uint32_t capacity, uint32_t* cand_key, uint32_t* cand_row,
                     uint32_t* cand_count, uint32_t cand_cap, uint32_t* err, int num_sms, cudaStream_t st,
                     uint32_t row_base) {
    if (!key.npages) return 0;
    size_t bloom_bytes = ht.bloom ? (sizeof(uint32_t) << ht.bloom_log2) : 0;
    if (bloom_bytes > kBloomSmemMax) bloom_bytes = 0;
    ScanArgs a{key,      ht,       2u, bloom_bytes ? 1u : 0u, 0u,
               ht.bloom_log2 ? (1u << ht.bloom_log2) : 0u, 1u << 27,
               nullptr, nullptr, cursor, out_rows, out_ents, out_mult, capacity, err, row_base,
               cand_key, cand_row, cand_count, cand_cap};
    launch_scan<true>(a, bloom_bytes, num_sms, st);
    k_probe_candidates<<<unsigned(num_sms) * 8, 256, 0, st>>>(a);  // 64 warps per SM (32 registers)
    return 2;
}

} // namespace bj
