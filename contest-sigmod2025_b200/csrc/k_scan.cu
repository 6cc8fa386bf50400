// K2 + K3 + K5 fused: the scan-side probe stage of a pipeline.
//
// The reference scans a base table morsel by morsel (TableScan::produceImpl,
// engine/op/TableScan.cpp:616-741): per 64-row step it loads the null bitmap,
// evaluates the restrictions (NOT NULL, bloom join filter, Hashtable.hpp:81-85)
// and hands survivors to the probe (HashtableProbe::operator(), :228-241).
//
// Here every warp owns whole pages of the probe key column and works on them
// without block-level barriers:
//  * a page without NULLs is read with 128-bit coalesced loads, four per lane
//    in flight (value v sits in 16-byte word (v+1)/4 because values start at
//    byte 4); a page with NULLs is read row by row, 32 rows per step, the null
//    bitmap word of those rows giving validity and (by popcount) the dense
//    index of each value;
//  * the hash table's bloom filter and the 2048-entry bloom mask table are
//    staged once per CTA in shared memory, so a miss costs two shared-memory
//    loads;
//  * survivors (bloom hits, or every non-null row when the probe is not
//    selective) are pushed into a per-warp buffer in shared memory with
//    ballots; the buffer is probed 128 entries at a time, four independent
//    bucket lookups per lane, so the L2 latency of the probes is paid once
//    per batch instead of once per hit;
//  * matches become items (row, entry, mult). With unique build keys a row
//    has at most one match: items are appended with one atomicAdd per batch
//    (mode 2). Otherwise a counting pass writes per-page counts (mode 0) and
//    an emitting pass writes at the scanned page offsets (mode 1).
#include "launch.h"

#include <algorithm>
#include <cstdlib>

namespace bj {
namespace {

constexpr int kWarpsPerCta = 16;
constexpr int kCtaThreads = kWarpsPerCta * 32;
constexpr int kPerLane = 4;                      // buffered candidates per lane
constexpr int kBatch = 32 * kPerLane;            // buffer entries per warp
constexpr size_t kBloomSmemMax = size_t(4) << kBloomMaxLog2;  // 64 KiB

struct ScanArgs {
    DevColumn key;             // probe key column (pages of the scanned table)
    HTView ht;
    uint32_t mode;             // 0 count per page, 1 emit at page offsets, 2 emit with atomics (unique keys)
    uint32_t use_bloom;        // stage ht.bloom in shared memory and test it
    uint32_t* page_counts;     // mode 0 output (npages)
    const uint32_t* page_off;  // mode 1 input (npages + 1)
    uint32_t* cursor;          // mode 2 global item counter
    uint32_t* out_rows;
    uint32_t* out_ents;
    uint64_t* out_mult;        // may be null when every entry has multiplicity 1
    uint32_t capacity;         // items the outputs can hold
    uint32_t* err;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// ---- TMA bulk copies into shared memory, completed on an mbarrier ----
constexpr uint32_t kWaitLimit = 1u << 24;  // mbarrier polls before a warp gives up (about a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait on one phase; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Orders this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One page (8 KiB, 16-byte aligned source) into shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load_page(void* dst, const void* src, uint64_t* bar) {
    mbar_expect_tx(bar, kPageSize);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(kPageSize), "r"(smem_u32(bar))
                 : "memory");
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
    uint2* buf;         // this warp's candidate buffer: (row within page, key)
    uint32_t n;         // entries buffered (warp-uniform)
    uint32_t page_cnt;  // matches counted / written for the current page
};

// Probes every buffered candidate; counts (mode 0) or writes items.
__device__ __forceinline__ void flush(const ScanArgs& a, WarpState& w, uint32_t page, uint32_t row0) {
    if (w.n == 0) return;
    __syncwarp();
    const uint32_t lane = lane_id();
    uint32_t key[kPerLane], rowi[kPerLane], lo[kPerLane], hi[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; i++) {
        uint32_t h = lane + 32 * i;
        lo[i] = hi[i] = 0;
        key[i] = rowi[i] = 0;
        if (h < w.n) {
            uint2 c = w.buf[h];
            rowi[i] = c.x;
            key[i] = c.y;
            uint32_t b = uint32_t(key_hash(c.y) >> a.ht.shift);
            lo[i] = a.ht.bucket_off[b];
            hi[i] = a.ht.bucket_off[b + 1];
        }
    }
    uint32_t cnt = 0;
    uint32_t cj[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; i++) {
        uint32_t c = 0, first = hi[i];
        for (uint32_t e = lo[i]; e < hi[i]; e++)
            if (a.ht.keys[e] == key[i]) {
                first = c ? first : e;
                c++;
            }
        lo[i] = first;
        cj[i] = c;
        cnt += c;
    }
    uint32_t total;
    uint32_t off = warp_excl(cnt, total);
    if (a.mode != 0 && total) {
        uint32_t base;
        if (a.mode == 2) {
            uint32_t b = 0;
            if (lane == 31) b = atomicAdd(a.cursor, total);
            base = __shfl_sync(0xffffffffu, b, 31);
        } else {
            base = a.page_off[page] + w.page_cnt;
        }
        uint32_t o = base + off;
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            uint32_t left = cj[i];
            for (uint32_t e = lo[i]; left; e++) {
                if (a.ht.keys[e] != key[i]) continue;
                left--;
                if (o < a.capacity) {
                    a.out_rows[o] = row0 + rowi[i];
                    a.out_ents[o] = e;
                    if (a.out_mult) a.out_mult[o] = a.ht.mult[e];
                } else {
                    record_error(a.err, kErrCapacity);
                }
                o++;
            }
        }
    }
    w.page_cnt += total;
    w.n = 0;
    __syncwarp();
}

// Pushes the candidates (row i, key) of this ballot round into the buffer.
__device__ __forceinline__ void push(const ScanArgs& a, WarpState& w, bool take, uint32_t i, uint32_t key,
                                     uint32_t page, uint32_t row0) {
    uint32_t mask = __ballot_sync(0xffffffffu, take);
    if (!mask) return;
    if (w.n + 32 > kBatch) flush(a, w, page, row0);
    if (take) w.buf[w.n + __popc(mask & ((1u << lane_id()) - 1))] = make_uint2(i, key);
    w.n += __popc(mask);
}

// Pushes up to four candidates per lane (bits of `take4`; value c has row
// index vi0 + c and key vals[c]).
__device__ __forceinline__ void push4(const ScanArgs& a, WarpState& w, uint32_t take4, int vi0, const uint32_t* vals,
                                      uint32_t page, uint32_t row0) {
    if (!__any_sync(0xffffffffu, take4 != 0)) return;
    uint32_t total;
    uint32_t off = warp_excl(__popc(take4), total);
    if (w.n + total > kBatch) flush(a, w, page, row0);
    uint32_t o = w.n + off;
#pragma unroll
    for (int c = 0; c < 4; c++)
        if ((take4 >> c) & 1) w.buf[o++] = make_uint2(uint32_t(vi0 + c), vals[c]);
    w.n += total;
}

// Bloom test with the high half of the key hash: the mask index is its low
// 11 bits (bits 32-42 of the hash), the word its top log2w bits.
__device__ __forceinline__ bool bloom_pass(const uint32_t* bloom, const uint32_t* masks, uint32_t wshift,
                                           uint32_t key) {
    uint32_t hh = key_hash_hi(key);
    uint32_t m = masks[hh & (kBloomMasks - 1)];
    return (bloom[hh >> wshift] & m) == m;
}

// Scans one page of the key column (pg: its bytes, in global or shared
// memory; p: its index) for one warp: validity, bloom test, candidates,
// batched probes, items.
__device__ __forceinline__ void scan_page(const ScanArgs& a, WarpState& w, const uint32_t* bloom,
                                          const uint32_t* masks, bool use_bloom, uint32_t wshift,
                                          const uint8_t* pg, uint32_t p) {
    const uint32_t lane = lane_id();
    uint32_t hdr = lane == 0 ? *reinterpret_cast<const uint32_t*>(pg) : 0;
    uint32_t row0 = lane == 0 ? a.key.row_start[p] : 0;
    hdr = __shfl_sync(0xffffffffu, hdr, 0);
    row0 = __shfl_sync(0xffffffffu, row0, 0);
    const uint32_t n = hdr & 0xffff, nn = hdr >> 16;
    w.page_cnt = 0;
    if (nn == n) {
        // 16-byte word m holds values 4m-1 .. 4m+2 (word 0 starts with the header).
        const uint4* v4 = reinterpret_cast<const uint4*>(pg);
        const uint32_t M = (4 + 4 * n + 15) / 16;
        for (uint32_t m0 = 0; m0 < M; m0 += 128) {
            uint4 q[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                uint32_t m = m0 + lane + 32 * u;
                q[u] = m < M ? v4[m] : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                uint32_t m = m0 + lane + 32 * u;
                uint32_t vals[4] = {q[u].x, q[u].y, q[u].z, q[u].w};
                int vi0 = int(4 * m) - 1;
                // Words strictly inside the value range need no bounds test.
                uint32_t valid4 = (m >= 1 && 4 * m + 3 <= n) ? 0xfu : 0u;
                if (!valid4) {
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        int vi = vi0 + c;
                        valid4 |= uint32_t(vi >= 0 && uint32_t(vi) < n) << c;
                    }
                }
                uint32_t take4 = valid4;
                if (use_bloom) {
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (!bloom_pass(bloom, masks, wshift, vals[c])) take4 &= ~(1u << c);
                }
                push4(a, w, take4, vi0, vals, p, row0);
            }
        }
    } else {
        // Rows r0 .. r0+31: bitmap word, validity, dense index, value.
        const uint32_t nbytes = (n + 7) >> 3;
        const uint8_t* bm = pg + kPageSize - nbytes;
        uint32_t running = 0;
        for (uint32_t r0 = 0; r0 < n; r0 += 32) {
            uint32_t wbits = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                uint32_t byte = (r0 >> 3) + b;
                if (byte < nbytes) wbits |= uint32_t(bm[byte]) << (8 * b);
            }
            uint32_t lim = n - r0 >= 32 ? 0xffffffffu : ((1u << (n - r0)) - 1);
            wbits &= lim;
            bool valid = (wbits >> lane) & 1;
            uint32_t d = running + __popc(wbits & ((1u << lane) - 1));
            uint32_t key = valid ? *reinterpret_cast<const uint32_t*>(pg + 4 + 4 * d) : 0;
            running += __popc(wbits);
            bool take = valid && (!use_bloom || bloom_pass(bloom, masks, wshift, key));
            push(a, w, take, r0 + lane, key, p, row0);
        }
    }
    flush(a, w, p, row0);
    if (a.mode == 0 && lane == 0) a.page_counts[p] = w.page_cnt;
}

__global__ void __launch_bounds__(kCtaThreads, 2) k_scan_probe(ScanArgs a) {
    extern __shared__ uint4 bloom4[];
    __shared__ uint2 bufs[kWarpsPerCta][kBatch];
    __shared__ uint32_t masks[kBloomMasks];
    const uint32_t* bloom = reinterpret_cast<const uint32_t*>(bloom4);
    const bool use_bloom = a.use_bloom != 0;
    if (use_bloom) {
        const uint4* src = reinterpret_cast<const uint4*>(a.ht.bloom);
        uint32_t n4 = (1u << a.ht.bloom_log2) / 4;
        for (uint32_t i = threadIdx.x; i < n4; i += kCtaThreads) bloom4[i] = src[i];
        for (uint32_t i = threadIdx.x; i < kBloomMasks; i += kCtaThreads) masks[i] = bloom_mask(i);
    }
    __syncthreads();

    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint32_t total_warps = gridDim.x * kWarpsPerCta;
    WarpState w{bufs[warp], 0, 0};
    const uint32_t wshift = 32 - a.ht.bloom_log2;  // bloom_log2 >= 5 whenever the bloom is used

    for (uint32_t p = blockIdx.x * kWarpsPerCta + warp; p < a.key.npages; p += total_warps)
        scan_page(a, w, bloom, masks, use_bloom, wshift, a.key.pages + size_t(p) * kPageSize, p);
}

// Same work, pages staged by TMA: each warp owns one 8 KiB slot of shared
// memory and a private mbarrier; lane 0 issues the bulk copy of the warp's
// next page as soon as the warp has finished reading the slot, so sixteen
// pages per SM are in flight without holding registers. No block-level
// barrier follows the prologue. Opt-in (see scan_probe below), for pages in
// device memory only.
__global__ void __launch_bounds__(kCtaThreads, 1) k_scan_probe_tma(ScanArgs a) {
    extern __shared__ __align__(128) uint8_t dyn[];
    uint8_t* slots = dyn;                                               // kWarpsPerCta * 8 KiB
    uint4* bloom4 = reinterpret_cast<uint4*>(dyn + kWarpsPerCta * kPageSize);
    __shared__ uint2 bufs[kWarpsPerCta][kBatch];
    __shared__ uint32_t masks[kBloomMasks];
    __shared__ __align__(8) uint64_t bars[kWarpsPerCta];
    const uint32_t* bloom = reinterpret_cast<const uint32_t*>(bloom4);
    const bool use_bloom = a.use_bloom != 0;
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint32_t total_warps = gridDim.x * kWarpsPerCta;
    const uint32_t first = blockIdx.x * kWarpsPerCta + warp;
    uint8_t* slot = slots + warp * kPageSize;
    if (lane == 0) {
        mbar_init(&bars[warp], 1);
        mbar_fence_init();
        if (first < a.key.npages) bulk_load_page(slot, a.key.pages + size_t(first) * kPageSize, &bars[warp]);
    }
    if (use_bloom) {
        const uint4* src = reinterpret_cast<const uint4*>(a.ht.bloom);
        uint32_t n4 = (1u << a.ht.bloom_log2) / 4;
        for (uint32_t i = threadIdx.x; i < n4; i += kCtaThreads) bloom4[i] = src[i];
        for (uint32_t i = threadIdx.x; i < kBloomMasks; i += kCtaThreads) masks[i] = bloom_mask(i);
    }
    __syncthreads();
    WarpState w{bufs[warp], 0, 0};
    const uint32_t wshift = 32 - a.ht.bloom_log2;
    uint32_t k = 0;
    for (uint32_t p = first; p < a.key.npages; p += total_warps, k++) {
        bool ok = mbar_wait(&bars[warp], k & 1);
        if (!__all_sync(0xffffffffu, ok)) {
            // Give up on this warp's pages: record it; the copy in flight (if
            // any) is waited for below, with a limit, before the warp exits.
            if (lane == 0) record_error(a.err, kErrTimeout);
            if (lane == 0) mbar_wait(&bars[warp], k & 1);
            __syncwarp();
            return;
        }
        scan_page(a, w, bloom, masks, use_bloom, wshift, slot, p);
        __syncwarp();
        const uint32_t pn = p + total_warps;
        if (lane == 0 && pn < a.key.npages) {
            fence_proxy_async();
            bulk_load_page(slot, a.key.pages + size_t(pn) * kPageSize, &bars[warp]);
        }
    }
}

} // namespace

size_t scan_probe_bloom_limit() { return kBloomSmemMax; }

int scan_probe(const DevColumn& key, const HTView& ht, int mode, bool bloom_smem, uint32_t* page_counts,
               const uint32_t* page_off, uint32_t* cursor, uint32_t* out_rows, uint32_t* out_ents, uint64_t* out_mult,
               uint32_t capacity, uint32_t* err, int num_sms, cudaStream_t st) {
    if (!key.npages) return 0;
    size_t bloom_bytes = bloom_smem && ht.bloom ? (sizeof(uint32_t) << ht.bloom_log2) : 0;
    if (bloom_bytes > kBloomSmemMax) bloom_bytes = 0;
    ScanArgs a{key, ht, uint32_t(mode), bloom_bytes ? 1u : 0u, page_counts, page_off, cursor,
               out_rows, out_ents, out_mult, capacity, err};
    // TMA staging (opt-in: B200JOIN_SCAN_TMA=1) needs device-memory pages
    // (not pages read in place from the host) with a 16-byte aligned base.
    // Measured on snowflake x0.7 it ran at 92 us against 68 us for the
    // load-based kernel: one 8 KiB slot per warp leaves room for only 16
    // warps per SM next to the bloom filter, too few to hide page latency.
    static const bool tma_opt_in = [] {
        const char* e = std::getenv("B200JOIN_SCAN_TMA");
        return e && std::atoi(e) != 0;
    }();
    const bool tma = tma_opt_in && !(key.flags & kColHostPages) && (reinterpret_cast<uintptr_t>(key.pages) % 16) == 0;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_scan_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBloomSmemMax));
        cudaFuncSetAttribute(k_scan_probe_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kWarpsPerCta * kPageSize + kBloomSmemMax));
        configured = true;
    }
    if (tma) {
        size_t smem = kWarpsPerCta * kPageSize + bloom_bytes;
        uint64_t ctas = std::min<uint64_t>((uint64_t(key.npages) + kWarpsPerCta - 1) / kWarpsPerCta, uint64_t(num_sms));
        k_scan_probe_tma<<<unsigned(ctas), kCtaThreads, smem, st>>>(a);
        return 1;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan_probe, kCtaThreads, bloom_bytes);
    per_sm = std::max(1, per_sm);
    uint64_t ctas = std::min<uint64_t>((uint64_t(key.npages) + kWarpsPerCta - 1) / kWarpsPerCta,
                                       uint64_t(num_sms) * per_sm);
    k_scan_probe<<<unsigned(ctas), kCtaThreads, bloom_bytes, st>>>(a);
    return 1;
}

} // namespace bj
