// K3/K4/K6: hash-table build.
//
// The reference builds a chaining table per partition: tuples are appended to
// per-thread chunks (HashtableBuild::operator(), engine/op/Hashtable.hpp:
// 176-203), then every partition is inserted bucket-head first, setting a
// 16-bit bloom word per bucket and folding a tuple into the bucket head when
// key and payload are equal (eager aggregation, engine/op/Hashtable.cpp:
// 208-263). Sizing: 2^max(bit_width(n), 4) buckets (Hashtable.cpp:94-104).
//
// On the GPU the build is three passes:
//  1. emit, eager aggregation and bucket counts (K6) in one kernel: each
//     thread writes its tuple (key, NULL mask, payload, multiplicity), makes
//     it visible device-wide, and inserts its index into an open-addressing
//     table keyed by the whole tuple. The first copy of each distinct tuple
//     claims a slot with atomicCAS and becomes its representative (and counts
//     itself into its bucket); every other copy adds its multiplicity to the
//     representative with atomicAdd. Unlike the reference, which only merges
//     with the current bucket head, this folds every duplicate.
//  2. an exclusive scan of the bucket counts (CSR offsets), then a scatter of
//     the representatives into their bucket's contiguous range that also sets
//     their bits in a blocked bloom filter (K3/K4). The same bucket index as
//     the reference: key_hash(key) >> shift. The filter is at most 128 KiB so
//     scans can stage it in shared memory; probes consult it before touching
//     the buckets.
//  3. flags of the finished table (repeated keys, multiplicities above 1).
// Every buffer that must start at zero is cleared by one memset per build.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {

__device__ __forceinline__ uint64_t tuple_hash(const TupleBuf& t, uint32_t i) {
    uint64_t h = mix64(uint64_t(t.keys[i]) ^ (uint64_t(t.pnull[i]) << 32));
    const uint64_t* p = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) h = mix64(h ^ (p[j] + 0x9E3779B97F4A7C15ull * (j + 1)));
    return h;
}

// Tuple a (written by another thread, read through L2) equals tuple b.
__device__ __forceinline__ bool tuple_equal_cg(const TupleBuf& t, uint32_t a, uint32_t b) {
    if (__ldcg(t.keys + a) != t.keys[b] || __ldcg(t.pnull + a) != t.pnull[b]) return false;
    const uint64_t* pa = t.pay + size_t(a) * t.width;
    const uint64_t* pb = t.pay + size_t(b) * t.width;
    for (uint32_t j = 0; j < t.width; j++)
        if (__ldcg(pa + j) != pb[j]) return false;
    return true;
}

__global__ void __launch_bounds__(256) k_emit_aggregate(BuildArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const TupleBuf& t = a.tb;
    if (i >= t.count) return;
    // Emit.
    const uint32_t row = item_row(a.in, i);
    uint64_t kv = 0;
    const bool key_ok = row < a.key.nrows && col_get(a.key, row, kv);
    if (row >= a.key.nrows) record_error(a.err, kErrRowRange);
    const uint64_t m = key_ok ? item_mult(a.in, i) : 0ull;
    t.keys[i] = uint32_t(kv);
    t.mult[i] = m;
    uint32_t nulls = 0;
    for (int j = 0; j < a.src.n; j++) {
        uint64_t v = 0;
        if (!slot_value(a.src.s[j], a.in, i, row, a.ps, v)) {
            nulls |= 1u << j;
            v = 0;
        }
        t.pay[size_t(i) * t.width + j] = v;
    }
    t.pnull[i] = nulls;
    if (m == 0) {
        a.is_rep[i] = 0;
        return;
    }
    // The tuple is visible device-wide before its index can be seen in the
    // table; other threads read it with L2 (.cg) loads.
    __threadfence();
    const uint32_t mask = (1u << a.tlog2) - 1;
    uint32_t pos = uint32_t(tuple_hash(t, i) >> (64 - a.tlog2)) & mask;
    for (uint32_t step = 0; step <= mask; step++) {
        const uint32_t cur = atomicCAS(&a.table[pos], 0u, i + 1);
        if (cur == 0) {
            a.is_rep[i] = 1;
            atomicAdd(&a.counts[uint32_t(key_hash(uint32_t(kv)) >> a.shift)], 1u);
            return;
        }
        if (tuple_equal_cg(t, cur - 1, i)) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&t.mult[cur - 1]), (unsigned long long)m);
            a.is_rep[i] = 0;
            return;
        }
        pos = (pos + 1) & mask;
    }
    a.is_rep[i] = 0;
    record_error(a.err, kErrCapacity);
}

__global__ void k_scatter_bloom(TupleBuf t, const uint32_t* __restrict__ is_rep, uint32_t shift,
                                uint2* __restrict__ buckets, uint32_t* __restrict__ cursor, HTView ht,
                                uint32_t* __restrict__ bloom, uint32_t log2w, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.count || !is_rep[i]) return;
    const uint32_t key = t.keys[i];
    const uint32_t b = uint32_t(key_hash(key) >> shift);
    const uint32_t first = buckets[b].x;
    const uint32_t pos = first + atomicAdd(&cursor[b], 1u);
    const uint32_t hh = key_hash_hi(key);
    if (bloom) atomicOr(&bloom[bloom_word_hi(hh, log2w)], bloom_bits_fast(hh, hh >> 5));
    if (pos >= buckets[b + 1].x || pos >= ht.nentries) {
        record_error(err, kErrCapacity);
        return;
    }
    if (pos == first) buckets[b].y = key;  // the bucket's first entry
    const_cast<uint32_t*>(ht.keys)[pos] = key;
    const_cast<uint64_t*>(ht.mult)[pos] = t.mult[i];
    const_cast<uint32_t*>(ht.pnull)[pos] = t.pnull[i];
    uint64_t* dst = const_cast<uint64_t*>(ht.pay) + size_t(pos) * t.width;
    const uint64_t* src = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) dst[j] = src[j];
}

__global__ void k_ht_flags(HTView ht, uint32_t nbuckets, uint32_t* __restrict__ flags) {
    const uint32_t n = ht.buckets[nbuckets].x;  // entries actually stored
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        if (ht.mult[e] > 1) flags[1] = 1;
        uint32_t key = ht.keys[e];
        uint32_t b = uint32_t(key_hash(key) >> ht.shift);
        uint32_t s = ht.buckets[b].x;
        if (e - s > 256) {
            flags[0] = 1;  // long bucket: assume repeats (only steers capacity choices)
            continue;
        }
        for (uint32_t j = s; j < e; j++)
            if (ht.keys[j] == key) {
                flags[0] = 1;
                break;
            }
    }
}

// Hit counts of evenly spaced sample rows against every probe of a pipeline:
// blockIdx.y selects the probe.
__global__ void k_sample_probes(SampleSet set, uint32_t nsample, uint32_t* hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const SampleProbe& sp = set.p[blockIdx.y];
    if (i >= nsample || sp.key.nrows == 0) return;
    const uint32_t row = uint32_t((uint64_t(i) * sp.key.nrows) / nsample);
    uint64_t v;
    if (!col_get(sp.key, row, v)) return;
    const uint32_t k = uint32_t(v);
    const uint32_t b = uint32_t(key_hash(k) >> sp.ht.shift);
    for (uint32_t j = sp.ht.buckets[b].x; j < sp.ht.buckets[b + 1].x; j++)
        if (sp.ht.keys[j] == k) {
            atomicAdd(hits + blockIdx.y, 1u);
            return;
        }
}

} // namespace

int emit_aggregate(const BuildArgs& a, cudaStream_t st) {
    if (!a.tb.count) return 0;
    k_emit_aggregate<<<(a.tb.count + 255) / 256, 256, 0, st>>>(a);
    return 1;
}

int scatter_bloom(TupleBuf t, const uint32_t* is_rep, uint32_t shift, uint2* buckets, uint32_t* cursor,
                  HTView ht_mut, uint32_t* bloom, uint32_t log2w, uint32_t* err, cudaStream_t st) {
    if (!t.count) return 0;
    k_scatter_bloom<<<(t.count + 255) / 256, 256, 0, st>>>(t, is_rep, shift, buckets, cursor, ht_mut, bloom, log2w,
                                                           err);
    return 1;
}

int ht_flags(HTView ht, uint32_t nbuckets, uint32_t* flags, int num_sms, cudaStream_t st) {
    if (!ht.nentries) return 0;
    uint32_t blocks = (ht.nentries + 255) / 256;
    if (blocks > uint32_t(num_sms) * 8) blocks = uint32_t(num_sms) * 8;
    k_ht_flags<<<blocks, 256, 0, st>>>(ht, nbuckets, flags);
    return 1;
}

int sample_probes(const SampleSet& set, uint32_t nsample, uint32_t* hits, cudaStream_t st) {
    cudaMemsetAsync(hits, 0, sizeof(uint32_t) * std::max(set.n, 1), st);
    if (!nsample || set.n <= 0) return 0;
    k_sample_probes<<<dim3((nsample + 255) / 256, unsigned(set.n)), 256, 0, st>>>(set, nsample, hits);
    return 1;
}

} // namespace bj
