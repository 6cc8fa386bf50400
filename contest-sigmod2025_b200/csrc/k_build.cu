// K3/K4/K6: hash-table build.
//
// The reference builds a chaining table per partition: tuples are appended to
// per-thread chunks (HashtableBuild::operator(), engine/op/Hashtable.hpp:
// 176-203), then every partition is inserted bucket-head first, setting a
// 16-bit bloom word per bucket and folding a tuple into the bucket head when
// key and payload are equal (eager aggregation, engine/op/Hashtable.cpp:
// 208-263). Sizing: 2^max(bit_width(n), 4) buckets (Hashtable.cpp:94-104).
//
// On the GPU the build is three passes over the emitted tuples:
//  1. eager aggregation (K6): an open-addressing table of tuple indices keyed
//     by the whole tuple (key, NULL mask, payload). The first copy of each
//     distinct tuple claims a slot with atomicCAS and becomes its
//     representative; every other copy adds its multiplicity to the
//     representative with atomicAdd. Unlike the reference, which only merges
//     with the current bucket head, this folds every duplicate.
//  2. bucket counts with atomicAdd, an exclusive scan, and a scatter of the
//     representatives into their bucket's contiguous range (K4). The same
//     bucket index as the reference: key_hash(key) >> shift.
//  3. a blocked bloom filter, one 32-bit word per key with 3-4 bits set (K3),
//     at most 128 KiB so scans can stage it in shared memory; probes consult
//     it before touching the buckets.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {

constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ uint64_t tuple_hash(const TupleBuf& t, uint32_t i) {
    uint64_t h = mix64(uint64_t(t.keys[i]) ^ (uint64_t(t.pnull[i]) << 32));
    const uint64_t* p = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) h = mix64(h ^ (p[j] + 0x9E3779B97F4A7C15ull * (j + 1)));
    return h;
}

__device__ __forceinline__ bool tuple_equal(const TupleBuf& t, uint32_t a, uint32_t b) {
    if (t.keys[a] != t.keys[b] || t.pnull[a] != t.pnull[b]) return false;
    const uint64_t* pa = t.pay + size_t(a) * t.width;
    const uint64_t* pb = t.pay + size_t(b) * t.width;
    for (uint32_t j = 0; j < t.width; j++)
        if (pa[j] != pb[j]) return false;
    return true;
}

__global__ void k_aggregate(TupleBuf t, uint32_t* __restrict__ table, uint32_t log2, uint32_t* __restrict__ is_rep,
                            uint32_t* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.count) return;
    if (t.mult[i] == 0) {
        is_rep[i] = 0;
        return;
    }
    uint32_t mask = (1u << log2) - 1;
    uint32_t pos = uint32_t(tuple_hash(t, i) >> (64 - log2)) & mask;
    for (uint32_t step = 0; step <= mask; step++) {
        uint32_t cur = table[pos];
        if (cur == kEmpty) {
            uint32_t old = atomicCAS(&table[pos], kEmpty, i);
            if (old == kEmpty) {
                is_rep[i] = 1;
                return;
            }
            cur = old;
        }
        if (tuple_equal(t, cur, i)) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&t.mult[cur]), (unsigned long long)t.mult[i]);
            is_rep[i] = 0;
            return;
        }
        pos = (pos + 1) & mask;
    }
    is_rep[i] = 0;
    record_error(err, kErrCapacity);
}

__global__ void k_bucket_count(TupleBuf t, const uint32_t* __restrict__ is_rep, uint32_t shift,
                               uint32_t* __restrict__ counts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.count || !is_rep[i]) return;
    atomicAdd(&counts[uint32_t(key_hash(t.keys[i]) >> shift)], 1u);
}

__global__ void k_bucket_scatter(TupleBuf t, const uint32_t* __restrict__ is_rep, uint32_t shift,
                                 const uint32_t* __restrict__ bucket_off, uint32_t* __restrict__ cursor, HTView ht,
                                 uint32_t* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.count || !is_rep[i]) return;
    uint32_t b = uint32_t(key_hash(t.keys[i]) >> shift);
    uint32_t pos = bucket_off[b] + atomicAdd(&cursor[b], 1u);
    if (pos >= bucket_off[b + 1] || pos >= ht.nentries) {
        record_error(err, kErrCapacity);
        return;
    }
    const_cast<uint32_t*>(ht.keys)[pos] = t.keys[i];
    const_cast<uint64_t*>(ht.mult)[pos] = t.mult[i];
    const_cast<uint32_t*>(ht.pnull)[pos] = t.pnull[i];
    uint64_t* dst = const_cast<uint64_t*>(ht.pay) + size_t(pos) * t.width;
    const uint64_t* src = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) dst[j] = src[j];
}

__global__ void k_bloom_build(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ mask, uint32_t n,
                              uint32_t* __restrict__ bloom, uint32_t log2w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (mask && !mask[i])) return;
    const uint32_t hh = key_hash_hi(keys[i]);
    atomicOr(&bloom[bloom_word_hi(hh, log2w)], bloom_bits_fast(hh, hh >> 5));
}

__global__ void k_ht_flags(HTView ht, uint32_t nbuckets, uint32_t* __restrict__ flags) {
    const uint32_t n = ht.bucket_off[nbuckets];  // entries actually stored
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        if (ht.mult[e] > 1) flags[1] = 1;
        uint32_t key = ht.keys[e];
        uint32_t b = uint32_t(key_hash(key) >> ht.shift);
        uint32_t s = ht.bucket_off[b];
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
    for (uint32_t j = sp.ht.bucket_off[b]; j < sp.ht.bucket_off[b + 1]; j++)
        if (sp.ht.keys[j] == k) {
            atomicAdd(hits + blockIdx.y, 1u);
            return;
        }
}

} // namespace

int aggregate_tuples(TupleBuf t, uint32_t* slot_table, uint32_t table_log2, uint32_t* is_rep, uint32_t* err,
                     cudaStream_t st) {
    if (!t.count) return 0;
    cudaMemsetAsync(slot_table, 0xff, sizeof(uint32_t) << table_log2, st);
    k_aggregate<<<(t.count + 255) / 256, 256, 0, st>>>(t, slot_table, table_log2, is_rep, err);
    return 1;
}

int bucket_count(TupleBuf t, const uint32_t* is_rep, uint32_t shift, uint32_t* counts, cudaStream_t st) {
    if (!t.count) return 0;
    k_bucket_count<<<(t.count + 255) / 256, 256, 0, st>>>(t, is_rep, shift, counts);
    return 1;
}

int bucket_scatter(TupleBuf t, const uint32_t* is_rep, uint32_t shift, const uint32_t* bucket_off, uint32_t* cursor,
                   HTView ht_mut, uint32_t* err, cudaStream_t st) {
    if (!t.count) return 0;
    k_bucket_scatter<<<(t.count + 255) / 256, 256, 0, st>>>(t, is_rep, shift, bucket_off, cursor, ht_mut, err);
    return 1;
}

int bloom_build(const uint32_t* keys, const uint32_t* mask, uint32_t n, uint32_t* bloom, uint32_t log2w,
                cudaStream_t st) {
    cudaMemsetAsync(bloom, 0, sizeof(uint32_t) << log2w, st);
    if (!n) return 0;
    k_bloom_build<<<(n + 255) / 256, 256, 0, st>>>(keys, mask, n, bloom, log2w);
    return 1;
}

int ht_flags(HTView ht, uint32_t nbuckets, uint32_t* flags, int num_sms, cudaStream_t st) {
    cudaMemsetAsync(flags, 0, 2 * sizeof(uint32_t), st);
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
