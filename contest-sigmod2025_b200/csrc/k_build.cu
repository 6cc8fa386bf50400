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
//  1. emit (each thread writes its tuple: key, NULL mask, payload,
//     multiplicity), then eager aggregation and bucket counts (K6) in the next
//     launch: each tuple's index goes into an open-addressing table keyed by
//     the whole tuple. The first copy of each distinct tuple claims a slot
//     with atomicCAS and becomes its representative (and counts itself into
//     its bucket); every other copy adds its multiplicity to the
//     representative with atomicAdd. Unlike the reference, which only merges
//     with the current bucket head, this folds every duplicate. Builds whose
//     tuples cannot repeat (BuildArgs::distinct) count in the emit and skip
//     the aggregation launch.
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
#include <cstdlib>

namespace bj {
namespace {

__device__ __forceinline__ uint64_t tuple_key(const TupleBuf& t, uint32_t i) {
    return uint64_t(t.keys[i]) | (t.keys_hi ? uint64_t(t.keys_hi[i]) << 32 : 0ull);
}

__device__ __forceinline__ uint64_t tuple_hash(const TupleBuf& t, uint32_t i) {
    uint64_t h = mix64(uint64_t(t.keys[i]) ^ (uint64_t(t.pnull[i]) << 32));
    if (t.keys_hi) h = mix64(h ^ t.keys_hi[i]);
    const uint64_t* p = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) h = mix64(h ^ (p[j] + 0x9E3779B97F4A7C15ull * (j + 1)));
    return h;
}

// Tuple a (written by another thread, read through L2) equals tuple b.
__device__ __forceinline__ bool tuple_equal_cg(const TupleBuf& t, uint32_t a, uint32_t b) {
    if (__ldcg(t.keys + a) != t.keys[b] || __ldcg(t.pnull + a) != t.pnull[b]) return false;
    if (t.keys_hi && __ldcg(t.keys_hi + a) != t.keys_hi[b]) return false;
    const uint64_t* pa = t.pay + size_t(a) * t.width;
    const uint64_t* pb = t.pay + size_t(b) * t.width;
    for (uint32_t j = 0; j < t.width; j++)
        if (__ldcg(pa + j) != pb[j]) return false;
    return true;
}

// Where a build's tuples go (the parts of BuildArgs the emit writes).
struct EmitTarget {
    TupleBuf tb;
    uint32_t* table;
    uint32_t tlog2;
    uint32_t* is_rep;
    uint32_t* counts;
    uint32_t shift;
    uint32_t distinct;
    uint32_t* err;
};

// Writes tuple i of a build (key kv; multiplicity m, 0 for a NULL key; the
// slot values from slot(j, v), false for NULL). A zero-multiplicity tuple
// represents nothing; a tuple of a distinct build represents itself and is
// counted into its bucket here. The others are folded by aggregate_tuple in
// a later launch, which sees every tuple written (no fence needed here).
template <typename Slot>
__device__ __forceinline__ void emit_tuple_to(const EmitTarget& a, uint32_t i, uint64_t kv, uint64_t m, int nslots,
                                              Slot&& slot) {
    const TupleBuf& t = a.tb;
    t.keys[i] = uint32_t(kv);
    if (t.keys_hi) t.keys_hi[i] = uint32_t(kv >> 32);
    t.mult[i] = m;
    uint32_t nulls = 0;
    for (int j = 0; j < nslots; j++) {
        uint64_t v = 0;
        if (!slot(j, v)) {
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
    if (a.distinct) {
        a.is_rep[i] = 1;
        atomicAdd(&a.counts[bucket_of(kv, t.keys_hi != nullptr, a.shift)], 1u);
    }
}

// Eager aggregation of tuple i (every tuple written by an earlier launch):
// the first copy of a distinct tuple to claim a slot of the open-addressing
// table keyed by the whole tuple represents it and is counted into its
// bucket; every other copy adds its multiplicity to the representative.
__device__ __forceinline__ void aggregate_tuple(const EmitTarget& a, uint32_t i) {
    const TupleBuf& t = a.tb;
    const uint64_t m = t.mult[i];  // only a representative's grows, after it claimed its slot
    if (m == 0) return;
    const uint32_t mask = (1u << a.tlog2) - 1;
    uint32_t pos = uint32_t(tuple_hash(t, i) >> (64 - a.tlog2)) & mask;
    for (uint32_t step = 0; step <= mask; step++) {
        const uint32_t cur = atomicCAS(&a.table[pos], 0u, i + 1);
        if (cur == 0) {
            a.is_rep[i] = 1;
            atomicAdd(&a.counts[bucket_of(tuple_key(t, i), t.keys_hi != nullptr, a.shift)], 1u);
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

__device__ __forceinline__ EmitTarget emit_target(const BuildArgs& a) {
    return EmitTarget{a.tb, a.table, a.tlog2, a.is_rep, a.counts, a.shift, a.distinct, a.err};
}

// Writes tuple i of a build.
__device__ __forceinline__ void emit_tuple(const BuildArgs& a, uint32_t i) {
    const uint32_t row = item_row(a.in, i);
    uint64_t kv = 0;
    bool key_ok;
    if (a.key_stage >= 0) {
        // The key is an attribute of an input probed by this pipeline.
        const HTView& src = a.ps.ht[a.key_stage];
        const uint32_t e = a.in.ents[a.key_stage][i];
        key_ok = !((src.pnull[e] >> a.key_slot) & 1);
        if (key_ok) kv = src.pay[size_t(e) * src.width + a.key_slot];
    } else {
        key_ok = row < a.key.nrows && col_get(a.key, row, kv);
        if (row >= a.key.nrows) record_error(a.err, kErrRowRange);
    }
    if (key_ok && a.rbloom && !bloom_may_contain(a.rbloom, a.rlog2w, uint32_t(kv))) key_ok = false;
    const uint64_t m = key_ok ? item_mult(a.in, i) : 0ull;
    emit_tuple_to(emit_target(a), i, kv, m, a.src.n,
                  [&](int j, uint64_t& v) { return slot_value(a.src.s[j], a.in, i, row, a.ps, v); });
}

__global__ void __launch_bounds__(256) k_emit(BuildArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.tb.count) emit_tuple(a, i);
}

__global__ void __launch_bounds__(256) k_aggregate(BuildArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.tb.count) aggregate_tuple(emit_target(a), i);
}

// Places representative i in its bucket's range and sets its bloom bits.
__device__ __forceinline__ void scatter_tuple(const TupleBuf& t, const uint32_t* __restrict__ is_rep, uint32_t shift,
                                              uint2* __restrict__ buckets, uint32_t* __restrict__ cursor,
                                              const HTView& ht, uint32_t* __restrict__ bloom, uint32_t log2w,
                                              uint32_t* __restrict__ err, uint32_t i) {
    if (!is_rep[i]) return;
    const uint32_t key = t.keys[i];
    const uint32_t b = bucket_of(tuple_key(t, i), t.keys_hi != nullptr, shift);
    const uint32_t first = buckets[b].x;
    const uint32_t pos = first + atomicAdd(&cursor[b], 1u);
    if (bloom) {  // INT32 keys only (INT64 tables are built without a filter)
        const uint32_t hh = key_hash_hi(key);
        atomicOr(&bloom[bloom_word_hi(hh, log2w)], bloom_bits_fast(hh, hh >> 5));
    }
    if (pos >= buckets[b + 1].x || pos >= ht.nentries) {
        record_error(err, kErrCapacity);
        return;
    }
    if (pos == first) buckets[b].y = key;  // the bucket's first entry
    const_cast<uint32_t*>(ht.keys)[pos] = key;
    if (t.keys_hi) const_cast<uint32_t*>(ht.keys_hi)[pos] = t.keys_hi[i];
    const_cast<uint64_t*>(ht.mult)[pos] = t.mult[i];
    const_cast<uint32_t*>(ht.pnull)[pos] = t.pnull[i];
    uint64_t* dst = const_cast<uint64_t*>(ht.pay) + size_t(pos) * t.width;
    const uint64_t* src = t.pay + size_t(i) * t.width;
    for (uint32_t j = 0; j < t.width; j++) dst[j] = src[j];
}

__global__ void k_scatter_bloom(TupleBuf t, const uint32_t* __restrict__ is_rep, uint32_t shift,
                                uint2* __restrict__ buckets, uint32_t* __restrict__ cursor, HTView ht,
                                uint32_t* __restrict__ bloom, uint32_t log2w, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < t.count) scatter_tuple(t, is_rep, shift, buckets, cursor, ht, bloom, log2w, err, i);
}

// Flags of entry e of a built table (see ht_flags).
__device__ __forceinline__ void flag_entry(const HTView& ht, uint32_t e, uint32_t* __restrict__ flags) {
    if (ht.mult[e] > 1) flags[1] = 1;
    const uint64_t key = ht_key(ht, e);
    uint32_t b = ht_bucket(ht, key);
    uint32_t s = ht.buckets[b].x;
    if (e - s > 256) {
        flags[0] = 1;  // long bucket: assume repeats (only steers capacity choices)
        return;
    }
    for (uint32_t j = s; j < e; j++)
        if (ht_key_eq(ht, j, key)) {
            flags[0] = 1;
            break;
        }
}

__global__ void k_ht_flags(HTView ht, uint32_t nbuckets, uint32_t* __restrict__ flags) {
    const uint32_t n = ht.buckets[nbuckets].x;  // entries actually stored
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        flag_entry(ht, e, flags);
}

// ---- leaf builds of a query, batched ----
//
// Builds whose input probes nothing (a query's leaves) run together: each of
// the passes above is one launch over all builds' tuples or buckets at once
// (blocks find their build from prefix sums of the builds' sizes), so the
// leaves of a query cost four launches (five with the table flags) instead
// of three or four per build, and the builds' small grids fill the GPU
// together: 1. emit + aggregation + bucket counts; 2a. sums of bucket tiles
// of 1024 counts; 2b. each tile's exclusive offsets (the sums of the earlier
// tiles of its build plus a block scan) into the buckets' x words, and the
// build's total into bucket nb; 3. scatter + bloom; 4. table flags.

constexpr uint32_t kLeafTile = 1024;  // bucket counts per tile in pass 2

__device__ __forceinline__ int leaf_of(const uint32_t* start, int n, uint32_t x) {
    int b = 0;
    while (b + 1 < n && x >= start[b + 1]) b++;
    return b;
}

__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v) {
    __shared__ uint32_t ws[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) t += ws[w];
    __syncthreads();
    return t;
}

// Exclusive prefix of v over the block (256 threads), in thread order.
__device__ __forceinline__ uint32_t block_excl_u32(uint32_t v) {
    __shared__ uint32_t ws[8];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= uint32_t(o)) inc += u;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    uint32_t base = 0;
    for (uint32_t w = 0; w < warp; w++) base += ws[w];
    __syncthreads();
    return base + inc - v;
}

// Blocks of 256 tuples, each within one build (block_start: prefix of the
// builds' block counts), so a block's build and its arguments are uniform.
__device__ __forceinline__ bool leaf_tuple(const LeafBatch& B, int& b, uint32_t& i) {
    b = leaf_of(B.block_start, B.n, blockIdx.x);
    i = (blockIdx.x - B.block_start[b]) * blockDim.x + threadIdx.x;
    return i < B.tuple_start[b + 1] - B.tuple_start[b];
}

__device__ __forceinline__ EmitTarget leaf_target(const LeafBatch& B, const LeafBuild& L) {
    return EmitTarget{L.tb, L.table, L.tlog2, L.is_rep, L.counts, L.shift, L.distinct, B.err};
}

__global__ void __launch_bounds__(256) k_leaf_emit(LeafBatch B) {
    int b;
    uint32_t i;
    if (!leaf_tuple(B, b, i)) return;
    const LeafBuild& L = B.l[b];
    // A leaf's item i is row i, multiplicity 1; its slots are its own columns.
    // A row whose key the restricting filter cannot hold joins nothing: it
    // is written with multiplicity 0, like a NULL key.
    uint64_t kv = 0;
    const bool key_ok = col_get(L.key, i, kv) && (!L.rbloom || bloom_may_contain(L.rbloom, L.rlog2w, uint32_t(kv)));
    emit_tuple_to(leaf_target(B, L), i, kv, key_ok ? 1ull : 0ull, L.nslots,
                  [&](int j, uint64_t& v) { return column_value(L.cols[j], i, v); });
}

// Aggregation pass of the leaves that are not distinct (launched only when
// some leaf of the batch is not).
__global__ void __launch_bounds__(256) k_leaf_aggregate(LeafBatch B) {
    int b;
    uint32_t i;
    if (!leaf_tuple(B, b, i)) return;
    const LeafBuild& L = B.l[b];
    if (!L.distinct) aggregate_tuple(leaf_target(B, L), i);
}

// One block per tile of 1024 bucket counts.
__global__ void __launch_bounds__(256) k_leaf_tile_sums(LeafBatch B) {
    const uint32_t tile = blockIdx.x;
    const int b = leaf_of(B.tile_start, B.n, tile);
    const LeafBuild& L = B.l[b];
    const uint32_t i0 = (tile - B.tile_start[b]) * kLeafTile, i1 = min(i0 + kLeafTile, L.nb);
    uint32_t v = 0;
    for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) v += L.counts[i];
    v = block_sum_u32(v);
    if (threadIdx.x == 0) B.tile_sums[tile] = v;
}

// One block per tile; thread k takes counts 4k..4k+3 of the tile.
__global__ void __launch_bounds__(256) k_leaf_offsets(LeafBatch B) {
    const uint32_t tile = blockIdx.x;
    const int b = leaf_of(B.tile_start, B.n, tile);
    const LeafBuild& L = B.l[b];
    const uint32_t first = B.tile_start[b];
    uint32_t before = 0;
    for (uint32_t k = first + threadIdx.x; k < tile; k += blockDim.x) before += B.tile_sums[k];
    before = block_sum_u32(before);
    const uint32_t i0 = (tile - first) * kLeafTile + 4 * threadIdx.x;
    uint32_t c[4], own = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        c[j] = i0 + j < L.nb ? L.counts[i0 + j] : 0u;
        own += c[j];
    }
    uint32_t run = before + block_excl_u32(own);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (i0 + j < L.nb) L.buckets[i0 + j].x = run;
        run += c[j];
    }
    if (i0 < L.nb && i0 + 4 >= L.nb) L.buckets[L.nb].x = run;  // the build's total
}

__global__ void __launch_bounds__(256) k_leaf_scatter(LeafBatch B) {
    int b;
    uint32_t i;
    if (!leaf_tuple(B, b, i)) return;
    const LeafBuild& L = B.l[b];
    scatter_tuple(L.tb, L.is_rep, L.shift, L.buckets, L.cursor, L.ht, L.bloom, L.log2w, B.err, i);
}

// Entries are numbered like tuples (a build stores at most its tuple count).
__global__ void __launch_bounds__(256) k_leaf_flags(LeafBatch B) {
    int b;
    uint32_t e;
    if (!leaf_tuple(B, b, e)) return;
    const LeafBuild& L = B.l[b];
    if (e < L.buckets[L.nb].x) flag_entry(L.ht, e, L.dflags);
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
    const uint32_t b = ht_bucket(sp.ht, v);
    for (uint32_t j = sp.ht.buckets[b].x; j < sp.ht.buckets[b + 1].x; j++)
        if (ht_key_eq(sp.ht, j, v)) {
            atomicAdd(hits + blockIdx.y, 1u);
            return;
        }
}

} // namespace

int emit_aggregate(const BuildArgs& a, cudaStream_t st) {
    if (!a.tb.count) return 0;
    const uint32_t blocks = (a.tb.count + 255) / 256;
    k_emit<<<blocks, 256, 0, st>>>(a);
    if (a.distinct) return 1;
    k_aggregate<<<blocks, 256, 0, st>>>(a);
    return 2;
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

int build_leaves(const LeafBatch& batch, cudaStream_t st) {
    const uint32_t tuples = batch.tuple_start[batch.n], tiles = batch.tile_start[batch.n];
    if (batch.n <= 0 || tuples == 0) return 0;
    const uint32_t blocks = batch.block_start[batch.n];
    bool all_distinct = true;
    for (int b = 0; b < batch.n; b++) all_distinct = all_distinct && batch.l[b].distinct;
    k_leaf_emit<<<blocks, 256, 0, st>>>(batch);
    if (!all_distinct) k_leaf_aggregate<<<blocks, 256, 0, st>>>(batch);
    k_leaf_tile_sums<<<tiles, 256, 0, st>>>(batch);
    k_leaf_offsets<<<tiles, 256, 0, st>>>(batch);
    k_leaf_scatter<<<blocks, 256, 0, st>>>(batch);
    const int launches = all_distinct ? 4 : 5;
    if (!batch.flags) return launches;
    k_leaf_flags<<<blocks, 256, 0, st>>>(batch);
    return launches + 1;
}

int sample_probes(const SampleSet& set, uint32_t nsample, uint32_t* hits, cudaStream_t st) {
    cudaMemsetAsync(hits, 0, sizeof(uint32_t) * std::max(set.n, 1), st);
    if (!nsample || set.n <= 0) return 0;
    k_sample_probes<<<dim3((nsample + 255) / 256, unsigned(set.n)), 256, 0, st>>>(set, nsample, hits);
    return 1;
}

} // namespace bj
