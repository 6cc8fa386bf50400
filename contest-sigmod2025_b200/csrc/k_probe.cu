// Pipeline kernels: probe stages, build-side tuple emit, output emit.
//
// Replaces the fused push pipeline of the reference
// (engine/pipeline/JoinPipeline.hpp:46-203: scan -> probe_0 -> probe_1 ->
// target, multiplicity = product of the matched tuples' multiplicities,
// :111-131) with stage kernels over item lists. An item is a row of the
// scanned input plus the hash-table entry matched by every probe so far.
// Against a table with unique keys a stage makes at most one item per input
// item, so it runs once, appending with warp-aggregated atomics and reading
// its input count on the device (no host round trip between stages).
// Otherwise it runs twice over tiles of 256 items: once counting matches per
// tile, once writing at the tile's offset (an exclusive scan of the counts in
// between).
//
// The probe itself follows HashtableProbe::operator() (engine/op/Hashtable.hpp:
// 228-241): hash the 32-bit key, find its bucket, compare every key in the
// bucket. Buckets here are contiguous runs of entries (CSR), not chains.
// INT64 keys (no reference counterpart: the reference reads every join key as
// 32 bits) hash all 64 bits and compare both halves.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {


// Entries of `ht` whose key equals `key`: calls fn(entry) for each.
// `key` is a value slot: an INT32 key zero-extended, or an INT64 key (the
// table then carries keys_hi and no bloom filter).
template <typename Fn>
__device__ __forceinline__ uint32_t for_matches(const HTView& ht, uint64_t key, bool use_bloom, Fn&& fn) {
    if (use_bloom && ht.bloom && !bloom_may_contain(ht.bloom, ht.bloom_log2, uint32_t(key))) return 0;
    const uint32_t b = ht_bucket(ht, key);
    const uint2 b0 = ht.buckets[b];
    const uint32_t e = ht.buckets[b + 1].x;
    uint32_t n = 0;
    if (b0.x < e && b0.y == uint32_t(key) && (!ht.keys_hi || ht.keys_hi[b0.x] == uint32_t(key >> 32))) {
        fn(b0.x);
        n++;
    }
    for (uint32_t j = b0.x + 1; j < e; j++) {
        if (ht_key_eq(ht, j, key)) {
            fn(j);
            n++;
        }
    }
    return n;
}

template <typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* total) {
    __shared__ T warp_sums[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        T w = lane < nw ? warp_sums[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        warp_sums[lane] = wi - w;
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    T r = warp_sums[warp] + inc - v;
    __syncthreads();
    return r;
}

// Key of item i (row `row`) for a stage: a column of the scanned input, or an
// earlier stage's payload.
__device__ __forceinline__ bool stage_key(const DevColumn& key, const KeySource& src, const Items& in, uint32_t i,
                                          uint32_t row, uint32_t* err, uint64_t& v) {
    if (src.stage >= 0) return payload_key(src, in.ents, i, v);
    if (row >= key.nrows) {
        record_error(err, kErrRowRange);
        return false;
    }
    return col_get(key, row, v);
}

template <int kMode>
__global__ void __launch_bounds__(256) k_probe_stage(Items in, DevColumn key, HTView ht, uint32_t* tile_counts,
                                                     const uint32_t* tile_offsets, ItemsOut out, int use_bloom,
                                                     uint32_t* err, uint32_t capacity, KeySource src) {
    uint32_t t0 = blockIdx.x * kTile;
    uint32_t t1 = min(in.count, t0 + kTile);
    unsigned long long mine = 0;
    for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
        uint32_t row = item_row(in, i);
        uint64_t v;
        if (!stage_key(key, src, in, i, row, err, v)) continue;
        mine += for_matches(ht, v, use_bloom != 0, [](uint32_t) {});
    }
    __shared__ unsigned long long total;
    const unsigned long long base = block_exclusive_sum<unsigned long long>(mine, &total);
    if (kMode == 0) {
        // A tile's matches beyond 2^32 - 1 cannot be items (their count is
        // 32-bit): saturate, and the host refuses the stage.
        if (threadIdx.x == 0) {
            if (total > 0xffffffffull) record_error(err, kErrCapacity);
            tile_counts[blockIdx.x] = uint32_t(min(total, 0xffffffffull));
        }
        return;
    }
    unsigned long long o = tile_offsets[blockIdx.x] + base;
    for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
        uint32_t row = item_row(in, i);
        uint64_t v;
        if (!stage_key(key, src, in, i, row, nullptr, v)) continue;
        uint64_t m = item_mult(in, i);
        for_matches(ht, v, use_bloom != 0, [&](uint32_t e) {
            if (o >= capacity) {
                record_error(err, kErrCapacity);
                return;
            }
            out.rows[o] = row;
            for (int p = 0; p < in.nprobes; p++) out.ents[p][o] = in.ents[p][i];
            out.ents[in.nprobes][o] = e;
            out.mult[o] = m * ht.mult[e];
            o++;
        });
    }
}

// A chain of consecutive probe stages against tables with unique keys: every
// item probes stage 0, and while it matches, the next stage, so a row that
// misses is dropped at its first miss (the fused probe_0 -> probe_1 -> ...
// of JoinPipeline.hpp:111-131, with early exit). Persistent grid-stride
// loop, at most one match per stage, warp-aggregated reservation of output
// slots.
__global__ void __launch_bounds__(256) k_probe_chain(Items in, ProbeChain ch, ItemsOut out, uint32_t* cursor,
                                                     uint32_t capacity, uint32_t* err, const uint32_t* dfirst,
                                                     uint32_t* dend) {
    const uint32_t n = in.dcount ? *in.dcount : in.count;
    const uint32_t first = dfirst ? *dfirst : 0u;
    if (dend && blockIdx.x == 0 && threadIdx.x == 0) *dend = n;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31;
    // Whole warps iterate together so the ballot sees every lane.
    for (uint32_t base = first + (blockIdx.x * blockDim.x + threadIdx.x) - lane; base < n; base += stride) {
        const uint32_t i = base + lane;
        bool hit = i < n;
        uint32_t row = 0;
        uint32_t e[kMaxChain];
        if (hit) row = item_row(in, i);
#pragma unroll
        for (int t = 0; t < kMaxChain; t++) {
            e[t] = 0;
            if (t >= ch.n || !hit) continue;
            const ChainStage& c = ch.st[t];
            uint64_t v;
            if (!stage_key(c.key, c.src, in, i, row, err, v)) {
                hit = false;
            } else {
                bool found = false;
                for_matches(c.ht, v, c.use_bloom != 0, [&](uint32_t j) {
                    if (!found) e[t] = j;
                    found = true;
                });
                hit = found;
            }
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, hit);
        if (!mask) continue;
        uint32_t wbase = 0;
        if (lane == 0) wbase = atomicAdd(cursor, __popc(mask));
        wbase = __shfl_sync(0xffffffffu, wbase, 0);
        if (!hit) continue;
        const uint32_t o = wbase + __popc(mask & ((1u << lane) - 1));
        if (o >= capacity) {
            record_error(err, kErrCapacity);
            continue;
        }
        out.rows[o] = row;
        for (int p = 0; p < in.nprobes; p++) out.ents[p][o] = in.ents[p][i];
        uint64_t m = item_mult(in, i);
#pragma unroll
        for (int t = 0; t < kMaxChain; t++) {
            if (t >= ch.n) continue;
            out.ents[in.nprobes + t][o] = e[t];
            m *= ch.st[t].ht.mult[e[t]];
        }
        if (out.mult) out.mult[o] = m;
    }
}

__global__ void k_items_mult(Items in, uint64_t* mult_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < in.count) mult_out[i] = item_mult(in, i);
}

__global__ void __launch_bounds__(256) k_emit_output(Items in, const uint64_t* out_off, SlotSources src, ProbeSet ps,
                                                     FlatOut out, uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= in.count) return;
    uint32_t row = item_row(in, i);
    // Without offsets every item is one output row.
    uint64_t o0 = out_off ? out_off[i] : i, o1 = out_off ? out_off[i + 1] : i + 1;
    for (int j = 0; j < src.n; j++) {
        if (!out.vals[j]) continue;  // a slot the page writer reads from the items
        uint64_t v = 0;
        bool ok = slot_value(src.s[j], in, i, row, ps, v);
        for (uint64_t o = o0; o < o1; o++) {
            out.vals[j][o] = ok ? v : 0;
            out.valid[j][o] = ok;
        }
    }
}

} // namespace

int probe_stage(const Items& in, const DevColumn& key, const HTView& ht, int mode, uint32_t* tile_counts,
                const uint32_t* tile_offsets, ItemsOut out, bool use_bloom, uint32_t* err, cudaStream_t st,
                uint32_t capacity, KeySource src) {
    uint32_t tiles = (in.count + kTile - 1) / kTile;
    if (!tiles) return 0;
    if (mode == 0)
        k_probe_stage<0><<<tiles, 256, 0, st>>>(in, key, ht, tile_counts, tile_offsets, out, use_bloom, err,
                                                 capacity, src);
    else
        k_probe_stage<1><<<tiles, 256, 0, st>>>(in, key, ht, tile_counts, tile_offsets, out, use_bloom, err,
                                                 capacity, src);
    return 1;
}

int probe_chain_unique(const Items& in, const ProbeChain& chain, ItemsOut out, uint32_t* cursor, uint32_t capacity,
                       uint32_t* err, int num_sms, cudaStream_t st, const uint32_t* dfirst, uint32_t* dend) {
    if (!in.count || chain.n <= 0) return 0;
    uint32_t blocks = std::min<uint32_t>((in.count + 255) / 256, uint32_t(num_sms) * 8);
    k_probe_chain<<<blocks, 256, 0, st>>>(in, chain, out, cursor, capacity, err, dfirst, dend);
    return 1;
}

int items_mult(const Items& in, uint64_t* mult_out, cudaStream_t st) {
    if (!in.count) return 0;
    k_items_mult<<<(in.count + 255) / 256, 256, 0, st>>>(in, mult_out);
    return 1;
}

int emit_output(const Items& in, const uint64_t* out_off, const SlotSources& src, const HTView* probes, FlatOut out,
                uint32_t* err, cudaStream_t st) {
    if (!in.count) return 0;
    k_emit_output<<<(in.count + 255) / 256, 256, 0, st>>>(in, out_off, src, make_probe_set(probes, in.nprobes), out,
                                                          err);
    return 1;
}

} // namespace bj
