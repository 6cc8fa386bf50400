// Column statistics, exact sub-plan cardinalities and join samples: the
// inputs of join ordering.
//
// The reference estimates cardinalities from 64 sampled rows per base table
// (engine/query/QueryPlan.cpp:719-746, TableScan.cpp:743-772): a row's key is
// tested against the restrictions of its equivalence class, and an input's
// cardinality is its rows times the share of sampled rows that pass
// (QueryPlan.cpp:67-72). The kernels here provide what join ordering needs on
// the device:
//
//  * k_col_stats: per join-key column, a 64-bin histogram of its non-null
//    values by the top six bits of the key hash, and a key -> count map (the
//    index the join samples and exact counts look keys up in);
//  * k_count_node: one table of a connected sub-plan in the exact count of
//    its join result, by weights instead of rows (a row's weight is the
//    number of join results it takes part in below it): children's maps are
//    looked up, weights multiplied, and summed into the parent-edge key's
//    map, or into the total at the root, so a count never materialises a
//    join result;
//  * k_sample_edges: for every directed join edge, how many of 64 sampled
//    rows of one side find their key in the other side's map (the
//    reference's join sample).
#include "launch.h"

#include <cuda_runtime.h>

namespace bj {
namespace {

constexpr unsigned long long kMapEmpty = ~0ull;

__device__ __forceinline__ uint32_t map_slot(uint64_t key, uint32_t log2cap) {
    return uint32_t(mix64(key) >> (64 - log2cap));
}

// Adds v to key's value (inserting the key). The key ~0ull, which marks empty
// slots, keeps its value in vals[cap].
__device__ __forceinline__ void map_add(const KeyMap& m, uint64_t key, unsigned long long v, unsigned int* distinct,
                                        uint32_t* err) {
    const uint32_t cap = 1u << m.log2cap;
    if (key == kMapEmpty) {
        if (atomicAdd(&m.vals[cap], v) == 0 && distinct) atomicAdd(distinct, 1u);
        return;
    }
    uint32_t pos = map_slot(key, m.log2cap);
    for (uint32_t step = 0; step < cap; step++) {
        unsigned long long cur = m.keys[pos];
        if (cur == kMapEmpty) {
            cur = atomicCAS(&m.keys[pos], kMapEmpty, key);
            if (cur == kMapEmpty) {
                if (distinct) atomicAdd(distinct, 1u);
                cur = key;
            }
        }
        if (cur == key) {
            atomicAdd(&m.vals[pos], v);
            return;
        }
        pos = (pos + 1) & (cap - 1);
    }
    record_error(err, kErrCapacity);
}

__device__ __forceinline__ unsigned long long map_get(const KeyMap& m, uint64_t key) {
    const uint32_t cap = 1u << m.log2cap;
    if (key == kMapEmpty) return m.vals[cap];
    uint32_t pos = map_slot(key, m.log2cap);
    for (uint32_t step = 0; step < cap; step++) {
        const unsigned long long cur = m.keys[pos];
        if (cur == key) return m.vals[pos];
        if (cur == kMapEmpty) return 0;
        pos = (pos + 1) & (cap - 1);
    }
    return 0;
}

__global__ void k_map_clear(KeyMap m) {
    const uint32_t cap = 1u << m.log2cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= cap; i += gridDim.x * blockDim.x) {
        if (i < cap) m.keys[i] = kMapEmpty;
        m.vals[i] = 0;
    }
}

// One CTA per page (grid-stride): a page stores its non-null values densely,
// so the histogram and the map need neither the bitmap nor the row index.
__global__ void __launch_bounds__(256) k_col_stats(DevColumn c, KeyMap m, uint32_t* hist, unsigned int* totals,
                                                   uint32_t* err) {
    __shared__ uint32_t h[kHistBins];
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t width = c.type == kInt32 ? 4 : 8;
    uint32_t nonnull = 0;
    for (uint32_t p = blockIdx.x; p < c.npages; p += gridDim.x) {
        const uint8_t* pg = c.pages + size_t(p) * kPageSize;
        const uint32_t hd = c.hdr ? c.hdr[p] : *reinterpret_cast<const uint32_t*>(pg);
        const uint32_t nn = hd >> 16;
        const uint32_t base = width;  // values start at byte 4 (INT32) or 8 (INT64)
        for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) {
            uint64_t key = width == 4 ? uint64_t(*reinterpret_cast<const uint32_t*>(pg + base + 4 * i))
                                      : *reinterpret_cast<const uint64_t*>(pg + base + 8 * size_t(i));
            atomicAdd(&h[key_hash_any(key, c.type) >> 58], 1u);
            map_add(m, key, 1ull, &totals[1], err);
            nonnull++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) nonnull += __shfl_down_sync(0xffffffffu, nonnull, o);
    if ((threadIdx.x & 31) == 0 && nonnull) atomicAdd(&totals[0], nonnull);
    __syncthreads();
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Saturating u64 product (a count beyond 2^64 - 1 sets the overflow flag).
__device__ __forceinline__ unsigned long long mul_sat(unsigned long long a, unsigned long long b, bool& over) {
    if (a && b && __umul64hi(a, b)) {
        over = true;
        return ~0ull;
    }
    return a * b;
}

__global__ void __launch_bounds__(256) k_count_node(CountNode n, uint32_t* err) {
    unsigned long long local = 0;
    bool over = false;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n.nrows; r += gridDim.x * blockDim.x) {
        unsigned long long w = 1;
        for (int j = 0; j < n.nch && w; j++) {
            uint64_t k;
            if (!col_get(n.ch[j].key, r, k)) {
                w = 0;
                break;
            }
            w = mul_sat(w, map_get(n.ch[j].map, k), over);
        }
        if (!w) continue;
        if (n.has_out) {
            uint64_t k;
            if (col_get(n.pkey, r, k)) map_add(n.out, k, w, nullptr, err);
        } else {
            const unsigned long long s = local + w;
            if (s < local) over = true;
            local = s;
        }
    }
    if (!n.has_out) {
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((threadIdx.x & 31) == 0 && local) atomicAdd(n.total, local);
    }
    if (over) atomicOr(n.flags, 1u);
}

// Row i of a sample: a seeded position (the reference samples 64 rows with
// its own seeded generator, engine/infra/Random.hpp:7-29).
__global__ void k_sample_edges(SampleEdges e, uint32_t nsample, uint32_t* hits) {
    const int d = blockIdx.x;
    if (d >= e.n) return;
    const SampleEdge& s = e.e[d];
    uint32_t mine = 0;
    for (uint32_t i = threadIdx.x; i < nsample && s.key.nrows; i += blockDim.x) {
        const uint32_t row = uint32_t(mix64(0x5a17ull * (d + 1) + i + (uint64_t(s.seed) << 32)) % s.key.nrows);
        uint64_t k;
        if (col_get(s.key, row, k) && map_get(s.map, k) != 0) mine++;
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&hits[d], mine);
}

} // namespace

int map_clear(const KeyMap& m, cudaStream_t st) {
    const uint32_t cap = 1u << m.log2cap;
    const uint32_t blocks = std::min<uint32_t>((cap + 256) / 256, 148 * 8);
    k_map_clear<<<blocks, 256, 0, st>>>(m);
    return 1;
}

int column_stats(const DevColumn& c, const KeyMap& m, uint32_t* hist, unsigned int* totals, uint32_t* err, int num_sms,
                 cudaStream_t st) {
    if (!c.npages) return 0;
    const uint32_t blocks = std::min<uint32_t>(c.npages, uint32_t(num_sms) * 8);
    k_col_stats<<<blocks, 256, 0, st>>>(c, m, hist, totals, err);
    return 1;
}

int count_node(const CountNode& n, uint32_t* err, int num_sms, cudaStream_t st) {
    if (!n.nrows) return 0;
    const uint32_t blocks = std::min<uint32_t>((n.nrows + 255) / 256, uint32_t(num_sms) * 8);
    k_count_node<<<blocks, 256, 0, st>>>(n, err);
    return 1;
}

int sample_edges(const SampleEdges& e, uint32_t nsample, uint32_t* hits, cudaStream_t st) {
    if (!e.n) return 0;
    k_sample_edges<<<e.n, 64, 0, st>>>(e, nsample, hits);
    return 1;
}

} // namespace bj
