// Device-wide exclusive prefix sums and fills.
// A single pass over tiles of 4096 values (1024 threads x 4) with decoupled
// look-back (Merrill and Garland, "Single-pass Parallel Prefix Scan with
// Decoupled Look-back", 2016): each CTA takes the next tile by ticket,
// publishes its tile sum, reads its predecessors' published sums or
// inclusive prefixes 32 at a time until it meets an inclusive one, and
// publishes its own inclusive prefix. One launch (plus one memset of the
// tile status words) for any n. Used for page row offsets, tile offsets of
// the pipeline stages, bucket offsets of the hash build and output row
// offsets.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr size_t kScanTile = size_t(kScanThreads) * kScanPer;
// Polls of a predecessor's status before the scan gives up (error
// kErrTimeout); predecessors hold earlier tickets, so they are running.
constexpr uint32_t kLookbackLimit = 1u << 22;

template <typename T>
__device__ __forceinline__ T warp_inclusive(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) >= o) v += u;
    }
    return v;
}

// Exclusive scan of one value per thread across the block; *total gets the sum.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T* total) {
    __shared__ T warp_sums[32];
    T inc = warp_inclusive(v);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        T w = lane < nw ? warp_sums[lane] : T(0);
        T wi = warp_inclusive(w);
        warp_sums[lane] = wi - w;
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    T res = warp_sums[warp] + inc - v;
    __syncthreads();
    return res;
}

// Tile status word: sum << 2 | flag, flag 1 = the tile's own sum, 2 = the
// inclusive prefix through the tile, 0 = not yet published. Sums must stay
// below 2^62.
__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

// One tile of a single-pass scan (the calling CTA takes its tile by ticket).
template <typename T>
__device__ __forceinline__ void scan_tile_lookback(const T* __restrict__ in, T* __restrict__ out, size_t n,
                                                   unsigned long long* status, uint32_t* ticket, uint32_t* err,
                                                   uint32_t ostride = 1) {
    __shared__ uint32_t s_tile;
    __shared__ T s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = size_t(tile) * kScanTile + size_t(threadIdx.x) * kScanPer;
    T v[kScanPer];
    T local = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = base + k < n ? in[base + k] : T(0);
        local += v[k];
    }
    __shared__ T total;
    const T ex = block_exclusive<T>(local, &total);
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        const T agg = total;
        if (tile == 0) {
            if (lane == 0) {
                __threadfence();
                atomicExch(status, (static_cast<unsigned long long>(agg) << 2) | 2ull);
                s_prefix = 0;
            }
        } else {
            if (lane == 0) {
                __threadfence();
                atomicExch(status + tile, (static_cast<unsigned long long>(agg) << 2) | 1ull);
            }
            T prefix = 0;
            int64_t j = int64_t(tile) - 1 - lane;  // lane 0 reads the nearest predecessor
            uint32_t polls = 0;
            for (;;) {
                unsigned long long st = j >= 0 ? ld_status(status + j) : 2ull;
                while (__any_sync(0xffffffffu, (st & 3) == 0)) {
                    if (++polls > kLookbackLimit) {
                        if (lane == 0) record_error(err, kErrTimeout);
                        st = 2ull;  // give up: treat as an inclusive zero
                        break;
                    }
                    if ((st & 3) == 0) st = ld_status(status + j);
                }
                const uint32_t incl = __ballot_sync(0xffffffffu, (st & 3) == 2);
                const uint32_t stop = incl ? uint32_t(__ffs(incl) - 1) : 32u;
                T val = lane <= stop ? T(st >> 2) : T(0);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
                prefix += val;
                if (incl) break;
                j -= 32;
            }
            if (lane == 0) {
                __threadfence();
                atomicExch(status + tile, (static_cast<unsigned long long>(prefix + agg) << 2) | 2ull);
                s_prefix = prefix;
            }
        }
    }
    __syncthreads();
    T run = s_prefix + ex;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        if (base + k < n) {
            out[(base + k) * ostride] = run;
            run += v[k];
            if (base + k == n - 1) out[n * ostride] = run;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_lookback(const T* __restrict__ in, T* __restrict__ out,
                                                                size_t n, unsigned long long* status,
                                                                uint32_t* ticket, uint32_t* err, uint32_t ostride) {
    scan_tile_lookback<T>(in, out, n, status, ticket, err, ostride);
}

// Independent scans of several u32 arrays (blockIdx.y = array); array k's
// tile status words start at status + status_off[k], its ticket at
// tickets + k. An empty array gets out[0] = 0.
__global__ void __launch_bounds__(kScanThreads) k_scan_segs(ScanSegs segs, unsigned long long* status,
                                                            uint32_t* tickets, uint32_t* err) {
    const ScanSeg& sg = segs.s[blockIdx.y];
    const uint32_t nt = uint32_t((sg.n + kScanTile - 1) / kScanTile);
    if (sg.n == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) sg.out[0] = 0;
        return;
    }
    if (blockIdx.x >= nt) return;
    scan_tile_lookback<uint32_t>(sg.in, sg.out, sg.n, status + segs.status_off[blockIdx.y], tickets + blockIdx.y,
                                 err);
}

// Output i goes to out[i * ostride].
template <typename T>
__global__ void k_tile_scan(const T* __restrict__ in, T* __restrict__ out, size_t n, const T* __restrict__ base_ex,
                            uint32_t ostride = 1) {
    size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanPer;
    T v[kScanPer];
    T local = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = base + k < n ? in[base + k] : T(0);
        local += v[k];
    }
    __shared__ T total;
    T run = block_exclusive<T>(local, &total) + (base_ex ? base_ex[blockIdx.x] : T(0));
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        if (base + k < n) {
            out[(base + k) * ostride] = run;
            run += v[k];
            if (base + k == n - 1) out[n * ostride] = run;
        }
    }
}

// Single-tile scans of several arrays of the same length (blockIdx.x = array).
__global__ void k_tile_scan_batch(ScanBatch64 b, size_t n) {
    const uint64_t* in = b.in[blockIdx.x];
    uint64_t* out = b.out[blockIdx.x];
    const size_t base = size_t(threadIdx.x) * kScanPer;
    uint64_t v[kScanPer];
    uint64_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = base + k < n ? in[base + k] : 0ull;
        local += v[k];
    }
    __shared__ uint64_t total;
    uint64_t run = block_exclusive<uint64_t>(local, &total);
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        if (base + k < n) {
            out[base + k] = run;
            run += v[k];
            if (base + k == n - 1) out[n] = run;
        }
    }
}

template <typename T>
__global__ void k_zero_one(T* p) {
    p[0] = 0;
}

size_t status_bytes(size_t n) {
    const size_t nt = (n + kScanTile - 1) / kScanTile;
    return nt > 1 ? (nt + 1) * sizeof(unsigned long long) : 0;  // tile words + ticket
}

// status: status_bytes(n) zero bytes (null when that is 0).
// Output i goes to out[i * ostride].
template <typename T>
int scan_launch(const T* in, T* out, size_t n, void* status, uint32_t* err, cudaStream_t st, uint32_t ostride = 1) {
    if (n == 0) {
        k_zero_one<T><<<1, 1, 0, st>>>(out);
        return 1;
    }
    const size_t nt = (n + kScanTile - 1) / kScanTile;
    if (nt == 1) {
        k_tile_scan<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, ostride);
        return 1;
    }
    auto* words = static_cast<unsigned long long*>(status);
    k_scan_lookback<T><<<unsigned(nt), kScanThreads, 0, st>>>(in, out, n, words, reinterpret_cast<uint32_t*>(words + nt),
                                                              err, ostride);
    return 1;
}

template <typename T>
int scan_impl(const T* in, T* out, size_t n, Scratch& s, cudaStream_t st) {
    const size_t bytes = status_bytes(n);
    void* status = nullptr;
    if (bytes) {
        status = s.alloc(bytes);
        cudaMemsetAsync(status, 0, bytes, st);
    }
    return scan_launch<T>(in, out, n, status, s.err, st);
}

__global__ void k_gather_values(GatherList g, uint64_t* dst) {
    const int i = threadIdx.x;
    if (i >= g.n) return;
    dst[g.slot[i]] = g.wide[i] ? *static_cast<const uint64_t*>(g.src[i]) : *static_cast<const uint32_t*>(g.src[i]);
}

// Sum of n u32 counts in 64 bits (one CTA): the total a u32 scan of the same
// counts would wrap.
__global__ void __launch_bounds__(1024) k_sum_u32_wide(const uint32_t* __restrict__ in, size_t n,
                                                       unsigned long long* __restrict__ out) {
    unsigned long long s = 0;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ unsigned long long part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < int(blockDim.x >> 5); w++) t += part[w];
        *out = t;
    }
}

__global__ void k_fill_u32(uint32_t* p, uint32_t v, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) p[i] = v;
}

} // namespace

int sum_u32_wide(const uint32_t* in, size_t n, unsigned long long* out, cudaStream_t st) {
    k_sum_u32_wide<<<1, 1024, 0, st>>>(in, n, out);
    return 1;
}

int scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, Scratch& s, cudaStream_t st) {
    return scan_impl<uint32_t>(in, out, n, s, st);
}
int scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, Scratch& s, cudaStream_t st) {
    return scan_impl<uint64_t>(in, out, n, s, st);
}
int scan_exclusive_u64_batch(const ScanBatch64& b, size_t n, Scratch& s, cudaStream_t st) {
    if (b.n <= 0) return 0;
    if (n == 0 || n > kScanTile) {
        int launches = 0;
        for (int i = 0; i < b.n; i++) launches += scan_impl<uint64_t>(b.in[i], b.out[i], n, s, st);
        return launches;
    }
    k_tile_scan_batch<<<unsigned(b.n), kScanThreads, 0, st>>>(b, n);
    return 1;
}

size_t scan_status_bytes(size_t n) { return status_bytes(n); }

int scan_exclusive_u32_segs(ScanSegs segs, Scratch& s, cudaStream_t st) {
    if (segs.n <= 0) return 0;
    size_t words = 0, max_nt = 1;
    for (int k = 0; k < segs.n; k++) {
        const size_t nt = (size_t(segs.s[k].n) + kScanTile - 1) / kScanTile;
        segs.status_off[k] = uint32_t(words);
        words += nt;
        max_nt = std::max(max_nt, nt);
    }
    const size_t bytes = words * sizeof(unsigned long long) + segs.n * sizeof(uint32_t);
    auto* status = static_cast<unsigned long long*>(s.alloc(std::max<size_t>(bytes, 16)));
    auto* tickets = reinterpret_cast<uint32_t*>(status + words);
    cudaMemsetAsync(status, 0, bytes, st);
    k_scan_segs<<<dim3(unsigned(max_nt), unsigned(segs.n)), kScanThreads, 0, st>>>(segs, status, tickets, s.err);
    return 1;
}

int gather_values(const GatherList& g, uint64_t* dst, cudaStream_t st) {
    if (g.n <= 0) return 0;
    k_gather_values<<<1, kMaxGather, 0, st>>>(g, dst);
    return 1;
}
int scan_exclusive_u32_zeroed(const uint32_t* in, uint32_t* out, size_t n, void* status, uint32_t* err,
                              cudaStream_t st, uint32_t out_stride) {
    return scan_launch<uint32_t>(in, out, n, status, err, st, out_stride);
}
int fill_u32(uint32_t* p, uint32_t v, size_t n, cudaStream_t st) {
    if (!n) return 0;
    unsigned blocks = unsigned(std::min<size_t>((n + 255) / 256, 148 * 16));
    k_fill_u32<<<blocks, 256, 0, st>>>(p, v, n);
    return 1;
}

} // namespace bj
