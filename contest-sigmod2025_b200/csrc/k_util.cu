// Device-wide exclusive prefix sums and fills.
// Reduce-then-scan over tiles of 4096 values (1024 threads x 4): one pass of
// per-tile sums, a recursive scan of those sums, and a pass that scans each
// tile and adds its base. Used for page row offsets, tile offsets of the
// pipeline stages, bucket offsets of the hash build and output row offsets.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr size_t kScanTile = size_t(kScanThreads) * kScanPer;

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

template <typename T>
__global__ void k_tile_reduce(const T* __restrict__ in, size_t n, T* __restrict__ partial) {
    size_t base = size_t(blockIdx.x) * kScanTile;
    T s = 0;
    for (int i = threadIdx.x; i < int(kScanTile); i += kScanThreads) {
        size_t j = base + i;
        if (j < n) s += in[j];
    }
    __shared__ T total;
    block_exclusive<T>(s, &total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

template <typename T>
__global__ void k_tile_scan(const T* __restrict__ in, T* __restrict__ out, size_t n, const T* __restrict__ base_ex) {
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

template <typename T>
int scan_impl(const T* in, T* out, size_t n, Scratch& s, cudaStream_t st) {
    if (n == 0) {
        k_zero_one<T><<<1, 1, 0, st>>>(out);
        return 1;
    }
    size_t nt = (n + kScanTile - 1) / kScanTile;
    if (nt == 1) {
        k_tile_scan<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr);
        return 1;
    }
    T* partial = static_cast<T*>(s.alloc(nt * sizeof(T)));
    T* partial_ex = static_cast<T*>(s.alloc((nt + 1) * sizeof(T)));
    k_tile_reduce<T><<<unsigned(nt), kScanThreads, 0, st>>>(in, n, partial);
    int launches = 1 + scan_impl<T>(partial, partial_ex, nt, s, st);
    k_tile_scan<T><<<unsigned(nt), kScanThreads, 0, st>>>(in, out, n, partial_ex);
    return launches + 1;
}

__global__ void k_fill_u32(uint32_t* p, uint32_t v, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) p[i] = v;
}

} // namespace

int scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, Scratch& s, cudaStream_t st) {
    return scan_impl<uint32_t>(in, out, n, s, st);
}
int scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, Scratch& s, cudaStream_t st) {
    return scan_impl<uint64_t>(in, out, n, s, st);
}
int fill_u32(uint32_t* p, uint32_t v, size_t n, cudaStream_t st) {
    if (!n) return 0;
    unsigned blocks = unsigned(std::min<size_t>((n + 255) / 256, 148 * 16));
    k_fill_u32<<<blocks, 256, 0, st>>>(p, v, n);
    return 1;
}

} // namespace bj
