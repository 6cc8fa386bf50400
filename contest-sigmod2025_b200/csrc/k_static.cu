// Join-count entry point that allocates nothing (bj_join_count_static).
//
// Some callers of this library cannot call cudaMalloc: their device memory is
// owned by another allocator (a framework's caching pool, or a fixed budget
// carved out at start-up), or they issue work from code where cudaMalloc's
// implicit device synchronisation is not acceptable. For them this entry point
// counts the rows of a two-table INT32 equi-join -- the row count bj_execute
// returns for Scan(A) JOIN Scan(B) on those columns -- using only the buffers
// the caller passes and one fixed scratch array compiled into the library.
//
// The scratch is a file-scope __device__ array of kStaticSlots 64-bit slots
// (4 MiB); every GPU that loads the library holds it until the process exits.
// Host code must not take its address directly (the host-side name is a
// stand-in, not a device address): the device address is obtained once per
// device with cudaGetSymbolAddress, with that device current, on the first
// call made on it. Make that first call before any stream capture.
//
// All calls share the array, and it keeps the last call's contents; each call
// clears it before use. Calls that overlap on the GPU (e.g. on two streams at
// once) race on the array and give wrong counts: serialise them.
//
// Bad input is reported through the count: a page whose header cannot be an
// INT32 page, or build pages holding more non-null values than build_rows,
// set a flag word in the scratch, and the last kernel then writes ~0ull
// (UINT64_MAX) to *out_count. The call itself only enqueues work, so its
// return status cannot carry what the kernels find.
//
// The device address is cached per device for the life of the process; after
// cudaDeviceReset the module may load at another address, so the entry point
// must not be used across a device reset.
#include "../../include/b200join.h"
#include "device.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace bj {
namespace {

constexpr uint32_t kStaticLog2 = 19;
constexpr uint32_t kStaticSlots = 1u << kStaticLog2;     // 4 MiB of 64-bit slots (+256 B)
constexpr uint64_t kStaticMaxBuildRows = kStaticSlots / 2; // load factor <= 1/2
constexpr uint64_t kSlotEmpty = ~0ull;

// Slot: key in the high 32 bits, count of build rows with that key in the low
// 32 bits. The all-ones pattern cannot occur as a filled slot because a count
// never reaches 2^32 - 1 (at most kStaticMaxBuildRows), so a key of -1
// (0xFFFFFFFF) is stored like any other. The word after the slots counts
// inserted values, so pages holding more values than the caller said can
// never fill the table past one half; the word after that collects error bits.
constexpr uint32_t kCounterWord = kStaticSlots;
constexpr uint32_t kErrorWord = kStaticSlots + 1;
constexpr unsigned long long kErrBadPage = 1;     // a page header that cannot be an INT32 page
constexpr unsigned long long kErrTooManyRows = 2; // more non-null build values than build_rows
static __device__ __align__(256) unsigned long long g_join_scratch[kStaticSlots + 32];

__global__ void k_static_clear(unsigned long long* slots) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kStaticSlots; i += gridDim.x * blockDim.x)
        slots[i] = kSlotEmpty;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        slots[kCounterWord] = 0;
        slots[kErrorWord] = 0;
    }
}

// Calls fn(key) for every non-null INT32 value of the pages, one CTA per page.
// A join count needs only the multiset of non-null keys, and a page stores its
// non-null values densely in slots 0..nn-1, so the bitmap need not be read.
// A page that cannot be an INT32 page is skipped and flagged in the error word.
template <typename Fn>
__device__ __forceinline__ void for_page_values(const uint8_t* pages, uint64_t npages, unsigned long long* slots,
                                                Fn&& fn) {
    for (uint64_t p = blockIdx.x; p < npages; p += gridDim.x) {
        const uint8_t* pg = pages + p * kPageSize;
        uint32_t n = ld16(pg), nn = ld16(pg + 2);
        uint32_t nbytes = (n + 7) >> 3;
        if (nn > n || 4 + 4 * nn + nbytes > kPageSize) {  // not a valid INT32 page
            if (threadIdx.x == 0) atomicOr(&slots[kErrorWord], kErrBadPage);
            continue;
        }
        for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) fn(*reinterpret_cast<const uint32_t*>(pg + 4 + 4 * i));
    }
}

__global__ void k_static_build(const uint8_t* pages, uint64_t npages, uint64_t build_rows,
                               unsigned long long* slots) {
    for_page_values(pages, npages, slots, [&](uint32_t key) {
        // build_rows <= kStaticMaxBuildRows, so the table stays at most half full.
        if (atomicAdd(&slots[kCounterWord], 1ull) >= build_rows) {
            atomicOr(&slots[kErrorWord], kErrTooManyRows);
            return;
        }
        uint32_t pos = uint32_t(key_hash(key) >> (64 - kStaticLog2));
        for (uint32_t step = 0; step < kStaticSlots; step++) {
            unsigned long long cur = slots[pos];
            if (cur == kSlotEmpty) {
                unsigned long long want = (static_cast<unsigned long long>(key) << 32) | 1ull;
                unsigned long long old = atomicCAS(&slots[pos], kSlotEmpty, want);
                if (old == kSlotEmpty) return;
                cur = old;
            }
            if (uint32_t(cur >> 32) == key) {
                atomicAdd(&slots[pos], 1ull);
                return;
            }
            pos = (pos + 1) & (kStaticSlots - 1);
        }
        // Unreachable: at most kStaticMaxBuildRows values are inserted, so
        // the table is at most half full.
    });
}

__global__ void k_static_probe(const uint8_t* pages, uint64_t npages, unsigned long long* slots,
                               unsigned long long* out_count) {
    unsigned long long mine = 0;
    for_page_values(pages, npages, slots, [&](uint32_t key) {
        uint32_t pos = uint32_t(key_hash(key) >> (64 - kStaticLog2));
        for (uint32_t step = 0; step < kStaticSlots; step++) {
            unsigned long long cur = slots[pos];
            if (cur == kSlotEmpty) return;
            if (uint32_t(cur >> 32) == key) {
                mine += cur & 0xffffffffull;
                return;
            }
            pos = (pos + 1) & (kStaticSlots - 1);
        }
    });
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(out_count, mine);
}

// Last step of every call: a flagged error replaces the count by ~0ull.
__global__ void k_static_finish(const unsigned long long* slots, unsigned long long* out_count) {
    if (slots[kErrorWord] != 0) *out_count = ~0ull;
}

// Device address of g_join_scratch, resolved once per device.
std::mutex g_static_mu;
unsigned long long* g_static_ptr[64] = {};

} // namespace
} // namespace bj

extern "C" BJ_API int bj_join_count_static(const void* build_pages, uint64_t build_num_pages, uint64_t build_rows,
                                           const void* probe_pages, uint64_t probe_num_pages,
                                           unsigned long long* out_count, void* stream) {
    using namespace bj;
    if (!out_count || (build_num_pages && !build_pages) || (probe_num_pages && !probe_pages)) return BJ_ERR_INVALID;
    if (build_rows > kStaticMaxBuildRows) return BJ_ERR_INVALID;  // beyond the fixed scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BJ_ERR_CUDA;
    unsigned long long* slots;
    {
        std::lock_guard<std::mutex> g(g_static_mu);
        if (!g_static_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_join_scratch) != cudaSuccess || !p) return BJ_ERR_CUDA;
            g_static_ptr[dev] = static_cast<unsigned long long*>(p);
        }
        slots = g_static_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(out_count, 0, sizeof(unsigned long long), st) != cudaSuccess) return BJ_ERR_CUDA;
    k_static_clear<<<148, 512, 0, st>>>(slots);
    if (build_num_pages) {
        unsigned grid = unsigned(build_num_pages < 148 * 8 ? build_num_pages : 148 * 8);
        k_static_build<<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(build_pages), build_num_pages, build_rows,
                                              slots);
    }
    if (probe_num_pages) {
        // Probe pages are read (and checked) even when the build side is empty.
        unsigned grid = unsigned(probe_num_pages < 148 * 8 ? probe_num_pages : 148 * 8);
        k_static_probe<<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(probe_pages), probe_num_pages, slots,
                                              out_count);
    }
    k_static_finish<<<1, 1, 0, st>>>(slots, out_count);
    return cudaGetLastError() == cudaSuccess ? BJ_OK : BJ_ERR_CUDA;
}
