// K1: page index of resident columns, every column of a batch per launch.
//
// Replaces the reference's per-query column preparation
// (TableScan::prepareColumn / makeSearchVector, engine/op/TableScan.cpp:546-582:
// an exclusive prefix of rows per page used by the readers' exponential page
// search) and the popcount-to-dense-index step of its readers
// (TableScan.cpp:113-238, 287-292). Pass 1 reads every page header (one
// thread per page), validates it against the page format and writes the
// page's contained rows and 64-row chunk count; two scans turn those into
// row_start / chunk_base. Pass 2 writes the dense-value base of every chunk
// and the page of every 1024-row block.
#include "launch.h"

#include <algorithm>

namespace bj {
namespace {

__global__ void k_page_headers(PageIndexBatch batch, uint32_t* __restrict__ err) {
    const PageIndexCol& col = batch.c[blockIdx.y];
    const uint8_t* __restrict__ pages = col.pages;
    const uint32_t npages = col.npages;
    const int32_t type = col.type;
    uint32_t* __restrict__ hdr = col.hdr;
    uint32_t* __restrict__ rows = col.rows;
    uint32_t* __restrict__ chunks = col.chunks;
    uint32_t* __restrict__ flags = col.flags;
    if (blockIdx.x * blockDim.x >= npages) return;  // whole CTA beyond this column
    // Page 0's header, read once per CTA (pages may be in host memory).
    __shared__ uint32_t s_h0;
    if (threadIdx.x == 0) s_h0 = *reinterpret_cast<const uint32_t*>(pages);
    __syncthreads();
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npages) return;
    const uint8_t* pg = pages + size_t(p) * kPageSize;
    const uint32_t h = *reinterpret_cast<const uint32_t*>(pg);
    hdr[p] = h;
    uint32_t n = h & 0xffff, nn = h >> 16;
    uint32_t r = n, c = (n + 63) >> 6;
    uint32_t f = 0;
    if (type == kVarchar && n >= 0xfffe) {
        // Long-string page: 1 row for the first page of the run, 0 for the rest.
        r = n == 0xffff ? 1 : 0;
        c = 0;
        f |= 2;
        if (nn > kPageSize - 4) record_error(err, kErrLongString);
        if (n == 0xfffe && (p == 0 || ld16(pages + size_t(p - 1) * kPageSize) < 0xfffe)) record_error(err, kErrLongString);
    } else {
        // Every later read of this page (values by dense index, string offsets)
        // stays inside it once these hold: bitmap and header fit, the bitmap's
        // population equals the non-null count, values / offsets / bytes fit.
        uint32_t nbytes = (n + 7) >> 3;
        bool ok = nn <= n && 4 + nbytes <= kPageSize;
        if (ok && nn != n) {
            f |= 1;
            const uint8_t* bm = pg + kPageSize - nbytes;
            uint32_t pop = 0;
            for (uint32_t b = 0; b < nbytes; b++) {
                uint32_t byte = bm[b];
                if (b == nbytes - 1 && (n & 7)) byte &= (1u << (n & 7)) - 1;
                pop += __popc(byte);
            }
            ok = pop == nn;
        }
        if (ok && type == kVarchar) {
            ok = 4 + 2 * nn + nbytes <= kPageSize;
            uint32_t prev = 0;
            for (uint32_t k = 0; ok && k < nn; k++) {
                uint32_t e = ld16(pg + 4 + 2 * k);
                ok = e >= prev;
                prev = e;
            }
            ok = ok && 4 + 2 * nn + prev + nbytes <= kPageSize;
        } else if (ok) {
            uint32_t w = type == kInt32 ? 4 : 8;
            uint32_t begin = type == kInt32 ? 4 : 8;
            ok = begin + nn * w + nbytes <= kPageSize;
        }
        if (!ok) {
            record_error(err, kErrPageHeader);
            r = 0;
            c = 0;
        }
    }
    // Uniform pages: every page but the last holds as many rows as page 0,
    // the last at most that many.
    const uint32_t h0 = s_h0;
    const uint32_t r0 = (type == kVarchar && (h0 & 0xffff) >= 0xfffe) ? 0u : (h0 & 0xffff);
    if (r0 == 0 || (r != r0 && (p + 1 < npages || r > r0)) || (f & 2)) f |= kColRaggedPages;
    rows[p] = r;
    chunks[p] = c;
    if (f) atomicOr(flags, f);
}

// One warp per page: dense base of each 64-row chunk (a running popcount of
// the page's null bitmap).
__global__ void k_page_dense(PageIndexBatch batch) {
    const PageIndexCol& col = batch.c[blockIdx.y];
    const uint8_t* __restrict__ pages = col.pages;
    const uint32_t* __restrict__ hdr = col.hdr;
    const uint32_t npages = col.npages;
    const uint32_t* __restrict__ chunk_base = col.chunk_base;
    uint32_t* __restrict__ dense_base = col.dense_base;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t lane = threadIdx.x & 31;
    if (warp >= npages) return;
    uint32_t p = warp;
    uint32_t c0 = chunk_base[p], nc = chunk_base[p + 1] - c0;
    if (!nc) return;
    const uint8_t* pg = pages + size_t(p) * kPageSize;
    uint32_t n = hdr[p] & 0xffff, nn = hdr[p] >> 16;
    uint32_t nbytes = (n + 7) >> 3;
    const uint8_t* bm = pg + kPageSize - nbytes;
    uint32_t carry = 0;
    for (uint32_t k0 = 0; k0 < nc; k0 += 32) {
        uint32_t k = k0 + lane;
        uint32_t cnt = 0;
        if (k < nc) {
            if (nn == n) {
                cnt = min(64u, n - k * 64);
            } else {
                uint64_t w = load_bits64(bm, k, nbytes);
                uint32_t valid_bits = min(64u, n - k * 64);
                if (valid_bits < 64) w &= (1ull << valid_bits) - 1;
                cnt = __popcll(w);
            }
        }
        // exclusive warp scan of cnt
        uint32_t inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= uint32_t(o)) inc += u;
        }
        if (k < nc) dense_base[c0 + k] = carry + inc - cnt;
        carry += __shfl_sync(0xffffffffu, inc, 31);
    }
}

// Page containing row b * 1024, for every block b (and the terminal entry).
__global__ void k_page_of_blk(PageIndexBatch batch) {
    const PageIndexCol& col = batch.c[blockIdx.y];
    const uint32_t* __restrict__ row_start = col.row_start;
    const uint32_t npages = col.npages, nrows = col.nrows;
    const uint32_t nblk = (nrows >> kBlkShift) + 2;
    uint32_t* __restrict__ page_of_blk = col.page_of_blk;
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    uint64_t row = uint64_t(b) << kBlkShift;
    uint32_t res;
    if (row >= nrows) {
        res = npages ? npages - 1 : 0;
    } else {
        uint32_t lo = 0, hi = npages - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (row_start[mid] <= row)
                lo = mid;
            else
                hi = mid - 1;
        }
        res = lo;
    }
    page_of_blk[b] = res;
}

} // namespace

int page_index_pass1(const PageIndexBatch& b, uint32_t* err, Scratch& s, cudaStream_t st) {
    if (b.n <= 0) return 0;
    uint32_t max_np = 0;
    ScanSegs segs{};
    for (int k = 0; k < b.n; k++) {
        max_np = std::max(max_np, b.c[k].npages);
        segs.s[segs.n++] = ScanSeg{b.c[k].rows, b.c[k].row_start, b.c[k].npages};
        segs.s[segs.n++] = ScanSeg{b.c[k].chunks, b.c[k].chunk_base, b.c[k].npages};
    }
    int launches = 0;
    if (max_np) {
        k_page_headers<<<dim3((max_np + 255) / 256, unsigned(b.n)), 256, 0, st>>>(b, err);
        launches++;
    }
    return launches + scan_exclusive_u32_segs(segs, s, st);
}

int page_index_pass2(const PageIndexBatch& b, cudaStream_t st) {
    if (b.n <= 0) return 0;
    uint32_t max_np = 0, max_blk = 0;
    for (int k = 0; k < b.n; k++) {
        max_np = std::max(max_np, b.c[k].npages);
        max_blk = std::max(max_blk, (b.c[k].nrows >> kBlkShift) + 2);
    }
    int launches = 0;
    if (max_np) {
        k_page_dense<<<dim3((max_np * 32 + 255) / 256, unsigned(b.n)), 256, 0, st>>>(b);
        launches++;
    }
    k_page_of_blk<<<dim3((max_blk + 255) / 256, unsigned(b.n)), 256, 0, st>>>(b);
    return launches + 1;
}

} // namespace bj
