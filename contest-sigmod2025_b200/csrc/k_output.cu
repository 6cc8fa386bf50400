// K7: materialisation of result rows into contest pages.
//
// Replaces the reference's output writers (impl::WriterT, engine/op/
// TableTarget.cpp:111-391, and the long-string page copy :243-250). The
// reference fills pages greedily per worker thread; here every page is built
// by one CTA in shared memory and stored with 16-byte writes:
//  * fixed width: a page holds a fixed number of rows (the most that fit when
//    none is NULL: 1984 for INT32, 1007 for INT64/FP64), so page p covers
//    rows [p*R, p*R+R) and all pages are independent. A block scan of the
//    validity flags places the non-null values densely, as the format wants.
//  * VARCHAR: per-row lengths first; then a greedy packer walks blocks of 4096
//    rows (one thread per block, same fill rule as the contest's converter,
//    src/build_table.cpp:640-660) and emits page descriptors; a string longer
//    than PAGE_SIZE-7 gets its own 0xffff/0xfffe page run. Finally one CTA
//    per descriptor gathers the strings from the source pages.
// Any packing that respects the format is a valid result: the harnesses
// compare row multisets (tests/read_sql.cpp:1208-1213).
#include "launch.h"

#include <stdexcept>

namespace bj {
namespace {

constexpr uint32_t kMaxShort = kPageSize - 7;  // longest string stored inline
constexpr uint32_t kLongChunk = kPageSize - 4; // bytes per long-string page

__device__ __forceinline__ uint32_t block_excl_u32(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? ws[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        ws[lane] = wi - w;
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    uint32_t r = ws[warp] + inc - v;
    __syncthreads();
    return r;
}

__device__ __forceinline__ void zero_smem_page(uint8_t* page) {
    uint4* p4 = reinterpret_cast<uint4*>(page);
    for (uint32_t i = threadIdx.x; i < kPageSize / 16; i += blockDim.x) p4[i] = make_uint4(0, 0, 0, 0);
}

__device__ __forceinline__ void store_page(const uint8_t* page, uint8_t* dst) {
    const uint4* s = reinterpret_cast<const uint4*>(page);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (uint32_t i = threadIdx.x; i < kPageSize / 16; i += blockDim.x) d[i] = s[i];
}

// Page pidx of a fixed-width column, by one CTA of 256 threads; each thread
// owns 8 consecutive rows. gather(r0, lo, nr, v8) fills v8[k] with the value
// of output row r0 + lo + k for the rows below nr and returns the mask of
// those that are not NULL.
template <typename Gather>
__device__ __forceinline__ void write_fixed_page(Gather&& gather, uint64_t n, int32_t type, uint32_t rpp, uint32_t pidx,
                                                 uint8_t* page, uint8_t* __restrict__ dst) {
    __shared__ uint32_t total;
    const uint64_t r0 = uint64_t(pidx) * rpp;
    const uint32_t nr = uint32_t(n - r0 < rpp ? n - r0 : rpp);
    zero_smem_page(page);
    const uint32_t t = threadIdx.x;
    const uint32_t lo = t * 8;
    uint64_t v8[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v8[k] = 0;
    const uint32_t bits = lo < nr ? gather(r0, lo, nr, v8) : 0u;
    uint32_t dense = block_excl_u32(__popc(bits), &total);
    uint8_t* data = page + (type == kInt32 ? 4 : 8);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (!((bits >> k) & 1)) continue;
        if (type == kInt32)
            *reinterpret_cast<uint32_t*>(data + 4 * dense) = uint32_t(v8[k]);
        else
            *reinterpret_cast<uint64_t*>(data + 8 * dense) = v8[k];
        dense++;
    }
    const uint32_t nbytes = (nr + 7) / 8;
    if (lo < nr) page[kPageSize - nbytes + t] = uint8_t(bits);
    if (t == 0) {
        *reinterpret_cast<uint16_t*>(page) = uint16_t(nr);
        *reinterpret_cast<uint16_t*>(page + 2) = uint16_t(total);
    }
    __syncthreads();
    store_page(page, dst);
}

// gather of a direct column (every item one output row) in two rounds of
// independent loads: the items' rows (or matched entries) of all 8 rows,
// then their 8 values -- not one row's two dependent loads after another's.
__device__ __forceinline__ uint32_t gather_direct(const OutColumns& cols, const SlotSource& s, uint64_t r0, uint32_t lo,
                                                  uint32_t nr, uint64_t (&v8)[8]) {
    const Items& in = cols.items;
    uint32_t a8[8];
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        a8[k] = 0;
        if (lo + k < nr) {
            const uint32_t i = uint32_t(r0 + lo + k);
            a8[k] = s.kind == 0 ? item_row(in, i) : in.ents[s.probe][i];
            live |= 1u << k;
        }
    }
    uint32_t bits = 0;
    if (s.kind == 0) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (((live >> k) & 1) && column_value(s.col, a8[k], v8[k])) bits |= 1u << k;
        return bits;
    }
    const HTView& ht = cols.ps.ht[s.probe];
    if (s.kind == 2) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            if ((live >> k) & 1) v8[k] = ht_key(ht, a8[k]);
        return live;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (!((live >> k) & 1)) continue;
        const uint32_t e = a8[k];
        v8[k] = ht.pay[size_t(e) * ht.width + s.slot];
        if (!((ht.pnull[e] >> s.slot) & 1)) bits |= 1u << k;
    }
    return bits;
}

// Byte range of a short string (page p, value d) in its source page.
__device__ __forceinline__ void short_string(const DevColumn& c, uint64_t h, const uint8_t*& bytes, uint32_t& len) {
    uint32_t p = str_handle_page(h), d = str_handle_dense(h);
    const uint8_t* pg = c.pages + size_t(p) * kPageSize;
    uint32_t nn = ld16(pg + 2);
    uint32_t end = ld16(pg + 4 + 2 * d);
    uint32_t begin = d ? ld16(pg + 4 + 2 * (d - 1)) : 0;
    bytes = pg + 4 + 2 * nn + begin;
    len = end - begin;
}

__device__ __forceinline__ uint32_t long_string_length(const DevColumn& c, uint32_t p, uint32_t* err) {
    uint32_t len = 0;
    for (uint32_t q = p; q < c.npages; q++) {
        const uint8_t* pg = c.pages + size_t(q) * kPageSize;
        uint32_t n = ld16(pg);
        if (q > p && n != 0xfffe) break;
        if (q == p && n != 0xffff) {
            record_error(err, kErrLongString);
            return 0;
        }
        len += ld16(pg + 2);
    }
    return len;
}

// Byte length (NULL -> 0) and packing cost of every row, all VARCHAR columns
// of the result (blockIdx.y = column). Cost: 8 * (2 + len) + 1 eighth-bytes
// if non-null (offset, bytes, bitmap bit), 1 if NULL; stats[0] = largest
// cost, stats[1] = 1 if some string is longer than PAGE_SIZE-7.
__global__ void k_string_len_cost(StrCols cols, uint64_t n, uint32_t* __restrict__ err) {
    const uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const StrCol& sc = cols.c[blockIdx.y];
    if (i >= n) return;
    uint32_t len = 0;
    bool v;
    uint64_t h = 0;
    if (sc.from_items) {
        v = slot_value(sc.slot, cols.items, uint32_t(i), item_row(cols.items, uint32_t(i)), cols.ps, h);
        sc.valid_out[i] = v;
        if (!sc.resolved) sc.vals_out[i] = v ? h : 0;
    } else {
        v = sc.valid[i];
        if (v) h = sc.handles[i];
    }
    if (v) {
        if (sc.resolved) {  // a row number of src: its string handle
            uint64_t rh = 0;
            if (h >= sc.src.nrows || !col_get(sc.src, uint32_t(h), rh)) {
                record_error(err, kErrRowRange);
                rh = make_str_handle(sc.src.npages, 0);  // out of range: reported below too
            }
            h = rh;
            sc.resolved[i] = h;
        }
        if (str_handle_page(h) >= sc.src.npages) {
            record_error(err, kErrRowRange);
        } else if (str_handle_dense(h) == 0xffff) {
            len = long_string_length(sc.src, str_handle_page(h), err);
        } else {
            const uint8_t* b;
            short_string(sc.src, h, b, len);
        }
    }
    if (sc.resolved && !v) sc.resolved[i] = 0;
    sc.lens[i] = len;
    const uint32_t c = v ? 8 * (2 + min(len, kPageSize)) + 1 : 1;
    sc.cost[i] = c;
    atomicMax(&sc.stats[0], c);
    if (v && len > kMaxShort) sc.stats[1] = 1;
}

// One thread per block of kStrBlock rows: greedy page packing.
__global__ void k_string_pack(const uint32_t* __restrict__ lens, const uint8_t* __restrict__ valid, uint64_t n,
                              int pass, uint32_t* __restrict__ block_pages, const uint32_t* __restrict__ block_off,
                              StrPageDesc* __restrict__ descs) {
    uint64_t blk = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint64_t r0 = blk * kStrBlock;
    if (r0 >= n) return;
    uint64_t r1 = n < r0 + kStrBlock ? n : r0 + kStrBlock;
    uint32_t pages = 0;
    uint32_t out = pass ? block_off[blk] : 0;
    uint32_t rows = 0, nv = 0, bytes = 0;
    uint64_t first = r0;
    auto close = [&](uint64_t next_first) {
        if (rows) {
            if (pass) descs[out + pages] = StrPageDesc{first, rows, 0xffffffffu};
            pages++;
        }
        rows = nv = bytes = 0;
        first = next_first;
    };
    for (uint64_t r = r0; r < r1; r++) {
        bool v = valid[r];
        uint32_t len = v ? lens[r] : 0;
        if (v && len > kMaxShort) {
            close(r);
            uint32_t chunks = (len + kLongChunk - 1) / kLongChunk;
            for (uint32_t c = 0; c < chunks; c++) {
                if (pass) descs[out + pages] = StrPageDesc{r, 1, c};
                pages++;
            }
            first = r + 1;
            continue;
        }
        uint32_t need = v ? 4 + (nv + 1) * 2 + bytes + len + (rows / 8 + 1) : 4 + nv * 2 + bytes + (rows / 8 + 1);
        if (need > kPageSize) close(r);
        if (rows == 0) first = r;
        rows++;
        if (v) {
            nv++;
            bytes += len;
        }
    }
    close(r1);
    if (!pass) block_pages[blk] = pages;
}

// One page of a VARCHAR column described by d, by one CTA.
__device__ __forceinline__ void write_string_page(const uint64_t* __restrict__ handles,
                                                  const uint8_t* __restrict__ valid,
                                                  const uint32_t* __restrict__ lens, const DevColumn& c,
                                                  StrPageDesc d, uint8_t* page, uint8_t* __restrict__ dst,
                                                  uint32_t* __restrict__ err) {
    __shared__ uint32_t tot_valid, tot_bytes, carry_valid, carry_bytes;
    zero_smem_page(page);
    __syncthreads();
    if (d.chunk != 0xffffffffu) {
        // Long-string page: chunk d.chunk of the string of row d.first_row.
        uint64_t h = handles[d.first_row];
        uint32_t len = lens[d.first_row];
        uint32_t off = d.chunk * kLongChunk;
        uint32_t cnt = min(kLongChunk, len - off);
        if (threadIdx.x == 0) {
            *reinterpret_cast<uint16_t*>(page) = d.chunk == 0 ? 0xffff : 0xfffe;
            *reinterpret_cast<uint16_t*>(page + 2) = uint16_t(cnt);
        }
        if (str_handle_dense(h) == 0xffff) {
            // Source is itself a long-string run: copy byte range [off, off+cnt).
            uint32_t p = str_handle_page(h), pos = 0;
            for (uint32_t q = p; q < c.npages && pos < off + cnt; q++) {
                const uint8_t* pg = c.pages + size_t(q) * kPageSize;
                uint32_t n = ld16(pg + 2);
                uint32_t a = max(pos, off), b = min(pos + n, off + cnt);
                for (uint32_t k = a + threadIdx.x; k < b; k += blockDim.x) page[4 + (k - off)] = pg[4 + (k - pos)];
                pos += n;
            }
        } else {
            record_error(err, kErrLongString);
        }
        __syncthreads();
        store_page(page, dst);
        return;
    }
    // Normal page: first pass counts valid rows (offset array size), second places data.
    if (threadIdx.x == 0) carry_valid = carry_bytes = 0;
    __syncthreads();
    uint32_t nv_total = 0;
    for (uint32_t base = 0; base < d.nrows; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < d.nrows ? valid[d.first_row + i] : 0;
        block_excl_u32(v, &tot_valid);
        nv_total += tot_valid;
    }
    uint8_t* chars = page + 4 + 2 * nv_total;
    uint32_t nbytes = (d.nrows + 7) / 8;
    uint8_t* bm = page + kPageSize - nbytes;
    for (uint32_t base = 0; base < d.nrows; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        bool v = i < d.nrows && valid[d.first_row + i];
        uint32_t len = v ? lens[d.first_row + i] : 0;
        uint32_t dv = block_excl_u32(v ? 1u : 0u, &tot_valid);
        uint32_t db = block_excl_u32(len, &tot_bytes);
        dv += carry_valid;
        db += carry_bytes;
        if (v) {
            const uint8_t* src;
            uint32_t slen;
            short_string(c, handles[d.first_row + i], src, slen);
            for (uint32_t k = 0; k < len; k++) chars[db + k] = src[k];
            *reinterpret_cast<uint16_t*>(page + 4 + 2 * dv) = uint16_t(db + len);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry_valid += tot_valid;
            carry_bytes += tot_bytes;
        }
        __syncthreads();
    }
    // Bitmap: one thread per byte.
    for (uint32_t byte = threadIdx.x; byte < nbytes; byte += blockDim.x) {
        uint32_t b = 0;
        for (uint32_t k = 0; k < 8; k++) {
            uint32_t i = byte * 8 + k;
            if (i < d.nrows && valid[d.first_row + i]) b |= 1u << k;
        }
        bm[byte] = uint8_t(b);
    }
    if (threadIdx.x == 0) {
        *reinterpret_cast<uint16_t*>(page) = uint16_t(d.nrows);
        *reinterpret_cast<uint16_t*>(page + 2) = uint16_t(nv_total);
    }
    __syncthreads();
    store_page(page, dst);
}

// Column and page of CTA g (OutColumns' order); false for a round's CTA whose
// column has no page starting in that round. The fixed-width pages of every
// column covering the same rows run together, so the items and gathered
// values they all read are still in L2 for the second and later columns.
// A page p of a column with rows per page q >= base starts in exactly one
// round, r = floor(p q / base), and p = ceil(r base / q) recovers it.
__device__ __forceinline__ bool cta_page(const OutColumns& cols, uint32_t g, int& k, uint32_t& p) {
    const uint32_t fixed_ctas = cols.nfixed * cols.rounds;
    if (g < fixed_ctas) {
        const uint32_t r = g / cols.nfixed;
        k = cols.fixed_col[g % cols.nfixed];
        const OutColumn& oc = cols.c[k];
        if (oc.rpp == cols.base_rpp) {
            p = r;
        } else {
            const uint64_t first = uint64_t(r) * cols.base_rpp;
            const uint64_t up = first + oc.rpp - 1;
            const uint64_t pp = up >> 32 ? up / oc.rpp : uint64_t(uint32_t(up) / oc.rpp);
            if (pp * oc.rpp >= first + cols.base_rpp) return false;
            p = uint32_t(pp);
        }
        return p < oc.npages;
    }
    uint32_t v = g - fixed_ctas;
    for (k = 0; k < cols.n; k++) {
        const OutColumn& oc = cols.c[k];
        if (oc.type != kVarchar) continue;
        if (v < oc.npages) {
            p = v;
            return true;
        }
        v -= oc.npages;
    }
    return false;
}

// Every page of the result, all columns, one CTA per page in cta_page's order.
__global__ void __launch_bounds__(256) k_write_pages(OutColumns cols, uint8_t* __restrict__ out,
                                                     uint32_t* __restrict__ err) {
    __shared__ __align__(16) uint8_t page[kPageSize];
    int k = 0;
    uint32_t p = 0;
    if (!cta_page(cols, blockIdx.x, k, p)) return;
    const OutColumn& oc = cols.c[k];
    uint8_t* dst = out + size_t(oc.page_base + p) * kPageSize;
    if (oc.type != kVarchar) {
        if (oc.direct) {
            // Values straight from the items (every item is one output row).
            write_fixed_page(
                [&](uint64_t r0, uint32_t lo, uint32_t nr, uint64_t(&v8)[8]) {
                    return gather_direct(cols, oc.slot, r0, lo, nr, v8);
                },
                cols.nrows, oc.type, oc.rpp, p, page, dst);
        } else {
            write_fixed_page(
                [&](uint64_t r0, uint32_t lo, uint32_t nr, uint64_t(&v8)[8]) {
                    uint32_t bits = 0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        if (lo + k >= nr) continue;
                        const uint64_t o = r0 + lo + k;
                        if (!oc.valid[o]) continue;
                        v8[k] = oc.vals[o];
                        bits |= 1u << k;
                    }
                    return bits;
                },
                cols.nrows, oc.type, oc.rpp, p, page, dst);
        }
        return;
    }
    StrPageDesc d = oc.descs[p];
    if (oc.floor) {
        d.nrows = uint32_t((p + 1 < oc.npages ? oc.descs[p + 1].first_row : cols.nrows) - d.first_row);
        d.chunk = 0xffffffffu;
    }
    write_string_page(oc.vals, oc.valid, oc.lens, oc.src, d, page, dst, err);
}

// Parallel page assignment for VARCHAR columns ("floor packing"). With S_i
// the exclusive prefix of row costs, row i goes to page floor(S_i / Cp),
// Cp = 65496 - max cost: a page then holds less than 65496 eighth-bytes, i.e.
// 4 + 2 nv + bytes + ceil(rows / 8) <= 8192, and consecutive rows advance by
// at most one page, so no page is empty. Used when no string is long
// (> PAGE_SIZE-7) and the longest is short enough to keep pages ~full. This
// pass records each page's first row (blockIdx.y = column); the page writer
// takes a page's row count from the next page's first row.
__global__ void k_floor_first(FloorCols cols, uint64_t n) {
    const uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const uint64_t* start = cols.start[blockIdx.y];
    const uint64_t cp = cols.cp[blockIdx.y];
    const uint64_t pg = start[i] / cp;
    if (i == 0 || start[i - 1] / cp != pg) cols.descs[blockIdx.y][pg].first_row = i;
}

} // namespace

int string_len_cost(const StrCols& cols, uint64_t n, uint32_t* err, cudaStream_t st) {
    if (!n || cols.n <= 0) return 0;
    k_string_len_cost<<<dim3(unsigned((n + 255) / 256), unsigned(cols.n)), 256, 0, st>>>(cols, n, err);
    return 1;
}

int string_floor_first(const FloorCols& cols, uint64_t n, cudaStream_t st) {
    if (!n || cols.n <= 0) return 0;
    k_floor_first<<<dim3(unsigned((n + 255) / 256), unsigned(cols.n)), 256, 0, st>>>(cols, n);
    return 1;
}

int string_pack(const uint32_t* lens, const uint8_t* valid, uint64_t n, int pass, uint32_t* block_pages,
                const uint32_t* block_page_off, StrPageDesc* descs, cudaStream_t st) {
    uint64_t blocks = (n + kStrBlock - 1) / kStrBlock;
    if (!blocks) return 0;
    k_string_pack<<<unsigned((blocks + 63) / 64), 64, 0, st>>>(lens, valid, n, pass, block_pages, block_page_off,
                                                               descs);
    return 1;
}

int write_pages(const OutColumns& cols_in, uint32_t total_pages, uint8_t* out_pages, uint32_t* err,
                cudaStream_t st) {
    if (!total_pages || cols_in.n <= 0) return 0;
    OutColumns cols = cols_in;
    cols.nfixed = 0;
    cols.base_rpp = 0;
    uint64_t varchar_pages = 0;
    for (int c = 0; c < cols.n; c++) {
        const OutColumn& oc = cols.c[c];
        if (oc.type == kVarchar) {
            varchar_pages += oc.npages;
            continue;
        }
        if (!oc.npages || !oc.rpp) continue;
        cols.fixed_col[cols.nfixed++] = c;
        if (!cols.base_rpp || oc.rpp < cols.base_rpp) cols.base_rpp = oc.rpp;
    }
    cols.rounds = cols.nfixed ? uint32_t((cols.nrows + cols.base_rpp - 1) / cols.base_rpp) : 0u;
    const uint64_t ctas = uint64_t(cols.nfixed) * cols.rounds + varchar_pages;
    if (ctas > 0x7fffffffull) throw std::length_error("result pages beyond one launch");
    k_write_pages<<<unsigned(ctas), 256, 0, st>>>(cols, out_pages, err);
    return 1;
}

} // namespace bj
