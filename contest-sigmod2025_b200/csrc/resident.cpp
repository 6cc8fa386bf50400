// Resident tables: upload of a table's pages into HBM once (page index and
// statistics kept with them), snapshots to and from files, and release.
// Replaces the reference's .cache.db of loaded tables for repeated queries.
#include "engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace bj;

extern "C" {

BJ_API int bj_resident_upload(bj_context* ctx, const bj_table* table, bj_resident** out) {
    if (!ctx || !table || !out) return BJ_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    auto r = std::make_unique<bj_resident>();
    try {
        DevTable& d = r->table;
        d.rows = table->num_rows;
        d.cols.assign(table->num_columns, DevColumn{});
        d.present.assign(table->num_columns, 0);
        if (table->num_rows >= (1ull << 32) - 2) throw Fail{BJ_ERR_UNSUPPORTED, "tables are limited to 2^32-2 rows"};
        std::vector<ColumnJob> jobs;
        if (table->num_rows) {
            if (table->num_columns && !table->columns) throw Fail{BJ_ERR_INVALID, "table without column array"};
            for (uint64_t c = 0; c < table->num_columns; c++) {
                const bj_column& hc = table->columns[c];
                if (hc.type < BJ_INT32 || hc.type > BJ_VARCHAR) throw Fail{BJ_ERR_INVALID, "unknown column type"};
                if (hc.num_pages && !hc.pages) throw Fail{BJ_ERR_INVALID, "column without page array"};
                d.cols[c].type = hc.type;
                d.present[c] = 1;
                uint8_t* dp = static_cast<uint8_t*>(r->mem.alloc(std::max<uint64_t>(hc.num_pages, 1) * kPageSize));
                uint8_t* mapped = nullptr;
                const uint8_t* pinned = pinned_base(hc, mapped);
                jobs.push_back(ColumnJob{&hc, dp, table->num_rows, &d.cols[c], false, pinned});
            }
        } else {
            for (uint64_t c = 0; c < table->num_columns; c++) d.present[c] = 1;
        }
        BJ_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
        upload_pages(ctx, jobs);
        index_columns(ctx, jobs, r->mem);
        BJ_CK(cudaStreamSynchronize(ctx->stream));
        ctx->arena.reset();
    } catch (const Fail& f) {
        return fail_to_status(ctx, f);
    } catch (const std::exception& e) {
        return fail_to_status(ctx, Fail{BJ_ERR_INTERNAL, e.what()});
    }
    *out = r.release();
    return BJ_OK;
}


// Snapshot of a resident table (bj_resident_save / bj_resident_load): the
// role of the reference's table cache file (engine/infra/DataSource.cpp:50-159),
// which reloads tables without re-parsing them. Layout (little-endian):
//   "BJRES001", u64 rows, u64 columns;
//   per column: i32 type, u32 present, u32 pages, u32 rows, u32 flags, u32 rpp,
//               u64 chunks, u64 blocks;
//   then per column: pages (pages * 8192 B), hdr (pages u32), row_start and
//   chunk_base (pages + 1 u32 each), dense_base (chunks u32), page_of_blk
//   (blocks u32).
// Loading copies the arrays straight to HBM: no page index pass.
namespace {
constexpr char kSnapMagic[8] = {'B', 'J', 'R', 'E', 'S', '0', '0', '1'};
struct SnapColumn {
    int32_t type;
    uint32_t present, npages, nrows, flags, rpp;
    uint64_t chunks, blocks;
};
constexpr size_t kSnapChunk = size_t(64) << 20;  // bytes per bounce copy

struct FileCloser {
    void operator()(std::FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<std::FILE, FileCloser>;

// Copies device bytes to the file through a pinned bounce buffer.
void snap_write(std::FILE* f, const void* dev, size_t bytes, uint8_t* bounce) {
    const uint8_t* src = static_cast<const uint8_t*>(dev);
    for (size_t off = 0; off < bytes; off += kSnapChunk) {
        const size_t n = std::min(kSnapChunk, bytes - off);
        BJ_CK(cudaMemcpy(bounce, src + off, n, cudaMemcpyDeviceToHost));
        if (std::fwrite(bounce, 1, n, f) != n) throw Fail{BJ_ERR_INVALID, "snapshot write failed"};
    }
}
// Reads file bytes into device memory through a pinned bounce buffer.
void snap_read(std::FILE* f, void* dev, size_t bytes, uint8_t* bounce) {
    uint8_t* dst = static_cast<uint8_t*>(dev);
    for (size_t off = 0; off < bytes; off += kSnapChunk) {
        const size_t n = std::min(kSnapChunk, bytes - off);
        if (std::fread(bounce, 1, n, f) != n) throw Fail{BJ_ERR_INVALID, "snapshot file is truncated"};
        BJ_CK(cudaMemcpy(dst + off, bounce, n, cudaMemcpyHostToDevice));
    }
}
struct Bounce {
    uint8_t* p = nullptr;
    Bounce() {
        if (cudaHostAlloc(reinterpret_cast<void**>(&p), kSnapChunk, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            throw Fail{BJ_ERR_OOM, "pinned bounce buffer allocation failed"};
        }
    }
    ~Bounce() {
        if (p) cudaFreeHost(p);
    }
};
} // namespace

BJ_API int bj_resident_save(bj_context* ctx, const bj_resident* t, const char* path) {
    if (!ctx || !t || !path) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    try {
        File f(std::fopen(path, "wb"));
        if (!f) throw Fail{BJ_ERR_INVALID, std::string("cannot open ") + path};
        BJ_CK(cudaStreamSynchronize(ctx->stream));
        const DevTable& d = t->table;
        std::vector<SnapColumn> cols(d.cols.size());
        for (size_t c = 0; c < d.cols.size(); c++) {
            const DevColumn& dc = d.cols[c];
            SnapColumn& sc = cols[c];
            sc = SnapColumn{dc.type, d.present[c], dc.npages, dc.nrows, dc.flags & ~kColHostPages, dc.rpp, 0, 0};
            if (dc.npages) {
                uint32_t chunks = 0;
                BJ_CK(cudaMemcpy(&chunks, dc.chunk_base + dc.npages, sizeof(chunks), cudaMemcpyDeviceToHost));
                sc.chunks = chunks;
                sc.blocks = (uint64_t(dc.nrows) >> kBlkShift) + 2;
            }
        }
        const uint64_t head[2] = {d.rows, uint64_t(d.cols.size())};
        bool ok = std::fwrite(kSnapMagic, 1, 8, f.get()) == 8 && std::fwrite(head, sizeof(head), 1, f.get()) == 1 &&
                  (cols.empty() || std::fwrite(cols.data(), sizeof(SnapColumn), cols.size(), f.get()) == cols.size());
        if (!ok) throw Fail{BJ_ERR_INVALID, "snapshot write failed"};
        Bounce b;
        for (size_t c = 0; c < d.cols.size(); c++) {
            const DevColumn& dc = d.cols[c];
            const SnapColumn& sc = cols[c];
            if (!sc.npages) continue;
            snap_write(f.get(), dc.pages, size_t(sc.npages) * kPageSize, b.p);
            snap_write(f.get(), dc.hdr, sizeof(uint32_t) * sc.npages, b.p);
            snap_write(f.get(), dc.row_start, sizeof(uint32_t) * (sc.npages + 1), b.p);
            snap_write(f.get(), dc.chunk_base, sizeof(uint32_t) * (sc.npages + 1), b.p);
            snap_write(f.get(), dc.dense_base, sizeof(uint32_t) * sc.chunks, b.p);
            snap_write(f.get(), dc.page_of_blk, sizeof(uint32_t) * sc.blocks, b.p);
        }
        if (std::fflush(f.get()) != 0) throw Fail{BJ_ERR_INVALID, "snapshot write failed"};
    } catch (const Fail& fl) {
        return fail_to_status(ctx, fl);
    } catch (const std::exception& e) {
        return fail_to_status(ctx, Fail{BJ_ERR_INTERNAL, e.what()});
    }
    ctx->last_error.clear();
    return BJ_OK;
}

BJ_API int bj_resident_load(bj_context* ctx, const char* path, bj_resident** out) {
    if (!ctx || !path || !out) return BJ_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    auto r = std::make_unique<bj_resident>();
    try {
        File f(std::fopen(path, "rb"));
        if (!f) throw Fail{BJ_ERR_INVALID, std::string("cannot open ") + path};
        char magic[8];
        uint64_t head[2];
        if (std::fread(magic, 1, 8, f.get()) != 8 || std::memcmp(magic, kSnapMagic, 8) != 0 ||
            std::fread(head, sizeof(head), 1, f.get()) != 1)
            throw Fail{BJ_ERR_INVALID, "not a resident table snapshot"};
        if (head[0] >= (1ull << 32) - 2 || head[1] > (1u << 20)) throw Fail{BJ_ERR_INVALID, "snapshot header out of range"};
        std::vector<SnapColumn> cols(head[1]);
        if (!cols.empty() && std::fread(cols.data(), sizeof(SnapColumn), cols.size(), f.get()) != cols.size())
            throw Fail{BJ_ERR_INVALID, "snapshot file is truncated"};
        DevTable& d = r->table;
        d.rows = head[0];
        d.cols.assign(cols.size(), DevColumn{});
        d.present.assign(cols.size(), 0);
        Bounce b;
        for (size_t c = 0; c < cols.size(); c++) {
            const SnapColumn& sc = cols[c];
            if (sc.type < BJ_INT32 || sc.type > BJ_VARCHAR || sc.present > 1 ||
                (sc.npages && (sc.nrows != d.rows || sc.chunks > uint64_t(sc.npages) * 1024 ||
                               sc.blocks != (uint64_t(sc.nrows) >> kBlkShift) + 2)))
                throw Fail{BJ_ERR_INVALID, "snapshot column descriptor out of range"};
            DevColumn& dc = d.cols[c];
            d.present[c] = uint8_t(sc.present);
            dc.type = sc.type;
            dc.npages = sc.npages;
            dc.nrows = sc.nrows;
            dc.flags = sc.flags;
            set_rpp(dc, sc.rpp);
            if (!sc.npages) continue;
            auto dev = [&](size_t bytes) { return r->mem.alloc(std::max<size_t>(bytes, 4)); };
            uint8_t* pages = static_cast<uint8_t*>(dev(size_t(sc.npages) * kPageSize));
            auto* hdr = static_cast<uint32_t*>(dev(sizeof(uint32_t) * sc.npages));
            auto* row_start = static_cast<uint32_t*>(dev(sizeof(uint32_t) * (sc.npages + 1)));
            auto* chunk_base = static_cast<uint32_t*>(dev(sizeof(uint32_t) * (sc.npages + 1)));
            auto* dense = static_cast<uint32_t*>(dev(sizeof(uint32_t) * sc.chunks));
            auto* pob = static_cast<uint32_t*>(dev(sizeof(uint32_t) * sc.blocks));
            snap_read(f.get(), pages, size_t(sc.npages) * kPageSize, b.p);
            snap_read(f.get(), hdr, sizeof(uint32_t) * sc.npages, b.p);
            snap_read(f.get(), row_start, sizeof(uint32_t) * (sc.npages + 1), b.p);
            snap_read(f.get(), chunk_base, sizeof(uint32_t) * (sc.npages + 1), b.p);
            snap_read(f.get(), dense, sizeof(uint32_t) * sc.chunks, b.p);
            snap_read(f.get(), pob, sizeof(uint32_t) * sc.blocks, b.p);
            dc.pages = pages;
            dc.hdr = hdr;
            dc.row_start = row_start;
            dc.chunk_base = chunk_base;
            dc.dense_base = dense;
            dc.page_of_blk = pob;
        }
    } catch (const Fail& fl) {
        return fail_to_status(ctx, fl);
    } catch (const std::exception& e) {
        return fail_to_status(ctx, Fail{BJ_ERR_INTERNAL, e.what()});
    }
    ctx->last_error.clear();
    *out = r.release();
    return BJ_OK;
}

BJ_API void bj_resident_free(bj_context* ctx, bj_resident* t) {
    if (!t) return;
    // Graphs that read this table are no longer valid.
    if (ctx) drop_graphs_using(ctx, t);
    delete t;
}

} // extern "C"
