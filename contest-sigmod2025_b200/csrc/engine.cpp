// Host side of the B200 join engine: page upload and indexing, the pipeline
// driver (Executor) and the shared execute path. The context's life cycle and
// the C ABI are in api.cpp, CUDA-graph replay in graphs.cpp, resident tables
// and snapshots in resident.cpp.
//
// Replaces, for the join path:
//  * Contest::build_context / execute / destroy_context (engine/Execute.cpp:
//    11-48): a context owns a CUDA stream, a device arena, pinned staging and
//    a host thread pool for page staging (the reference's scheduler threads,
//    engine/infra/Scheduler.cpp, are replaced by CTAs on the device);
//  * the per-query bump allocator (engine/infra/QueryMemory.cpp:86-139): the
//    device arena is reset after every call;
//  * QueryPlan::runPipeline (engine/query/QueryPlan.cpp:414-678): each
//    pipeline of the ExecPlan (planner.h) runs as probe stages, then either a
//    hash build or the result materialisation.
#include "engine.h"

#include <cuda_runtime.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <future>
#include <atomic>
#include <vector>


using namespace bj;

namespace bj {

// Phase durations from the five phase marks of a call (bj_stats.phase_ms).
void phase_stats(const std::vector<cudaEvent_t>& marks, bj_stats& st) {
    if (marks.size() != kPhaseMarks) return;
    for (size_t i = 0; i + 1 < kPhaseMarks; i++) {
        float ms = 0;
        BJ_CK(cudaEventElapsedTime(&ms, marks[i], marks[i + 1]));
        st.phase_ms[i] = ms;
    }
}


// Reads back `n` u64 slots of ctx->d_small after the stream drains; checks the
// device error word.
// Host-side trace of a call (B200JOIN_TRACE=1): milliseconds since the call
// began and since the previous mark, to stderr. B200JOIN_TRACE=2 drains the
// call's stream at every mark first, so that a mark's delta is the device
// time of the work enqueued since the previous one (and the call runs
// serialised: for locating time, not for timing).
int trace_level() {
    static const int level = [] {
        const char* e = std::getenv("B200JOIN_TRACE");
        return e ? std::atoi(e) : 0;
    }();
    return level;
}
bool trace_on() { return trace_level() != 0; }
thread_local std::chrono::steady_clock::time_point g_trace_t0, g_trace_last;
thread_local cudaStream_t g_trace_stream = nullptr;
void trace_begin(cudaStream_t st) {
    g_trace_stream = st;
    if (trace_on()) g_trace_t0 = g_trace_last = std::chrono::steady_clock::now();
}
void trace(const char* what) {
    if (!trace_on()) return;
    if (trace_level() >= 2 && g_trace_stream) cudaStreamSynchronize(g_trace_stream);
    auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[b200join] %8.3f ms (+%7.3f) %s\n",
                 std::chrono::duration<double, std::milli>(now - g_trace_t0).count(),
                 std::chrono::duration<double, std::milli>(now - g_trace_last).count(), what);
    g_trace_last = now;
}

void readback(bj_context* ctx, int n) {
    (void)n;
    if (ctx->tape_mode == 2) {
        ReadbackTape& t = *ctx->tape;
        if (t.pos >= t.slots.size()) throw Fail{BJ_ERR_INTERNAL, "graph capture diverged from its recording"};
        std::memcpy(ctx->h_small, t.slots[t.pos++].data(), sizeof(uint64_t) * 64);
        return;
    }
    ctx->launches += uint64_t(gather_values(ctx->gather, ctx->d_small, ctx->stream));
    ctx->gather.n = 0;
    BJ_CK(cudaMemcpyAsync(ctx->h_small, ctx->d_small, sizeof(uint64_t) * 64, cudaMemcpyDeviceToHost, ctx->stream));
    trace("read-back issued");
    BJ_CK(cudaStreamSynchronize(ctx->stream));
    trace("read-back done");
    uint32_t code = uint32_t(ctx->h_small[63]);
    if (code) throw Fail{BJ_ERR_INVALID, std::string("device check failed: ") + dev_error_text(code)};
    if (ctx->tape_mode == 1) {
        std::array<uint64_t, 64> snap;
        std::memcpy(snap.data(), ctx->h_small, sizeof(snap));
        ctx->tape->slots.push_back(snap);
    }
}

// Queue a device u32/u64 value for the next read-back, into slot i; the
// queued values are gathered by one kernel when the read-back is issued.
void stash_value(bj_context* ctx, const void* src, int i, bool wide) {
    if (ctx->tape_mode == 2) return;
    GatherList& g = ctx->gather;
    if (g.n >= kMaxGather) throw Fail{BJ_ERR_INTERNAL, "too many read-back values"};
    g.src[g.n] = src;
    g.slot[g.n] = uint8_t(i);
    g.wide[g.n++] = wide ? 1 : 0;
}
void stash_u32(bj_context* ctx, const uint32_t* src, int i) { stash_value(ctx, src, i, false); }
void stash_u64(bj_context* ctx, const uint64_t* src, int i) { stash_value(ctx, src, i, true); }
void stash_err(bj_context* ctx) { stash_value(ctx, ctx->d_err, 63, false); }

// ---------------------------------------------------------------------------
// Page upload and indexing.


// A column's pages when they lie back to back in pinned host memory (the
// first and the last byte pinned, both mapped to one device range when
// mapped): the host address, and in `dev` the device address of the mapping
// or nullptr. Returns nullptr for pageable or scattered pages.
const uint8_t* pinned_base(const bj_column& hc, uint8_t*& dev) {
    dev = nullptr;
    if (!hc.num_pages || !hc.pages || !hc.pages[0]) return nullptr;
    const uint8_t* p0 = static_cast<const uint8_t*>(hc.pages[0]);
    for (uint64_t k = 1; k < hc.num_pages; k++)
        if (hc.pages[k] != p0 + k * kPageSize) return nullptr;
    cudaPointerAttributes a0{}, a1{};
    if (cudaPointerGetAttributes(&a0, p0) != cudaSuccess ||
        cudaPointerGetAttributes(&a1, p0 + hc.num_pages * kPageSize - 1) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || a1.type != cudaMemoryTypeHost) return nullptr;
    uint8_t* d0 = static_cast<uint8_t*>(a0.devicePointer);
    if (d0 && static_cast<uint8_t*>(a1.devicePointer) == d0 + hc.num_pages * kPageSize - 1) dev = d0;
    return p0;
}

// Columns of pinned, mapped pages at least this large are read in place
// (their device address is `dev` of pinned_base, 16-byte aligned for the
// kernels' 16-byte loads). Smaller ones are copied even from pinned memory:
// a copy is cheap, while reading them in place would pay a host-link round
// trip per random access.
constexpr uint64_t kInPlaceMinPages = 2048;  // 16 MiB

bool read_in_place(const bj_column& hc, const uint8_t* dev) {
    return dev && hc.num_pages >= kInPlaceMinPages && reinterpret_cast<uintptr_t>(dev) % 16 == 0;
}

// One 8 KiB page into pinned staging with non-temporal stores: the staging
// lines go to memory without being read first or left dirty in the CPU's
// caches, so the copy moves half the bytes a plain memcpy does and the DMA
// that follows reads them from memory instead of snooping them out of cache.
// `dst` is 16-byte aligned (page-aligned staging); `src` needs no alignment.
inline void copy_page_streaming(uint8_t* dst, const void* src) {
#if !defined(__x86_64__)
    std::memcpy(dst, src, kPageSize);  // other hosts: a plain copy
#else
    const __m128i* s = static_cast<const __m128i*>(src);
    __m128i* d = reinterpret_cast<__m128i*>(dst);
    for (size_t k = 0; k < kPageSize / 16; k += 4) {
        const __m128i a = _mm_loadu_si128(s + k), b = _mm_loadu_si128(s + k + 1);
        const __m128i c = _mm_loadu_si128(s + k + 2), e = _mm_loadu_si128(s + k + 3);
        _mm_stream_si128(d + k, a);
        _mm_stream_si128(d + k + 1, b);
        _mm_stream_si128(d + k + 2, c);
        _mm_stream_si128(d + k + 3, e);
    }
#endif
}

// Orders this thread's streaming stores before the host hands the staging to
// the copy engine.
inline void staging_fence() {
#if defined(__x86_64__)
    _mm_sfence();
#else
    std::atomic_thread_fence(std::memory_order_release);
#endif
}

// Copies host pages into `dst` on the device: pages are gathered into pinned
// staging by the thread pool, chunk by chunk, each chunk's DMA overlapping
// the next chunk's gathering.
uint64_t upload_pages(bj_context* ctx, const std::vector<ColumnJob>& jobs) {
    // Pinned pages lying back to back go to the device in one DMA each,
    // straight from where they are. (DMA out of staging that the host has
    // just written ran at about a tenth of the link rate on a B200 host.)
    uint64_t direct = 0, total = 0;
    for (auto& j : jobs) {
        if (j.in_place) continue;
        if (j.pinned) {
            const size_t b = j.src->num_pages * kPageSize;
            if (b) BJ_CK(cudaMemcpyAsync(j.dpages, j.pinned, b, cudaMemcpyHostToDevice, ctx->stream));
            direct += b;
            continue;
        }
        total += j.src->num_pages;
    }
    if (!total) return direct;
    size_t bytes = total * kPageSize;
    if (ctx->stage.size < bytes) {
        if (ctx->stage.p) {
            BJ_CK(cudaStreamSynchronize(ctx->stream));
            cudaFreeHost(ctx->stage.p);
            ctx->stage = PinnedBlock{};
        }
        size_t sz = bytes + bytes / 4;
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&ctx->stage.p), sz, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ctx->stage = PinnedBlock{};
            throw Fail{BJ_ERR_OOM, "pinned staging allocation failed"};
        }
        ctx->stage.size = sz;
    }
    // Flatten (column, page) pairs.
    struct Src {
        const void* page;
        uint8_t* dst;
        size_t job;
    };
    std::vector<Src> all;
    all.reserve(total);
    for (size_t ji = 0; ji < jobs.size(); ji++) {
        const ColumnJob& j = jobs[ji];
        if (j.in_place || j.pinned) continue;
        for (uint64_t p = 0; p < j.src->num_pages; p++) {
            if (!j.src->pages[p]) throw Fail{BJ_ERR_INVALID, "null page pointer"};
            all.push_back(Src{j.src->pages[p], j.dpages + p * kPageSize, ji});
        }
    }
    const size_t chunk = 2048;  // pages per DMA
    uint8_t* stage = ctx->stage.p;
    for (size_t c0 = 0; c0 < all.size(); c0 += chunk) {
        size_t c1 = std::min(all.size(), c0 + chunk);
        size_t per = 64;
        ctx->pool->parallel_for((c1 - c0 + per - 1) / per, [&](size_t t) {
            for (size_t i = c0 + t * per; i < std::min(c1, c0 + (t + 1) * per); i++)
                copy_page_streaming(stage + i * kPageSize, all[i].page);
            staging_fence();  // this thread's streaming stores are in memory before the DMA is issued
        });
        // Consecutive pages of one column (one device allocation) become one
        // copy; a copy never spans two allocations.
        size_t i = c0;
        while (i < c1) {
            size_t k = i + 1;
            while (k < c1 && all[k].job == all[i].job && all[k].dst == all[k - 1].dst + kPageSize) k++;
            BJ_CK(cudaMemcpyAsync(all[i].dst, stage + i * kPageSize, (k - i) * kPageSize, cudaMemcpyHostToDevice,
                                  ctx->stream));
            i = k;
        }
    }
    return bytes + direct;
}

// Builds the page index of every job's column (pages already on the device).
void index_columns(bj_context* ctx, std::vector<ColumnJob>& jobs, Scratch& mem) {
    Arena& sc = ctx->arena;
    // Batches of up to 15 columns: one launch per pass, one read-back
    // (4 slots per column) between the passes.
    for (size_t i0 = 0; i0 < jobs.size(); i0 += 15) {
        const size_t i1 = std::min(jobs.size(), i0 + 15);
        PageIndexBatch b{};
        uint32_t* flags = static_cast<uint32_t*>(sc.alloc(sizeof(uint32_t) * (i1 - i0)));
        BJ_CK(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * (i1 - i0), ctx->stream));
        for (size_t i = i0; i < i1; i++) {
            const uint32_t np = uint32_t(jobs[i].src ? jobs[i].src->num_pages : 0);
            PageIndexCol& c = b.c[b.n++];
            c.pages = jobs[i].dpages;
            c.npages = np;
            c.type = jobs[i].out->type;
            c.hdr = static_cast<uint32_t*>(mem.alloc(sizeof(uint32_t) * std::max<size_t>(np, 1)));
            c.rows = static_cast<uint32_t*>(sc.alloc(sizeof(uint32_t) * std::max<size_t>(np, 1)));
            c.chunks = static_cast<uint32_t*>(sc.alloc(sizeof(uint32_t) * std::max<size_t>(np, 1)));
            c.row_start = static_cast<uint32_t*>(mem.alloc(sizeof(uint32_t) * (np + 1)));
            c.chunk_base = static_cast<uint32_t*>(mem.alloc(sizeof(uint32_t) * (np + 1)));
            c.flags = flags + (i - i0);
        }
        ctx->launches += page_index_pass1(b, ctx->d_err, sc, ctx->stream);
        trace("page index pass 1 enqueued");
        // Row totals, chunk totals, flags and the rows of page 0.
        for (size_t i = i0; i < i1; i++) {
            const PageIndexCol& c = b.c[i - i0];
            const int s = int(4 * (i - i0));
            stash_u32(ctx, c.row_start + c.npages, s);
            stash_u32(ctx, c.chunk_base + c.npages, s + 1);
            stash_u32(ctx, c.flags, s + 2);
            stash_u32(ctx, c.rows, s + 3);
        }
        stash_err(ctx);
        readback(ctx, 0);
        for (size_t i = i0; i < i1; i++) {
            PageIndexCol& pc = b.c[i - i0];
            const int s = int(4 * (i - i0));
            const uint64_t rows = ctx->h_small[s], chunks = ctx->h_small[s + 1], flg = ctx->h_small[s + 2];
            const uint64_t rows0 = pc.npages ? ctx->h_small[s + 3] : 0;
            if (rows != jobs[i].rows)
                throw Fail{BJ_ERR_INVALID, "a column's pages hold " + std::to_string(rows) + " rows but its table has " +
                                               std::to_string(jobs[i].rows)};
            DevColumn& c = *jobs[i].out;
            c.pages = jobs[i].dpages;
            c.npages = pc.npages;
            c.nrows = uint32_t(rows);
            c.flags = uint32_t(flg) | (jobs[i].in_place ? kColHostPages : 0u);
            set_rpp(c, (c.flags & kColRaggedPages) ? 0u : uint32_t(rows0));
            c.hdr = pc.hdr;
            c.row_start = pc.row_start;
            c.chunk_base = pc.chunk_base;
            pc.nrows = c.nrows;
            pc.dense_base = static_cast<uint32_t*>(mem.alloc(sizeof(uint32_t) * std::max<uint64_t>(chunks, 1)));
            pc.page_of_blk = static_cast<uint32_t*>(mem.alloc(sizeof(uint32_t) * ((c.nrows >> kBlkShift) + 2)));
            c.dense_base = pc.dense_base;
            c.page_of_blk = pc.page_of_blk;
        }
        ctx->launches += page_index_pass2(b, ctx->stream);
    }
}

// Device copies of the columns of `t` that the plan's scans of `table_id` read.
void collect_columns(const ExecPlan& ex, uint32_t table_id, uint64_t ncols, std::vector<uint8_t>& used) {
    used.assign(ncols, 0);
    for (const PlanAttr& a : ex.attrs)
        if (ex.inputs[a.input].table == table_id && a.column < ncols) used[a.column] = 1;
}

// ---------------------------------------------------------------------------
// Pipeline execution.

struct BuiltHT {
    HTView view{};
    bool empty = true;
    uint32_t* dflags = nullptr;  // device: [0] some key repeats, [1] some multiplicity > 1
    bool unique = false;         // host copies, valid once the parent pipeline read them back
    bool unit_mult = false;
};

// Streamed scans (Executor::streamed_scan): windows of 16 MiB, three in flight.
constexpr uint32_t kWindowPages = 2048;
constexpr uint32_t kWindowRing = 3;

// Begins the copies of the first windows of a host-mapped column (pages,
// npages) on the copy stream, after the work enqueued on `after` so far (the
// small inputs' copies keep the host link first), before the executor has
// chosen what to scan; streamed_scan takes them over if it scans this column.
void start_window_prefetch(bj_context* ctx, const uint8_t* pages, uint32_t npages, cudaStream_t after) {
    const uint32_t nwin = (npages + kWindowPages - 1) / kWindowPages;
    const uint32_t n = std::min(kWindowRing, nwin);
    cudaEvent_t* ev = ctx->events(ctx->window_events, 2 * kWindowRing + 2);
    if (!ev || n == 0) return;
    BJ_CK(cudaEventRecord(ev[2 * kWindowRing], after));
    BJ_CK(cudaStreamWaitEvent(ctx->copy, ev[2 * kWindowRing], 0));
    bj_context::WindowPrefetch& pf = ctx->prefetch;
    pf.src = pages;
    pf.enqueued = 0;
    for (uint32_t r = 0; r < n; r++) {
        pf.win[r] = static_cast<uint8_t*>(ctx->arena.alloc(size_t(kWindowPages) * kPageSize));
        const uint32_t np = std::min(kWindowPages, npages - r * kWindowPages);
        BJ_CK(cudaMemcpyAsync(pf.win[r], pages + size_t(r) * kWindowPages * kPageSize, size_t(np) * kPageSize,
                              cudaMemcpyDefault, ctx->copy));
        BJ_CK(cudaEventRecord(ev[r], ctx->copy));
        pf.enqueued++;
    }
}

// Makes `st` wait for every prefetched window copy (used or not) and clears
// the prefetch, so the call's arena outlives the copies into it.
void end_window_prefetch(bj_context* ctx, cudaStream_t st) {
    if (!ctx->prefetch.src) return;
    cudaEvent_t* ev = ctx->events(ctx->window_events, 2 * kWindowRing + 2);
    if (ev) {
        BJ_CK(cudaEventRecord(ev[2 * kWindowRing + 1], ctx->copy));
        BJ_CK(cudaStreamWaitEvent(st, ev[2 * kWindowRing + 1], 0));
    } else {
        BJ_CK(cudaStreamSynchronize(ctx->copy));
    }
    ctx->prefetch = bj_context::WindowPrefetch{};
}

// The probe of the output pipeline the device's sampling will most likely
// rank first (the most selective): the one whose build input's key column is
// the sparsest over its key range (values / (max - min + 1)), read from the
// host pages of INT32 key columns of at most 2^20 rows. -1: no guess.
int guess_first_probe(const ExecPlan& ex, const bj_plan& plan) {
    if (ex.pipelines.empty()) return -1;
    const PipelinePlan& root = ex.pipelines.back();
    int best = -1;
    double best_density = 2.0;
    for (size_t k = 0; k < root.probes.size(); k++) {
        const PipelinePlan& child = ex.pipelines[root.probes[k].child];
        if (child.build_key < 0 || root.probes[k].key_probe >= 0 || child.build_key_probe >= 0) continue;
        const PlanAttr& a = ex.attrs[size_t(child.build_key)];
        const uint32_t table = ex.inputs[a.input].table;
        if (table >= plan.num_inputs || a.column >= plan.inputs[table].num_columns) continue;
        const bj_column& hc = plan.inputs[table].columns[a.column];
        if (hc.type != BJ_INT32 || plan.inputs[table].num_rows > (1u << 20) || !hc.pages) continue;
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        uint64_t values = 0;
        for (uint64_t p = 0; p < hc.num_pages; p++) {
            const uint8_t* pg = static_cast<const uint8_t*>(hc.pages[p]);
            if (!pg) return -1;
            uint16_t nn;
            std::memcpy(&nn, pg + 2, 2);
            if (4 + 4 * uint64_t(nn) > kPageSize) return -1;
            for (uint32_t v = 0; v < nn; v++) {
                int32_t x;
                std::memcpy(&x, pg + 4 + 4 * v, 4);
                lo = std::min<int64_t>(lo, x);
                hi = std::max<int64_t>(hi, x);
            }
            values += nn;
        }
        if (!values) continue;
        const double density = double(values) / double(hi - lo + 1);
        if (density < best_density) {
            best_density = density;
            best = int(k);
        }
    }
    return best;
}

// Shape class of a plan for the autotuner: the rows of its largest and its
// second largest input (powers of two) and its number of inputs -- what
// the plan is, not how it was ordered. Plans of one class share tuned build
// and scan parameters.
uint64_t shape_class(const ExecPlan& ex) {
    uint64_t a = 0, b = 0;
    for (const PlanInput& in : ex.inputs) {
        if (in.rows > a) {
            b = a;
            a = in.rows;
        } else if (in.rows > b) {
            b = in.rows;
        }
    }
    return (uint64_t(bit_width(a)) << 16) | (uint64_t(bit_width(b)) << 8) | std::min<uint64_t>(ex.inputs.size(), 255);
}

// The parameters of a call: the tuner's override, else the class's tuned
// ones, else the defaults.
TuneConfig tune_for(const bj_context* ctx, const ExecPlan& ex) {
    if (ctx->tune_override) return *ctx->tune_override;
    const uint64_t key = shape_class(ex);
    for (const auto& [k, c] : ctx->tuned)
        if (k == key) return c;
    return TuneConfig{};
}

namespace {

class Executor {
    public:
    Executor(bj_context* ctx, const ExecPlan& ex, std::vector<const DevTable*> tables)
        : ctx_(ctx), ex_(ex), tables_(std::move(tables)), st_(ctx->stream), A_(ctx->arena) {}

    // Runs every pipeline; returns false if the result is empty. Pipelines
    // without probes (leaf builds) need no host round trip: they run first,
    // batched (each pass one launch over all of them), or one per side stream;
    // a pipeline that probes waits for its children's events and runs on the
    // main stream.
    bool run(bj_result& res, int flags) {
        const size_t np = ex_.pipelines.size();
        hts_.resize(np);
        restricted_by_.assign(np, -1);
        batched_.assign(np, 0);
        cudaStream_t main = ctx_->stream;
        cudaEvent_t start = ctx_->pipe_event(np);
        if (!start) throw Fail{BJ_ERR_CUDA, "event creation failed"};
        BJ_CK(cudaEventRecord(start, main));
        st_ = main;
        mark_phase();
        int next_side = 0;
        // Leaf builds: batched, each pass one launch over all of them, on the
        // main stream (B200JOIN_LEAF_BATCH=0: one pipeline per side stream).
        // Leaves restricted by another leaf's filter (PipelinePlan::
        // restrict_by; B200JOIN_SIDEWAYS=0: none) form a second batch, after
        // the first has built their providers.
        std::vector<uint8_t> batched(np, 0);
        if (ctx_->leaf_batch) {
            std::vector<size_t> leaves;
            for (size_t p = 0; p + 1 < np; p++)
                if (ex_.pipelines[p].probes.empty() && ex_.pipelines[p].slots.size() <= size_t(kMaxLeafSlots))
                    leaves.push_back(p);
            if (!leaves.empty()) {
                std::vector<int32_t> by(np, -1);
                std::vector<size_t> first, second;
                if (ctx_->sideways) {
                    std::vector<uint8_t> leaf(np, 0);
                    for (size_t p : leaves) leaf[p] = 1;
                    for (size_t p : leaves) {
                        const int32_t l = ex_.pipelines[p].restrict_by;
                        if (l >= 0 && leaf[size_t(l)] && ex_.pipelines[size_t(l)].restrict_by < 0) by[p] = l;
                    }
                }
                for (size_t p : leaves) (by[p] >= 0 ? second : first).push_back(p);
                build_leaf_batch(first, by);
                if (!second.empty()) build_leaf_batch(second, by);
                trace("leaf builds enqueued");
                for (size_t p : leaves) {
                    cudaEvent_t done = ctx_->pipe_event(p);
                    if (!done) throw Fail{BJ_ERR_CUDA, "event creation failed"};
                    BJ_CK(cudaEventRecord(done, main));
                    batched[p] = 1;
                    batched_[p] = 1;
                }
            }
        }
        for (size_t p = 0; p < np; p++) {
            if (batched[p]) continue;
            const PipelinePlan& pp = ex_.pipelines[p];
            bool leaf = pp.probes.empty() && p + 1 < np;
            cudaEvent_t done = ctx_->pipe_event(p);
            if (!done) throw Fail{BJ_ERR_CUDA, "event creation failed"};
            if (leaf) {
                st_ = ctx_->side[next_side++ % bj_context::kSideStreams];
                BJ_CK(cudaStreamWaitEvent(st_, start, 0));
            } else {
                st_ = main;
                for (const auto& pr : pp.probes) BJ_CK(cudaStreamWaitEvent(main, ctx_->pipe_event(pr.child), 0));
            }
            bool ok = p + 1 < np ? run_pipeline(p, nullptr, 0) : run_pipeline(p, &res, flags);
            trace(leaf ? "leaf pipeline enqueued" : "pipeline done");
            BJ_CK(cudaEventRecord(done, st_));
            if (!ok) {
                st_ = main;
                for (size_t q = 0; q <= p; q++) BJ_CK(cudaStreamWaitEvent(main, ctx_->pipe_event(q), 0));
                return false;
            }
        }
        st_ = main;
        return true;
    }
    uint64_t pipelines_run() const { return pipes_; }

    private:
    const DevColumn& col(uint32_t attr) const {
        const PlanAttr& a = ex_.attrs[attr];
        const DevTable* t = tables_[ex_.inputs[a.input].table];
        return t->cols[a.column];
    }
    template <typename T>
    T* alloc(size_t n) {
        return static_cast<T*>(A_.alloc(sizeof(T) * std::max<size_t>(n, 1)));
    }
    void launched(int n) { ctx_->launches += uint64_t(n); }
    void record_timed() {
        cudaEvent_t e;
        BJ_CK(cudaEventCreate(&e));
        ctx_->prof_events.push_back(e);
        // Inside a graph capture the record must become a graph node.
        BJ_CK(cudaEventRecordWithFlags(e, st_, ctx_->graph_output ? cudaEventRecordExternal : cudaEventRecordDefault));
    }
    void begin_timed() { record_timed(); }
    // Phase marks on the main stream (profiling only): the call's start, the
    // root pipeline's start, its probe order fixed, its stages done, its
    // output written.
    void mark_phase() {
        if (!ctx_->profile) return;
        cudaEvent_t e;
        BJ_CK(cudaEventCreate(&e));
        ctx_->phase_events.push_back(e);
        BJ_CK(cudaEventRecordWithFlags(e, st_, ctx_->graph_output ? cudaEventRecordExternal : cudaEventRecordDefault));
    }
    void end_timed(uint64_t bytes) {
        record_timed();
        ctx_->prof_bytes += bytes;
    }

    // A fused chain of the unique-key stages s, s + 1, ... (up to kMaxChain)
    // over `in`: the stages, the outputs (room for in.count items) and the
    // items it leaves, whose count is on the device.
    struct ChainRun {
        ProbeChain ch{};
        ItemsOut out{};
        uint32_t* cursor = nullptr;
        uint32_t cap = 0;
        size_t s2 = 0;  // first stage after the chain
        Items result{};
    };
    ChainRun plan_chain(const PipelinePlan& pp, const std::vector<uint32_t>& order,
                        const std::vector<HTView>& by_stage, const std::vector<double>& rate, size_t s,
                        const Items& in) {
        ChainRun r;
        bool unit = in.mult == nullptr;
        size_t s2 = s;
        while (s2 < order.size() && r.ch.n < kMaxChain && hts_[pp.probes[order[s2]].child].unique) {
            const uint32_t k2 = order[s2];
            const PipelinePlan::Probe& pr = pp.probes[k2];
            KeySource src{-1, 0, HTView{}};
            if (pr.key_probe >= 0) {
                // Keyed on an earlier stage's payload: that stage's entries
                // must come from an earlier launch, so a source inside this
                // chain ends the chain here.
                const size_t pos = size_t(std::find(order.begin(), order.end(), uint32_t(pr.key_probe)) - order.begin());
                if (pos >= s) break;
                src = KeySource{int32_t(pos), pr.key_slot, by_stage[pos]};
            }
            ChainStage& c = r.ch.st[r.ch.n++];
            c.key = col(pr.probe_attr);
            c.src = src;
            c.ht = by_stage[s2];
            c.use_bloom = (c.ht.bloom && rate[k2] < 0.5) ? 1 : 0;
            unit = unit && hts_[pp.probes[k2].child].unit_mult;
            s2++;
        }
        r.s2 = s2;
        r.cap = in.count;
        r.out.rows = alloc<uint32_t>(r.cap);
        for (size_t j = 0; j < s2; j++) r.out.ents[j] = alloc<uint32_t>(r.cap);
        r.out.mult = unit ? nullptr : alloc<uint64_t>(r.cap);
        r.cursor = alloc<uint32_t>(1);
        BJ_CK(cudaMemsetAsync(r.cursor, 0, sizeof(uint32_t), st_));
        r.result.rows = r.out.rows;
        for (size_t j = 0; j < s2; j++) r.result.ents[j] = r.out.ents[j];
        r.result.mult = r.out.mult;
        r.result.count = r.cap;
        r.result.dcount = r.cursor;
        r.result.nprobes = int(s2);
        return r;
    }

    // Scan-side probe (append mode) of a column whose pages are in pinned
    // host memory: the pages cross the host link by DMA, a window of
    // kWindowPages at a time, into a ring of kRing windows in HBM, and each
    // window is scanned once its copy has landed while the next ones are in
    // flight. The copy engine moves pages at the link's rate (53.6 GB/s on
    // a B200 host against 46.5 GB/s for the kernel's own 16-byte loads of
    // mapped memory), and the scan of a window in HBM takes a few percent of
    // its copy, so the stage runs at about the link's rate.
    //
    // With `chain`, the chain runs after each window's scan over the items
    // that window appended (from the count the previous chain launch saw to
    // the cursor), on the main stream while the next copies are in flight.
    void streamed_scan(const DevColumn& key, const HTView& ht, bool bloom, uint32_t* cursor, const ItemsOut& out,
                       uint32_t cap, ChainRun* chain, const Items& scanned) {
        constexpr uint32_t kRing = kWindowRing;
        const uint32_t nwin = (key.npages + kWindowPages - 1) / kWindowPages;
        const uint32_t ring = std::min(kRing, nwin);
        // Windows whose copies the call began before this column was chosen.
        const bool pre = ctx_->prefetch.src == key.pages && ctx_->prefetch.enqueued > 0;
        uint8_t* win[kRing] = {};
        for (uint32_t r = 0; r < ring; r++)
            win[r] = pre ? ctx_->prefetch.win[r] : alloc<uint8_t>(size_t(kWindowPages) * kPageSize);
        // [0, kRing): window copied; [kRing, 2 kRing): window scanned; then: start, prefetch done.
        cudaEvent_t* ev = ctx_->events(ctx_->window_events, 2 * kRing + 2);
        if (!ev) throw Fail{BJ_ERR_CUDA, "event creation failed"};
        cudaStream_t cp = ctx_->copy;
        uint32_t* marks = nullptr;  // marks[i]: items appended before window i
        if (chain) {
            marks = alloc<uint32_t>(nwin + 1);
            BJ_CK(cudaMemsetAsync(marks, 0, sizeof(uint32_t), st_));
        }
        BJ_CK(cudaEventRecord(ev[2 * kRing], st_));
        BJ_CK(cudaStreamWaitEvent(cp, ev[2 * kRing], 0));
        for (uint32_t i = 0; i < nwin; i++) {
            const uint32_t p0 = i * kWindowPages, np = std::min(kWindowPages, key.npages - p0), r = i % kRing;
            if (!(pre && i < ctx_->prefetch.enqueued)) {
                if (i >= kRing) BJ_CK(cudaStreamWaitEvent(cp, ev[kRing + r], 0));
                // key.pages is the mapped (unified) address of the pinned pages.
                BJ_CK(cudaMemcpyAsync(win[r], key.pages + size_t(p0) * kPageSize, size_t(np) * kPageSize,
                                      cudaMemcpyDefault, cp));
                BJ_CK(cudaEventRecord(ev[r], cp));
            }
            BJ_CK(cudaStreamWaitEvent(st_, ev[r], 0));
            DevColumn w = key;
            w.pages = win[r];
            w.npages = np;
            w.flags &= ~kColHostPages;
            if (w.hdr) w.hdr += p0;
            if (w.row_start) w.row_start += p0;
            if (w.chunk_base) w.chunk_base += p0;
            launched(scan_probe(w, ht, 2, bloom, nullptr, nullptr, cursor, out.rows, out.ents[0], out.mult, cap,
                                ctx_->d_err, ctx_->num_sms, st_, key.rpp ? p0 * key.rpp : 0));
            BJ_CK(cudaEventRecord(ev[kRing + r], st_));
            if (chain)
                launched(probe_chain_unique(scanned, chain->ch, chain->out, chain->cursor, chain->cap, ctx_->d_err,
                                            ctx_->num_sms, st_, marks + i, marks + i + 1));
        }
    }

    // Exclusive scan of tile counts; returns the total (synchronises).
    uint32_t scan_total_u32(const uint32_t* in, uint32_t* out, size_t n) {
        launched(scan_exclusive_u32(in, out, n, A_, st_));
        stash_u32(ctx_, out + n, 0);
        stash_err(ctx_);
        readback(ctx_, 1);
        return uint32_t(ctx_->h_small[0]);
    }
    // The same for counts of items (rows of an intermediate result), which are
    // 32-bit: the counts are also summed in 64 bits, and a join step whose
    // result would not fit fails with kItemOverflow instead of wrapping.
    uint32_t item_total(const uint32_t* in, uint32_t* out, size_t n) {
        launched(scan_exclusive_u32(in, out, n, A_, st_));
        auto* wide = reinterpret_cast<unsigned long long*>(alloc<uint64_t>(1));
        launched(sum_u32_wide(in, n, wide, st_));
        stash_u32(ctx_, out + n, 0);
        stash_u64(ctx_, reinterpret_cast<const uint64_t*>(wide), 1);
        stash_err(ctx_);
        readback(ctx_, 2);
        if (ctx_->h_small[1] > 0xfffffffeull) {
            ctx_->item_overflow = true;
            throw Fail{BJ_ERR_UNSUPPORTED, "a join step yields " + std::to_string(ctx_->h_small[1]) +
                                               " intermediate rows, more than 2^32 - 2"};
        }
        return uint32_t(ctx_->h_small[0]);
    }
    uint64_t scan_total_u64(const uint64_t* in, uint64_t* out, size_t n) {
        launched(scan_exclusive_u64(in, out, n, A_, st_));
        stash_u64(ctx_, out + n, 0);
        stash_err(ctx_);
        readback(ctx_, 1);
        return ctx_->h_small[0];
    }

    // Replaces a device-side item count by the exact count (one read-back).
    void resolve(Items& items) {
        if (!items.dcount) return;
        stash_u32(ctx_, items.dcount, 0);
        stash_err(ctx_);
        readback(ctx_, 1);
        items.count = uint32_t(ctx_->h_small[0]);
        items.dcount = nullptr;
    }

    bool run_pipeline(size_t pi, bj_result* res, int flags) {
        pipes_++;
        const PipelinePlan& pp = ex_.pipelines[pi];
        const PlanInput& in = ex_.inputs[pp.input];
        Items items{};
        items.count = uint32_t(in.rows);
        items.nprobes = 0;
        const bool root = res != nullptr;
        if (root) mark_phase();

        // Probe order: ascending sampled hit rate (most selective first).
        size_t np = pp.probes.size();
        std::vector<uint32_t> order(np);
        std::iota(order.begin(), order.end(), 0u);
        std::vector<double> rate(np, 1.0);
        if (np) {
            // Sample rows read from pinned host memory cross the host link one
            // by one, beside the scan windows' copies: fewer of them there.
            bool host_keys = false;
            for (size_t k = 0; k < np; k++) host_keys = host_keys || (col(pp.probes[k].probe_attr).flags & kColHostPages);
            uint32_t nsample = uint32_t(std::min<uint64_t>(in.rows, host_keys ? 1024 : 4096));
            uint32_t* hits = alloc<uint32_t>(np);
            SampleSet set{};
            set.n = int(np);
            for (size_t k = 0; k < np; k++) {
                set.p[k].key = col(pp.probes[k].probe_attr);
                set.p[k].ht = hts_[pp.probes[k].child].view;
            }
            // The hit counts (and the tables' flags) only steer host decisions;
            // while a graph is captured those come from the recorded tape, so
            // the kernels producing them are left out of the graph.
            if (ctx_->tape_mode != 2) launched(sample_probes(set, nsample, hits, st_));
            for (size_t k = 0; k < np; k++) {
                BuiltHT& child = hts_[pp.probes[k].child];
                stash_u32(ctx_, hits + k, int(k));
                stash_u32(ctx_, child.dflags, int(16 + 2 * k));
                stash_u32(ctx_, child.dflags + 1, int(17 + 2 * k));
            }
            stash_err(ctx_);
            readback(ctx_, int(np));
            for (size_t k = 0; k < np; k++) {
                rate[k] = nsample ? double(ctx_->h_small[k]) / nsample : 1.0;
                BuiltHT& child = hts_[pp.probes[k].child];
                child.unique = ctx_->h_small[16 + 2 * k] == 0;
                child.unit_mult = ctx_->h_small[17 + 2 * k] == 0;
            }
            // A table whose build was restricted by another probed here holds
            // only keys that one's filter passes, so it can only look more
            // selective; when it has no filter of its own (a large build) and
            // the other has one, the other goes first, and the restricted
            // table right after it at the latest.
            std::vector<double> sort_rate = rate;
            std::vector<uint8_t> after(np, 0);
            for (size_t k = 0; k < np; k++)
                for (size_t j = 0; j < np; j++)
                    if (j != k && restricted_by_[pp.probes[k].child] == int32_t(pp.probes[j].child) &&
                        !hts_[pp.probes[k].child].view.bloom) {
                        sort_rate[k] = std::max(sort_rate[k], rate[j]);
                        after[k] = 1;
                    }
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
                return sort_rate[a] != sort_rate[b] ? sort_rate[a] < sort_rate[b] : after[a] < after[b];
            });
            // A probe keyed on an earlier probe's payload runs after it (the
            // first stage is then always keyed on the scanned input).
            std::vector<uint32_t> placed;
            std::vector<uint8_t> done(np, 0);
            while (placed.size() < np) {
                size_t before = placed.size();
                for (uint32_t k : order)
                    if (!done[k] && (pp.probes[k].key_probe < 0 || done[size_t(pp.probes[k].key_probe)])) {
                        placed.push_back(k);
                        done[k] = 1;
                        break;
                    }
                if (placed.size() == before) throw Fail{BJ_ERR_INTERNAL, "probe keys depend on each other"};
            }
            order = placed;
        }
        if (root) mark_phase();
        std::vector<uint32_t> stage_of(np);
        std::vector<HTView> by_stage(np);
        for (size_t s = 0; s < np; s++) {
            stage_of[order[s]] = uint32_t(s);
            by_stage[s] = hts_[pp.probes[order[s]].child].view;
        }
        for (size_t s = 0; s < np; s++) {
            uint32_t k = order[s];
            const HTView& ht = by_stage[s];
            if (items.rows == nullptr && col(pp.probes[k].probe_attr).type == kInt32) {
                // Scan stage: stream the key pages of the scanned table. (An
                // INT64 key column takes the item stages below, over the
                // implicit items 0..rows-1.)
                const BuiltHT& bh = hts_[pp.probes[k].child];
                const DevColumn& key = col(pp.probes[k].probe_attr);
                bool bloom = ht.bloom && rate[k] < 0.5;
                uint64_t page_bytes = uint64_t(key.npages) * kPageSize;
                ItemsOut out{};
                uint32_t total = 0;
                if (bh.unique) {
                    uint32_t cap = key.nrows;
                    out.rows = alloc<uint32_t>(cap);
                    out.ents[0] = alloc<uint32_t>(cap);
                    out.mult = bh.unit_mult ? nullptr : alloc<uint64_t>(cap);
                    uint32_t* cursor = alloc<uint32_t>(2);  // item cursor, candidate count (split scan)
                    BJ_CK(cudaMemsetAsync(cursor, 0, 2 * sizeof(uint32_t), st_));
                    // The next stage reads the count on the device.
                    Items next{};
                    next.rows = out.rows;
                    next.ents[0] = out.ents[0];
                    next.mult = out.mult;
                    next.count = cap;
                    next.dcount = cursor;
                    next.nprobes = 1;
                    bool timed = ctx_->profile;
                    if (timed) begin_timed();
                    if ((key.flags & kColHostPages) && ctx_->stream_scans && ctx_->tape_mode == 0) {
                        // Pages in host memory stream through HBM windows; the
                        // unique-key stages right after the scan run window by
                        // window too, so their reads of host columns overlap
                        // the next windows' copies.
                        const bool fuse = s + 1 < np && hts_[pp.probes[order[s + 1]].child].unique;
                        ChainRun chain;
                        if (fuse) chain = plan_chain(pp, order, by_stage, rate, s + 1, next);
                        streamed_scan(key, ht, bloom, cursor, out, cap, fuse ? &chain : nullptr, next);
                        if (timed) end_timed(page_bytes);
                        trace("streamed scan enqueued");
                        if (fuse) {
                            items = chain.result;
                            s = chain.s2 - 1;
                        } else {
                            items = next;
                        }
                        continue;
                    }
                    if (ctx_->scan_split && ctx_->tune.scan_split) {
                        // Scan + filter (the bloom, or NOT NULL alone), then a
                        // probe of the survivors (two kernels; the scan carries
                        // no probe code). The candidate count is the cursor's
                        // neighbour, zeroed with it.
                        uint32_t* cand = alloc<uint32_t>(2 * size_t(cap));
                        launched(scan_probe_split(key, ht, cursor, out.rows, out.ents[0], out.mult, cap, cand,
                                                  cand + cap, cursor + 1, cap, ctx_->d_err, ctx_->num_sms, st_));
                    } else {
                        launched(scan_probe(key, ht, 2, bloom, nullptr, nullptr, cursor, out.rows, out.ents[0],
                                            out.mult, cap, ctx_->d_err, ctx_->num_sms, st_));
                    }
                    if (timed) end_timed(page_bytes);
                    trace("scan-side probe enqueued");
                    items = next;
                    continue;
                } else {
                    // Counts per work unit of the scan (a few per page).
                    const uint32_t units = scan_probe_units(key.npages);
                    uint32_t* pc = alloc<uint32_t>(units);
                    uint32_t* poff = alloc<uint32_t>(size_t(units) + 1);
                    bool timed = ctx_->profile;
                    if (timed) begin_timed();
                    launched(scan_probe(key, ht, 0, bloom, pc, nullptr, nullptr, nullptr, nullptr, nullptr, 0,
                                        ctx_->d_err, ctx_->num_sms, st_));
                    if (timed) end_timed(page_bytes);
                    total = item_total(pc, poff, units);
                    if (total) {
                        out.rows = alloc<uint32_t>(total);
                        out.ents[0] = alloc<uint32_t>(total);
                        out.mult = bh.unit_mult ? nullptr : alloc<uint64_t>(total);
                        if (timed) begin_timed();
                        launched(scan_probe(key, ht, 1, bloom, nullptr, poff, nullptr, out.rows, out.ents[0],
                                            out.mult, total, ctx_->d_err, ctx_->num_sms, st_));
                        if (timed) end_timed(page_bytes);
                    }
                }
                if (total == 0) return false;
                Items next{};
                next.rows = out.rows;
                next.ents[0] = out.ents[0];
                next.mult = out.mult;
                next.count = total;
                next.nprobes = 1;
                items = next;
                continue;
            }
            const BuiltHT& bh = hts_[pp.probes[k].child];
            bool bloom = ht.bloom && rate[k] < 0.5;
            const DevColumn& key = col(pp.probes[k].probe_attr);
            KeySource ksrc{-1, 0, HTView{}};
            if (pp.probes[k].key_probe >= 0) {
                const uint32_t src_stage = stage_of[size_t(pp.probes[k].key_probe)];
                ksrc = KeySource{int32_t(src_stage), pp.probes[k].key_slot, by_stage[src_stage]};
            }
            if (bh.unique) {
                // This stage and the unique-key stages right after it run as
                // one fused chain.
                ChainRun chain = plan_chain(pp, order, by_stage, rate, s, items);
                launched(probe_chain_unique(items, chain.ch, chain.out, chain.cursor, chain.cap, ctx_->d_err,
                                            ctx_->num_sms, st_));
                trace("probe chain enqueued");
                items = chain.result;
                s = chain.s2 - 1;
                continue;
            }
            resolve(items);
            if (items.count == 0) return false;
            uint32_t tiles = (items.count + kTile - 1) / kTile;
            uint32_t* tc = alloc<uint32_t>(tiles);
            uint32_t* toff = alloc<uint32_t>(tiles + 1);
            ItemsOut none{};
            launched(probe_stage(items, key, ht, 0, tc, nullptr, none, bloom, ctx_->d_err, st_, 0xffffffffu, ksrc));
            uint32_t total = item_total(tc, toff, tiles);
            if (total == 0) return false;
            ItemsOut out{};
            out.rows = alloc<uint32_t>(total);
            for (size_t j = 0; j <= s; j++) out.ents[j] = alloc<uint32_t>(total);
            out.mult = alloc<uint64_t>(total);
            launched(probe_stage(items, key, ht, 1, nullptr, toff, out, bloom, ctx_->d_err, st_, total, ksrc));
            Items next{};
            next.rows = out.rows;
            for (size_t j = 0; j <= s; j++) next.ents[j] = out.ents[j];
            next.mult = out.mult;
            next.count = total;
            next.nprobes = int(s + 1);
            items = next;
        }
        resolve(items);
        if (items.count == 0) return false;

        SlotSources src{};
        src.n = int(pp.slots.size());
        for (size_t j = 0; j < pp.slots.size(); j++) {
            const SlotPlan& sp = pp.slots[j];
            SlotSource& s = src.s[j];
            s.kind = sp.kind;
            if (sp.kind == 0) {
                s.col = col(sp.attr);
                // A probe key column of this input: every item matched an
                // entry with that key, so the value is the entry's key (one
                // load, never NULL) instead of a lookup in the column's pages.
                for (size_t k = 0; k < np; k++)
                    if (pp.probes[k].probe_attr == sp.attr) {
                        s.kind = 2;
                        s.probe = int(stage_of[k]);
                        break;
                    }
            } else {
                s.probe = int(stage_of[sp.probe]);
                s.slot = int(sp.slot);
            }
        }
        if (pp.build_key >= 0)
            return build(pi, items, src, by_stage,
                         pp.build_key_probe >= 0 ? int32_t(stage_of[size_t(pp.build_key_probe)]) : -1);
        mark_phase();
        output(items, src, by_stage, *res, flags);
        mark_phase();
        return true;
    }

    // A build's buffers and sizes; the buffers that must start at zero lie
    // in one region of zbytes bytes, placed by place_zero.
    struct PreparedBuild {
        BuildArgs ba{};
        HTView ht{};
        uint2* buckets = nullptr;
        uint32_t nb = 0;
        bool with_bloom = false;
        uint32_t wlog2 = 0;
        size_t zb_table = 0, zb_counts = 0, zb_cursor = 0, zb_bloom = 0, zb_flags = 256, zb_scan = 0;
        size_t zbytes = 0;
        uint32_t* cursor = nullptr;
        uint32_t* bloom = nullptr;
        uint32_t* dflags = nullptr;
        void* scan_status = nullptr;
    };
    static size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

    PreparedBuild prepare_build(size_t pi, const Items& items, const SlotSources& src,
                                const std::vector<HTView>& probes, int32_t key_stage = -1) {
        const PipelinePlan& pp = ex_.pipelines[pi];
        PreparedBuild pb;
        const uint32_t n = items.count;
        const uint32_t width = uint32_t(src.n);
        BuildArgs& ba = pb.ba;
        ba.in = items;
        ba.key = col(uint32_t(pp.build_key));
        // Keyed on an attribute of a probed input (key_stage >= 0: the stage
        // of that probe in this pipeline), carried as its payload.
        ba.key_stage = key_stage;
        ba.key_slot = key_stage >= 0 ? pp.build_key_slot : 0;
        ba.src = src;
        ba.ps = make_probe_set(probes.data(), items.nprobes);
        TupleBuf& tb = ba.tb;
        // INT64 keys (no reference counterpart) keep their high halves beside
        // the low ones and build no bloom filter.
        const bool wide = ba.key.type == kInt64;
        tb.keys = alloc<uint32_t>(n);
        tb.keys_hi = wide ? alloc<uint32_t>(n) : nullptr;
        tb.mult = alloc<uint64_t>(n);
        tb.pay = alloc<uint64_t>(size_t(n) * std::max<uint32_t>(width, 1));
        tb.pnull = alloc<uint32_t>(n);
        tb.count = n;
        tb.width = width;
        ba.is_rep = alloc<uint32_t>(n);
        ba.err = ctx_->d_err;
        // Sizes. Aggregation table: at least 2n slots. Buckets:
        // 2^max(bit_width(n), 4) (engine/op/Hashtable.cpp:94-104), sized by the
        // tuple count n, an upper bound of the distinct tuples, so the build
        // needs no host round trip. Bloom filter: about 16 bits per key, at
        // most 128 KiB (shared-memory staging); none when that leaves fewer
        // than 8 bits per key (over 131,072 tuples), where it would pass
        // most keys and its build would be contended atomics for nothing.
        // A leaf (items are the input's rows 0..n-1, multiplicity 1) is built
        // without eager aggregation: its tuples can only repeat where whole
        // rows repeat (or, without payload, where keys repeat), and such
        // copies may stay separate entries of multiplicity 1 (the same result
        // rows; the table's flags then report repeated keys and probes take
        // the path for them). Folding pays off in builds fed by probes, where
        // one row comes back once per match.
        ba.distinct = items.rows == nullptr && items.mult == nullptr && items.nprobes == 0 ? 1u : 0u;
        ba.tlog2 = ba.distinct ? 1u : std::max<uint32_t>(1, bit_width(uint64_t(n) * 2));
        const uint32_t nrep = n;
        // Autotuned: bucket count (fill factor) and bloom bits per key.
        const TuneConfig& tc = ctx_->tune;
        const uint32_t blog2 = std::min<uint32_t>(31, std::max<uint32_t>(bit_width(nrep), 4) + tc.bucket_extra);
        ba.shift = 64 - blog2;
        pb.nb = uint32_t(1) << blog2;
        pb.with_bloom = !wide && uint64_t(nrep) * 8 <= (uint64_t(32) << kBloomMaxLog2);
        pb.wlog2 = pb.with_bloom ? std::min<uint32_t>(kBloomMaxLog2,
                                                      std::max<uint32_t>(5, bit_width((uint64_t(nrep) * tc.bloom_bits + 31) / 32 - 1)))
                                 : 0;
        pb.zb_table = sizeof(uint32_t) << ba.tlog2;
        pb.zb_counts = sizeof(uint32_t) * pb.nb;
        pb.zb_cursor = sizeof(uint32_t) * pb.nb;
        pb.zb_bloom = pb.with_bloom ? sizeof(uint32_t) << pb.wlog2 : 0;
        pb.zb_scan = scan_status_bytes(pb.nb);
        pb.zbytes = round256(pb.zb_table) + round256(pb.zb_counts) + round256(pb.zb_cursor) + round256(pb.zb_bloom) +
                    pb.zb_flags + round256(pb.zb_scan);
        // Bucket offsets go into the x words of the interleaved bucket array;
        // the scatter fills each non-empty bucket's y (its first key).
        pb.buckets = alloc<uint2>(size_t(pb.nb) + 1);
        HTView& ht = pb.ht;
        ht.buckets = pb.buckets;
        ht.keys = alloc<uint32_t>(nrep);
        ht.keys_hi = wide ? alloc<uint32_t>(nrep) : nullptr;
        ht.mult = alloc<uint64_t>(nrep);
        ht.pay = alloc<uint64_t>(size_t(nrep) * std::max<uint32_t>(width, 1));
        ht.pnull = alloc<uint32_t>(nrep);
        ht.shift = ba.shift;
        ht.nentries = nrep;
        ht.width = width;
        return pb;
    }

    // Points the build's zero-start buffers into z (zbytes, zeroed by the caller).
    static void place_zero(PreparedBuild& pb, uint8_t* z) {
        pb.ba.table = reinterpret_cast<uint32_t*>(z);
        z += round256(pb.zb_table);
        pb.ba.counts = reinterpret_cast<uint32_t*>(z);
        z += round256(pb.zb_counts);
        pb.cursor = reinterpret_cast<uint32_t*>(z);
        z += round256(pb.zb_cursor);
        pb.bloom = reinterpret_cast<uint32_t*>(z);
        z += round256(pb.zb_bloom);
        pb.dflags = reinterpret_cast<uint32_t*>(z);
        z += pb.zb_flags;
        pb.scan_status = pb.zb_scan ? z : nullptr;
    }

    void publish(size_t pi, PreparedBuild& pb) {
        pb.ht.bloom = pb.with_bloom ? pb.bloom : nullptr;
        pb.ht.bloom_log2 = pb.wlog2;
        hts_[pi].view = pb.ht;
        hts_[pi].empty = false;
        hts_[pi].dflags = pb.dflags;
    }

    bool build(size_t pi, const Items& items, const SlotSources& src, const std::vector<HTView>& probes,
               int32_t key_stage) {
        PreparedBuild pb = prepare_build(pi, items, src, probes, key_stage);
        // Sideways restriction by a batched leaf's filter (built on the main
        // stream before any pipeline that probes).
        const int32_t r = ex_.pipelines[pi].restrict_by;
        if (r >= 0 && ctx_->sideways && batched_[size_t(r)] && restricted_by_[size_t(r)] < 0 &&
            hts_[size_t(r)].view.bloom && pb.ba.key.type == kInt32) {
            pb.ba.rbloom = hts_[size_t(r)].view.bloom;
            pb.ba.rlog2w = hts_[size_t(r)].view.bloom_log2;
            restricted_by_[pi] = r;
        }
        uint8_t* z = alloc<uint8_t>(pb.zbytes);
        BJ_CK(cudaMemsetAsync(z, 0, pb.zbytes, st_));
        place_zero(pb, z);
        launched(emit_aggregate(pb.ba, st_));
        launched(scan_exclusive_u32_zeroed(pb.ba.counts, reinterpret_cast<uint32_t*>(pb.buckets), pb.nb,
                                           pb.scan_status, ctx_->d_err, st_, 2));
        launched(scatter_bloom(pb.ba.tb, pb.ba.is_rep, pb.ba.shift, pb.buckets, pb.cursor, pb.ht,
                               pb.with_bloom ? pb.bloom : nullptr, pb.wlog2, ctx_->d_err, st_));
        publish(pi, pb);
        if (ctx_->tape_mode != 2) launched(ht_flags(hts_[pi].view, pb.nb, pb.dflags, ctx_->num_sms, st_));
        return true;
    }

    static_assert(size_t(kMaxLeafSlots) == kLeafBatchMaxSlots, "the planner marks restrictions on batched leaves");
    // The builds of the pipelines in `leaves` (inputs that probe nothing),
    // kMaxLeafBuilds at a time, each pass one launch over all of them on the
    // current stream, with one memset for all their zero-start buffers.
    // by[p] >= 0: leaf p's rows are restricted by the bloom filter of the
    // table of pipeline by[p] (built earlier on this stream), when it has one.
    void build_leaf_batch(const std::vector<size_t>& leaves, const std::vector<int32_t>& by) {
        for (size_t i0 = 0; i0 < leaves.size(); i0 += kMaxLeafBuilds) {
            const size_t i1 = std::min(leaves.size(), i0 + kMaxLeafBuilds);
            std::vector<PreparedBuild> pbs;
            size_t zbytes = 0;
            for (size_t i = i0; i < i1; i++) {
                const size_t pi = leaves[i];
                pipes_++;
                const PipelinePlan& pp = ex_.pipelines[pi];
                Items items{};
                items.count = uint32_t(ex_.inputs[pp.input].rows);
                SlotSources src{};
                src.n = int(pp.slots.size());
                for (size_t j = 0; j < pp.slots.size(); j++) {
                    src.s[j].kind = 0;  // a leaf's slots are its own columns
                    src.s[j].col = col(pp.slots[j].attr);
                }
                pbs.push_back(prepare_build(pi, items, src, {}));
                zbytes += pbs.back().zbytes;
            }
            uint8_t* z = alloc<uint8_t>(zbytes);
            BJ_CK(cudaMemsetAsync(z, 0, zbytes, st_));
            LeafBatch batch{};
            batch.err = ctx_->d_err;
            batch.flags = ctx_->tape_mode != 2 ? 1 : 0;
            size_t zoff = 0;
            for (size_t k = 0; k < pbs.size(); k++) {
                PreparedBuild& pb = pbs[k];
                place_zero(pb, z + zoff);
                zoff += pb.zbytes;
                LeafBuild& L = batch.l[batch.n];
                L.key = pb.ba.key;
                L.nslots = pb.ba.src.n;
                for (int j = 0; j < pb.ba.src.n; j++) L.cols[j] = pb.ba.src.s[j].col;
                L.tb = pb.ba.tb;
                L.table = pb.ba.table;
                L.tlog2 = pb.ba.tlog2;
                L.is_rep = pb.ba.is_rep;
                L.counts = pb.ba.counts;
                L.shift = pb.ba.shift;
                L.distinct = pb.ba.distinct;
                L.buckets = pb.buckets;
                L.nb = pb.nb;
                L.cursor = pb.cursor;
                L.bloom = pb.with_bloom ? pb.bloom : nullptr;
                L.log2w = pb.wlog2;
                L.dflags = pb.dflags;
                L.ht = pb.ht;
                const int32_t r = by[leaves[i0 + k]];
                if (r >= 0 && hts_[size_t(r)].view.bloom) {
                    L.rbloom = hts_[size_t(r)].view.bloom;
                    L.rlog2w = hts_[size_t(r)].view.bloom_log2;
                    restricted_by_[leaves[i0 + k]] = r;
                }
                batch.tuple_start[batch.n + 1] = batch.tuple_start[batch.n] + pb.ba.tb.count;
                batch.block_start[batch.n + 1] = batch.block_start[batch.n] + (pb.ba.tb.count + 255) / 256;
                batch.tile_start[batch.n + 1] =
                    batch.tile_start[batch.n] + (pb.nb + kLeafTileBuckets - 1) / kLeafTileBuckets;
                batch.n++;
            }
            batch.tile_sums = alloc<uint32_t>(batch.tile_start[batch.n]);
            launched(build_leaves(batch, st_));
            for (size_t k = 0; k < pbs.size(); k++) publish(leaves[i0 + k], pbs[k]);
        }
    }

    void output(const Items& items, const SlotSources& src, const std::vector<HTView>& probes, bj_result& res,
                int flags) {
        const uint32_t n = items.count;
        // Output row offsets: the scan of the item multiplicities, or the
        // identity when every item has multiplicity 1.
        uint64_t* off = nullptr;
        uint64_t N = n;
        if (items.mult) {
            uint64_t* mult = alloc<uint64_t>(n);
            launched(items_mult(items, mult, st_));
            off = alloc<uint64_t>(size_t(n) + 1);
            N = scan_total_u64(mult, off, n);
        }
        res.rows = N;
        const size_t ncol = ex_.out_slot.size();
        // When every item is one output row, fixed-width columns are written
        // straight from the items; only the slots VARCHAR columns use (their
        // lengths are needed first) go through flat arrays.
        const bool direct = items.mult == nullptr;
        std::vector<uint8_t> flat(src.n, direct ? 0 : 1);
        for (size_t c = 0; c < ncol; c++)
            if (ex_.out_types[c] == BJ_VARCHAR) flat[ex_.out_slot[c]] = 1;
        FlatOut fo{};
        fo.n = src.n;
        bool any_flat = false;
        for (int j = 0; j < src.n; j++) {
            if (!flat[j]) continue;
            fo.vals[j] = alloc<uint64_t>(N);
            fo.valid[j] = alloc<uint8_t>(N);
            any_flat = true;
        }
        // With every item one result row the only flat slots are VARCHAR
        // ones, and the length pass computes them from the items itself.
        if (any_flat && !direct) launched(emit_output(items, off, src, probes.data(), fo, ctx_->d_err, st_));
        // Page counts per result column.
        res.npages.assign(ncol, 0);
        struct StrPlan {
            uint32_t* lens = nullptr;
            uint64_t* start = nullptr;   // exclusive scan of row costs
            uint32_t* stats = nullptr;   // [0] max cost, [1] long string present
            uint32_t* block_off = nullptr;
            uint64_t* resolved = nullptr;  // string handles of row-number values
            bool floor = false;
            uint64_t cp = 0;
        };
        std::vector<StrPlan> sp(ncol);
        std::vector<size_t> strcols;
        for (size_t c = 0; c < ncol; c++) {
            const int32_t t = ex_.out_types[c];
            if (t == BJ_VARCHAR) {
                strcols.push_back(c);
                continue;
            }
            const size_t rpp = full_page_rows(t == BJ_INT32 ? 4 : 8);
            res.npages[c] = (N + rpp - 1) / rpp;
        }
        // Lengths, costs and cost scans of every VARCHAR column (batches of up
        // to kMaxOut columns, one launch each), then one read-back.
        for (size_t i0 = 0; i0 < strcols.size(); i0 += 20) {
            const size_t i1 = std::min(strcols.size(), i0 + 20);
            uint32_t* stats = alloc<uint32_t>(2 * (i1 - i0));
            BJ_CK(cudaMemsetAsync(stats, 0, sizeof(uint32_t) * 2 * (i1 - i0), st_));
            StrCols sc{};
            sc.items = items;
            sc.ps = make_probe_set(probes.data(), items.nprobes);
            ScanBatch64 sb{};
            for (size_t i = i0; i < i1; i++) {
                const size_t c = strcols[i];
                const uint32_t j = ex_.out_slot[c];
                StrCol& x = sc.c[sc.n++];
                x.handles = fo.vals[j];
                x.valid = fo.valid[j];
                if (direct) {
                    x.from_items = 1;
                    x.slot = src.s[j];
                    x.vals_out = fo.vals[j];
                    x.valid_out = fo.valid[j];
                }
                x.src = col(ex_.pipelines.back().slots[j].attr);
                // Values of a VARCHAR column without NULLs are its row numbers
                // (slot_value); the length pass turns them into string handles.
                if (!(x.src.flags & kColNulls)) x.resolved = sp[c].resolved = alloc<uint64_t>(N);
                x.lens = sp[c].lens = alloc<uint32_t>(N);
                x.cost = alloc<uint64_t>(N);
                x.stats = sp[c].stats = stats + 2 * (i - i0);
                sp[c].start = alloc<uint64_t>(N + 1);
                sb.in[sb.n] = x.cost;
                sb.out[sb.n++] = sp[c].start;
            }
            launched(string_len_cost(sc, N, ctx_->d_err, st_));
            launched(scan_exclusive_u64_batch(sb, N, A_, st_));
            for (size_t i = i0; i < i1; i++) {
                const StrPlan& q = sp[strcols[i]];
                const int slot = int(3 * (i - i0));
                if (N) stash_u64(ctx_, q.start + (N - 1), slot);
                stash_u32(ctx_, q.stats, slot + 1);
                stash_u32(ctx_, q.stats + 1, slot + 2);
            }
            stash_err(ctx_);
            readback(ctx_, 0);
            for (size_t i = i0; i < i1; i++) {
                StrPlan& q = sp[strcols[i]];
                const int slot = int(3 * (i - i0));
                const uint64_t last_start = N ? ctx_->h_small[slot] : 0;
                const uint64_t maxc = ctx_->h_small[slot + 1];
                const bool has_long = ctx_->h_small[slot + 2] != 0;
                // Floor packing while the longest string keeps pages at least ~87% full.
                if (!has_long && maxc <= kStrPageUnits / 8) {
                    q.floor = true;
                    q.cp = kStrPageUnits - maxc;
                    res.npages[strcols[i]] = N ? last_start / q.cp + 1 : 0;
                }
            }
        }
        for (size_t c : strcols) {
            if (sp[c].floor) continue;
            const uint32_t j = ex_.out_slot[c];
            const size_t nblocks = (N + kStrBlock - 1) / kStrBlock;
            uint32_t* bp = alloc<uint32_t>(nblocks);
            sp[c].block_off = alloc<uint32_t>(nblocks + 1);
            launched(string_pack(sp[c].lens, fo.valid[j], N, 0, bp, nullptr, nullptr, st_));
            res.npages[c] = scan_total_u32(bp, sp[c].block_off, nblocks);
        }
        res.page_base.assign(ncol, 0);
        uint64_t total = 0;
        for (size_t c = 0; c < ncol; c++) {
            res.page_base[c] = total;
            total += res.npages[c];
        }
        res.total_pages = total;
        uint8_t* dst = nullptr;
        if (ctx_->graph_output) {
            dst = alloc<uint8_t>(total * kPageSize);
            res.arena_pages = dst;
        } else if (flags & BJ_RESULT_DEVICE) {
            if (total) BJ_CK(cudaMallocAsync(reinterpret_cast<void**>(&res.dev), total * kPageSize, st_));
            dst = res.dev;
        } else {
            dst = alloc<uint8_t>(total * kPageSize);
        }
        // Page descriptors of the VARCHAR columns: floor-packed ones in one
        // launch, greedy-packed ones per column.
        std::vector<StrPageDesc*> descs(ncol, nullptr);
        FloorCols fc{};
        for (size_t c : strcols) {
            descs[c] = alloc<StrPageDesc>(std::max<uint64_t>(res.npages[c], 1));
            const uint32_t j = ex_.out_slot[c];
            if (!sp[c].floor) {
                launched(string_pack(sp[c].lens, fo.valid[j], N, 1, nullptr, sp[c].block_off, descs[c], st_));
                continue;
            }
            fc.start[fc.n] = sp[c].start;
            fc.descs[fc.n] = descs[c];
            fc.cp[fc.n++] = sp[c].cp;
            if (fc.n == kMaxOut) {
                launched(string_floor_first(fc, N, st_));
                fc = FloorCols{};
            }
        }
        launched(string_floor_first(fc, N, st_));
        // Every page of every column, up to kMaxOut columns per launch.
        for (size_t c0 = 0; c0 < ncol; c0 += kMaxOut) {
            const size_t c1 = std::min(ncol, c0 + kMaxOut);
            OutColumns oc{};
            oc.nrows = N;
            oc.items = items;
            oc.ps = make_probe_set(probes.data(), items.nprobes);
            for (size_t c = c0; c < c1; c++) {
                const int32_t t = ex_.out_types[c];
                const uint32_t j = ex_.out_slot[c];
                OutColumn& o = oc.c[oc.n++];
                o.type = t;
                o.vals = fo.vals[j];
                o.valid = fo.valid[j];
                o.page_base = uint32_t(res.page_base[c] - res.page_base[c0]);
                o.npages = uint32_t(res.npages[c]);
                if (t != BJ_VARCHAR) {
                    o.rpp = uint32_t(full_page_rows(t == BJ_INT32 ? 4 : 8));
                    if (!flat[j]) {
                        o.direct = 1;
                        o.slot = src.s[j];
                    }
                } else {
                    o.floor = sp[c].floor ? 1u : 0u;
                    o.lens = sp[c].lens;
                    o.descs = descs[c];
                    o.src = col(ex_.pipelines.back().slots[j].attr);
                    if (sp[c].resolved) o.vals = sp[c].resolved;
                }
            }
            const uint64_t pages = res.page_base[c1 - 1] + res.npages[c1 - 1] - res.page_base[c0];
            launched(write_pages(oc, uint32_t(pages), dst + res.page_base[c0] * kPageSize, ctx_->d_err, st_));
        }
        if (!ctx_->graph_output && !(flags & BJ_RESULT_DEVICE) && total) {
            res.host = ctx_->take_pinned(total * kPageSize);
            BJ_CK(cudaMemcpyAsync(res.host.p, dst, total * kPageSize, cudaMemcpyDeviceToHost, st_));
            res.stats.d2h_bytes += total * kPageSize;
        }
        res.stats.output_pages = total;
    }

    bj_context* ctx_;
    const ExecPlan& ex_;
    std::vector<const DevTable*> tables_;
    cudaStream_t st_;
    Arena& A_;
    std::vector<BuiltHT> hts_;
    std::vector<int32_t> restricted_by_;  // per pipeline: the pipeline whose filter restricted its build, or -1
    std::vector<uint8_t> batched_;        // per pipeline: a leaf built in the batches before every other pipeline
    uint64_t pipes_ = 0;
};

void set_empty_result(bj_result& r, const ExecPlan& ex) {
    r.rows = 0;
    r.types = ex.out_types;
    r.npages.assign(ex.out_types.size(), 0);
    r.page_base.assign(ex.out_types.size(), 0);
    r.total_pages = 0;
}

} // namespace

bool run_pipelines(bj_context* ctx, const ExecPlan& ex, const std::vector<const DevTable*>& tables, bj_result& res,
                   int flags, uint64_t& pipelines) {
    Executor exe(ctx, ex, tables);
    const bool nonempty = exe.run(res, flags);
    pipelines = exe.pipelines_run();
    return nonempty;
}

int fail_to_status(bj_context* ctx, const Fail& f) {
    ctx->last_error = f.msg;
    ctx->gather.n = 0;
    for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
    ctx->prof_events.clear();
    for (cudaEvent_t e : ctx->phase_events) cudaEventDestroy(e);
    ctx->phase_events.clear();
    ctx->prof_bytes = 0;
    // Leave every stream idle and the arena reusable after a failure.
    ctx->sync_all();
    ctx->prefetch = bj_context::WindowPrefetch{};
    cudaGetLastError();
    uint32_t zero = 0;
    cudaMemcpy(ctx->d_err, &zero, sizeof(zero), cudaMemcpyHostToDevice);
    ctx->arena.reset();
    return f.status;
}

namespace {

// Speculative layout of a host-resident fixed-width column read in place:
// page 0 and the last page (read directly, they are in host memory) both
// without NULLs, page 0 holding rpp rows that fit the page format, the last
// at most rpp, and (pages - 1) * rpp + last rows = the table's rows. The
// column then runs without a device page index (row r is on page r / rpp);
// every other page's header must equal page 0's, which host threads check
// while the GPU works (SpecCheck); a mismatch reruns the call with the full
// index. Reads stay inside pages either way.
bool guess_uniform(const bj_column& hc, uint64_t rows, uint32_t& h0_out) {
    if ((hc.type != BJ_INT32 && hc.type != BJ_INT64 && hc.type != BJ_FP64) || hc.num_pages == 0) return false;
    const uint32_t h0 = *static_cast<const uint32_t*>(hc.pages[0]);
    const uint32_t hl = *static_cast<const uint32_t*>(hc.pages[hc.num_pages - 1]);
    const uint32_t n0 = h0 & 0xffff, nl = hl & 0xffff;
    const uint32_t w = hc.type == BJ_INT32 ? 4 : 8;
    if (n0 == 0 || (h0 >> 16) != n0 || w + uint64_t(w) * n0 + (n0 + 7) / 8 > kPageSize) return false;
    if (nl == 0 || nl > n0 || (hl >> 16) != nl) return false;
    if (uint64_t(hc.num_pages - 1) * n0 + nl != rows) return false;
    h0_out = h0;
    return true;
}

struct SpecMiss {};  // a speculative page layout was wrong: rerun with the page index

// Asynchronous check of the speculated columns' page headers.
struct SpecCheck {
    std::vector<std::pair<const bj_column*, uint32_t>> cols;  // column, expected header
    std::future<bool> ok;
    void start(ThreadPool* pool) {
        if (cols.empty()) return;
        ok = std::async(std::launch::async, [this, pool] {
            std::atomic<bool> good{true};
            for (const auto& [hc, h0] : cols) {
                const uint64_t np = hc->num_pages, per = 4096;
                if (np < 3) continue;
                pool->parallel_for((np - 2 + per - 1) / per, [&, hc = hc, h0 = h0](size_t t) {
                    const uint64_t lo = 1 + t * per, hi = std::min<uint64_t>(np - 1, lo + per);
                    for (uint64_t q = lo; q < hi && good.load(std::memory_order_relaxed); q++)
                        if (*static_cast<const uint32_t*>(hc->pages[q]) != h0) good = false;
                });
            }
            return good.load();
        });
    }
    int result = -1;  // -1 unknown, 0 a header differs, 1 all match
    bool passed() {
        if (result < 0) result = (!ok.valid() || ok.get()) ? 1 : 0;
        return result == 1;
    }
    ~SpecCheck() {
        if (ok.valid()) ok.wait();
    }
};

} // namespace

// Shared tail of bj_execute / bj_execute_resident.
int execute_common(bj_context* ctx, const bj_plan* plan, bj_resident* const* resident, int flags, bj_result** out,
                   bool speculate) {
    auto t0 = std::chrono::steady_clock::now();
    if (!ctx || !plan || !out) return BJ_ERR_INVALID;
    trace_begin(ctx->stream);
    ctx->prefetch = bj_context::WindowPrefetch{};  // a prefetch never outlives its call
    ctx->drain_releases();
    *out = nullptr;
    std::unique_ptr<bj_result> res(new bj_result);
    res->ctx = ctx;
    SpecCheck spec;
    bool planned_with_cards = false;
    bool planned_reference = false;
    ctx->item_overflow = false;
    try {
        ExecPlan ex;
        std::string err;
        // Set cardinalities for the join-order program of a resident plan:
        // a graph's recorded ones, or fresh estimates under the context's
        // ordering mode (none: the row-count model).
        std::vector<double> cards;
        const std::vector<double>* use_cards = nullptr;
        const int ordering = ctx->retry_ordering >= 0 ? ctx->retry_ordering : ctx->ordering;
        if (resident && ctx->cards_in) {
            use_cards = ctx->cards_in->empty() ? nullptr : ctx->cards_in;
        } else if (resident && ordering == BJ_ORDER_ROWS) {
            if (ctx->cards_out) ctx->cards_out->clear();
        } else if (resident) {
            {
                const int saved = ctx->ordering;
                ctx->ordering = ordering;
                try {
                    estimate_set_cards(ctx, *plan, resident, cards);
                } catch (...) {
                    ctx->ordering = saved;
                    throw;
                }
                ctx->ordering = saved;
                if (!cards.empty()) use_cards = &cards;
                if (ctx->cards_out) *ctx->cards_out = cards;
            }
        }
        planned_with_cards = use_cards != nullptr;
        const PlanSpace space =
            ctx->space_in ? *ctx->space_in : ctx->retry_rooted ? PlanSpace::Rooted : ctx->plan_space;
        int st = make_exec_plan(*plan, ex, err, false, use_cards, space);
        planned_reference = ex.reference_space;
        if (ctx->space_out) *ctx->space_out = space;
        if (st != BJ_OK) throw Fail{st, err};
        ctx->tune = tune_for(ctx, ex);
        res->types = ex.out_types;
        uint64_t launches0 = ctx->launches;
        BJ_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
        BJ_CK(cudaEventRecord(ctx->ev0, ctx->stream));
        std::vector<DevTable> owned;
        std::vector<const DevTable*> tables(plan->num_inputs, nullptr);
        if (resident) {
            for (uint64_t i = 0; i < plan->num_inputs; i++) {
                if (!resident[i]) throw Fail{BJ_ERR_INVALID, "missing resident table"};
                tables[i] = &resident[i]->table;
            }
        } else {
            // Upload only the columns the scans read.
            owned.resize(plan->num_inputs);
            std::vector<ColumnJob> jobs;
            for (uint64_t i = 0; i < plan->num_inputs; i++) {
                const bj_table& t = plan->inputs[i];
                DevTable& d = owned[i];
                d.rows = t.num_rows;
                d.cols.assign(t.num_columns, DevColumn{});
                collect_columns(ex, uint32_t(i), t.num_columns, d.present);
                tables[i] = &d;
                if (t.num_rows == 0) continue;
                if (t.num_columns && !t.columns) throw Fail{BJ_ERR_INVALID, "table without column array"};
                for (uint64_t c = 0; c < t.num_columns; c++) {
                    if (!d.present[c]) continue;
                    const bj_column& hc = t.columns[c];
                    if (hc.num_pages && !hc.pages) throw Fail{BJ_ERR_INVALID, "column without page array"};
                    d.cols[c].type = hc.type;
                    res->stats.input_pages += hc.num_pages;
                    uint8_t* mapped = nullptr;
                    const uint8_t* pinned = pinned_base(hc, mapped);
                    if (!ctx->zero_copy || !read_in_place(hc, mapped)) mapped = nullptr;
                    if (mapped) {
                        res->stats.mapped_input_bytes += hc.num_pages * kPageSize;
                        uint32_t h0 = 0;
                        if (speculate && guess_uniform(hc, t.num_rows, h0)) {
                            DevColumn& dc = d.cols[c];
                            dc.pages = mapped;
                            dc.npages = uint32_t(hc.num_pages);
                            dc.nrows = uint32_t(t.num_rows);
                            dc.flags = kColHostPages;
                            set_rpp(dc, h0 & 0xffff);
                            spec.cols.emplace_back(&hc, h0);
                            continue;
                        }
                        jobs.push_back(ColumnJob{&hc, mapped, t.num_rows, &d.cols[c], true});
                        continue;
                    }
                    uint8_t* dp = static_cast<uint8_t*>(ctx->arena.alloc(std::max<uint64_t>(hc.num_pages, 1) * kPageSize));
                    jobs.push_back(ColumnJob{&hc, dp, t.num_rows, &d.cols[c], false, pinned});
                }
            }
            trace("plan and input columns");
            if (!ex.empty) {
                res->stats.h2d_bytes += upload_pages(ctx, jobs);
                trace("pages staged");
            }
            if (!ex.empty && ctx->stream_scans && ctx->zero_copy) {
                // Begin streaming the key column the output pipeline will most
                // likely scan once the small inputs are across the host link,
                // while they are indexed and built; the executor takes the
                // windows over if it agrees.
                const int k = guess_first_probe(ex, *plan);
                if (k >= 0) {
                    const PipelinePlan& root = ex.pipelines.back();
                    const PlanAttr& pa = ex.attrs[root.probes[size_t(k)].probe_attr];
                    const uint32_t table = ex.inputs[pa.input].table;
                    const DevColumn& dc = owned[table].cols[pa.column];
                    const uint8_t* pages = dc.pages;
                    uint32_t npages = dc.npages;
                    if (!pages)  // a mapped column indexed below: its job has the address
                        for (const ColumnJob& j : jobs)
                            if (j.out == &dc && j.in_place) {
                                pages = j.dpages;
                                npages = uint32_t(j.src->num_pages);
                            }
                    if (pages && npages >= kWindowPages && (dc.flags & kColHostPages || !dc.pages)) {
                        start_window_prefetch(ctx, pages, npages, ctx->stream);
                        trace("scan windows prefetching");
                    }
                }
            }
            if (!ex.empty) {
                index_columns(ctx, jobs, ctx->arena);
                trace("pages indexed");
                spec.start(ctx->pool.get());
            }
        }
        if (resident) {
            for (uint64_t i = 0; i < plan->num_inputs; i++) {
                std::vector<uint8_t> used;
                collect_columns(ex, uint32_t(i), tables[i]->cols.size(), used);
                for (size_t c = 0; c < used.size(); c++)
                    if (used[c]) {
                        if (!tables[i]->present[c]) throw Fail{BJ_ERR_INVALID, "resident table lacks a scanned column"};
                        res->stats.input_pages += tables[i]->cols[c].npages;
                    }
            }
        }
        bool nonempty = false;
        uint64_t pipes = 0;
        if (!ex.empty) {
            Executor exe(ctx, ex, tables);
            nonempty = exe.run(*res, flags);
            pipes = exe.pipelines_run();
        }
        end_window_prefetch(ctx, ctx->stream);
        if (!nonempty) {
            if (res->dev) cudaFreeAsync(res->dev, ctx->stream);
            res->dev = nullptr;
            ctx->give_pinned(res->host);
            res->host = PinnedBlock{};
            set_empty_result(*res, ex);
        }
        trace("executor done");
        BJ_CK(cudaEventRecord(ctx->ev1, ctx->stream));
        stash_err(ctx);
        readback(ctx, 0);
        if (!spec.passed()) throw SpecMiss{};
        trace("page layouts confirmed");
        float ms = 0;
        BJ_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        res->stats.device_ms = ms;
        for (size_t i = 0; i + 1 < ctx->prof_events.size(); i += 2) {
            float k = 0;
            BJ_CK(cudaEventElapsedTime(&k, ctx->prof_events[i], ctx->prof_events[i + 1]));
            res->stats.scan_kernel_ms += k;
            res->stats.scan_kernel_launches++;
        }
        phase_stats(ctx->phase_events, res->stats);
        res->stats.scan_kernel_bytes = ctx->prof_bytes;
        for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
        ctx->prof_events.clear();
        for (cudaEvent_t e : ctx->phase_events) cudaEventDestroy(e);
        ctx->phase_events.clear();
        ctx->prof_bytes = 0;
        res->stats.kernel_launches = ctx->launches - launches0;
        res->stats.pipelines = pipes;
        res->stats.arena_bytes = ctx->arena.used_total();
        ctx->arena.reset();
    } catch (const SpecMiss&) {
        // Not an error: the call runs again with a page index for every column.
        if (res->dev) cudaFree(res->dev);
        res->dev = nullptr;
        ctx->give_pinned(res->host);
        res->host = PinnedBlock{};
        for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
        ctx->prof_events.clear();
        for (cudaEvent_t e : ctx->phase_events) cudaEventDestroy(e);
        ctx->phase_events.clear();
        ctx->prof_bytes = 0;
        ctx->arena.reset();
        res.reset();
        return execute_common(ctx, plan, resident, flags, out, false);
    } catch (const Fail& f) {
        if (res->dev) cudaFree(res->dev);
        res->dev = nullptr;
        ctx->give_pinned(res->host);
        res->host = PinnedBlock{};
        // A device check that failed on a speculated layout that was wrong:
        // clear the error and run again with the page index.
        if (!spec.cols.empty() && !spec.passed()) {
            fail_to_status(ctx, f);
            ctx->last_error.clear();
            res.reset();
            return execute_common(ctx, plan, resident, flags, out, false);
        }
        // A join order whose intermediate result outgrew 32-bit item counts
        // or the device memory: a rerun with another plan, one change at a
        // time -- the rooted plan of the same cardinalities after a plan of
        // the reference's space; then (resident tables) the other
        // cardinality source: the row-count model after estimates, join
        // samples after the row-count model.
        const bool too_big = ctx->item_overflow || f.status == BJ_ERR_OOM;
        const bool to_rooted = planned_reference && !ctx->retry_rooted;
        const bool to_cards = !to_rooted && ctx->retry_ordering < 0 && (planned_with_cards || resident);
        if (too_big && !ctx->cards_in && !ctx->space_in && (to_rooted || to_cards)) {
            fail_to_status(ctx, f);
            ctx->last_error.clear();
            res.reset();
            if (ctx->tape && ctx->tape_mode == 1) ctx->tape->slots.clear();
            const int saved_ordering = ctx->retry_ordering;
            const bool saved_rooted = ctx->retry_rooted;
            if (to_rooted) {
                ctx->retry_rooted = true;
            } else {
                ctx->retry_ordering = planned_with_cards ? BJ_ORDER_ROWS : BJ_ORDER_SAMPLING;
                ctx->retry_rooted = false;
            }
            const int rst = execute_common(ctx, plan, resident, flags, out, speculate);
            ctx->retry_ordering = saved_ordering;
            ctx->retry_rooted = saved_rooted;
            return rst;
        }
        return fail_to_status(ctx, f);
    } catch (const std::bad_alloc&) {
        return fail_to_status(ctx, Fail{BJ_ERR_OOM, "host allocation failed"});
    } catch (const std::exception& e) {
        return fail_to_status(ctx, Fail{BJ_ERR_INTERNAL, e.what()});
    }
    res->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->live_results++;
    ctx->last_error.clear();
    *out = res.release();
    return BJ_OK;
}

} // namespace bj
