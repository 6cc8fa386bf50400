// Internal declarations shared by the engine's host sources (engine.cpp,
// graphs.cpp, resident.cpp, api.cpp, estimator.cpp): error type,
// host thread pool, device arena and persistent allocations, the context,
// resident tables and results. Not part of the public ABI (include/b200join.h).
#pragma once

#include "../../include/b200join.h"
#include "launch.h"
#include "planner.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace bj {

struct Fail {
    int status;
    std::string msg;
};

#define BJ_CK(call)                                                                                      \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw Fail{e_ == cudaErrorMemoryAllocation ? BJ_ERR_OOM : BJ_ERR_CUDA,                       \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};                              \
    } while (0)

inline uint32_t bit_width(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

inline size_t full_page_rows(size_t width) {
    size_t begin = width == 8 ? 8 : 4, n = 0;
    while (begin + (n + 1) * width + (n / 8 + 1) <= kPageSize) n++;
    return n;
}

// ---------------------------------------------------------------------------
// Host thread pool (page staging).
class ThreadPool {
    public:
    explicit ThreadPool(unsigned n) {
        for (unsigned i = 0; i < n; i++) workers_.emplace_back([this] { loop(); });
    }
    ~ThreadPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    size_t size() const { return workers_.size() + 1; }
    // Runs fn(i) for i in [0, n) on the pool and the calling thread.
    void parallel_for(size_t n, const std::function<void(size_t)>& fn) {
        if (n == 0) return;
        if (workers_.empty() || n == 1) {
            for (size_t i = 0; i < n; i++) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &fn;
            n_ = n;
            next_ = 0;
            active_ = workers_.size();
            gen_++;
        }
        cv_.notify_all();
        run_items();
        std::unique_lock<std::mutex> g(m_);
        done_cv_.wait(g, [this] { return active_ == 0; });
        job_ = nullptr;
    }

    private:
    void run_items() {
        for (;;) {
            size_t i = next_.fetch_add(1);
            if (i >= n_) break;
            (*job_)(i);
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            run_items();
            {
                std::lock_guard<std::mutex> g(m_);
                if (--active_ == 0) done_cv_.notify_all();
            }
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(size_t)>* job_ = nullptr;
    std::atomic<size_t> next_{0};
    size_t n_ = 0, active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// ---------------------------------------------------------------------------
// Device arena: bump allocation over large chunks, reset after each call.
class Arena : public Scratch {
    public:
    ~Arena() override {
        for (auto& c : chunks_) cudaFree(c.p);
    }
    void* alloc(size_t bytes) override {
        bytes = (bytes + 255) & ~size_t(255);
        if (bytes == 0) bytes = 256;
        for (; cur_ < chunks_.size(); cur_++) {
            Chunk& c = chunks_[cur_];
            if (c.used + bytes <= c.size) {
                void* p = c.p + c.used;
                c.used += bytes;
                high_ = std::max(high_, used_total() );
                return p;
            }
        }
        size_t sz = std::max<size_t>(bytes, size_t(1) << 30);
        uint8_t* p = nullptr;
        cudaError_t e = cudaMalloc(&p, sz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Fail{BJ_ERR_OOM, "device arena: cudaMalloc of " + std::to_string(sz) + " bytes failed"};
        }
        chunks_.push_back(Chunk{p, sz, bytes});
        cur_ = chunks_.size() - 1;
        return p;
    }
    void reset() {
        for (auto& c : chunks_) c.used = 0;
        cur_ = 0;
    }
    size_t used_total() const {
        size_t u = 0;
        for (auto& c : chunks_) u += c.used;
        return u;
    }

    private:
    struct Chunk {
        uint8_t* p;
        size_t size;
        size_t used;
    };
    std::vector<Chunk> chunks_;
    size_t cur_ = 0, high_ = 0;
};

// Persistent allocations (resident tables): plain cudaMalloc, freed together.
class PersistentAlloc : public Scratch {
    public:
    ~PersistentAlloc() override { release(); }
    void* alloc(size_t bytes) override {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Fail{BJ_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed"};
        }
        ptrs_.push_back(p);
        return p;
    }
    void release() {
        for (void* p : ptrs_) cudaFree(p);
        ptrs_.clear();
    }

    private:
    std::vector<void*> ptrs_;
};

struct PinnedBlock {
    uint8_t* p = nullptr;
    size_t size = 0;
};

// One column resident on the device.
struct DevTable {
    uint64_t rows = 0;
    std::vector<DevColumn> cols;
    std::vector<uint8_t> present;
};

inline const char* dev_error_text(uint32_t code) {
    switch (code) {
    case kErrPageHeader: return "a page header contradicts the page format";
    case kErrRowRange: return "a row index beyond its column (malformed pages)";
    case kErrCapacity: return "an internal buffer overflowed";
    case kErrLongString: return "a long-string page run is malformed";
    default: return "unknown device error";
    }
}

// Host read-backs of one query, in order: recorded on the first run of a
// repeated resident query and replayed while that query is captured into a
// CUDA graph (the capture must not synchronise).
struct ReadbackTape {
    std::vector<std::array<uint64_t, 64>> slots;
    size_t pos = 0;
};

// Build and scan parameters the autotuner chooses per plan shape class
// (bj_context_autotune): the defaults are the engine's fixed choices.
struct TuneConfig {
    uint8_t scan_split = 0;    // scan-side probe: filter + candidate probe kernels (1) or fused (0)
    uint8_t bloom_bits = 16;   // bloom filter bits per key (capped at 128 KiB per filter)
    uint8_t bucket_extra = 0;  // buckets = 2^(bit_width(tuples) + extra): lower fill factors for extra > 0
    bool operator==(const TuneConfig& o) const {
        return scan_split == o.scan_split && bloom_bits == o.bloom_bits && bucket_extra == o.bucket_extra;
    }
};

// Statistics of one join-key column of a resident table (estimator.cpp).
struct ColStats {
    bool ready = false;
    KeyMap map{};                  // key -> count of its non-null rows
    uint32_t hist[kHistBins] = {}; // non-null values by the top six bits of the key hash
    uint64_t nonnull = 0, distinct = 0;
};

// A repeated resident query captured into a CUDA graph.
struct GraphEntry {
    std::vector<uint64_t> key;               // plan, resident handles, flags
    uint64_t hash = 0;                       // of key
    std::vector<bj_resident*> tables;
    ReadbackTape tape;
    cudaGraphExec_t exec = nullptr;
    bool failed = false;                     // capture failed: always run normally
    uint64_t rows = 0;
    std::vector<uint64_t> npages, page_base;
    uint64_t total_pages = 0;
    uint8_t* pages = nullptr;                // arena pages the graph writes the result to
    std::vector<int32_t> out_types;          // result column types
    bj_stats stats{};                        // launches, pipelines, input pages of one run
    std::vector<cudaEvent_t> prof;           // timed-kernel event pairs inside the graph
    std::vector<cudaEvent_t> phase;          // phase marks inside the graph
    uint64_t prof_bytes = 0;
    std::vector<double> cards;               // set cardinalities the first run planned with (empty: none)
    PlanSpace space = PlanSpace::Auto;       // plan space the first run used
};

// Records a failed call's message on the context, leaves its streams idle and
// its arena reusable, and returns the status (engine.cpp).
int fail_to_status(bj_context* ctx, const Fail& f);

// Set cardinalities (2^inputs entries, by input mask) for the join-order
// program of a resident plan under the context's ordering mode; left empty
// for BJ_ORDER_ROWS or a plan it does not estimate (estimator.cpp).
void estimate_set_cards(bj_context* ctx, const bj_plan& plan, bj_resident* const* tables, std::vector<double>& cards);

// ---- Page upload and indexing (engine.cpp) ----

// One column to bring onto the device: its host pages and where they go.
struct ColumnJob {
    const bj_column* src;  // host pages
    uint8_t* dpages;       // device-accessible address of the pages
    uint64_t rows;         // rows the table claims
    DevColumn* out;
    bool in_place = false; // pages are read where they are (pinned host memory): no copy
    const uint8_t* pinned = nullptr;  // pages back to back in pinned host memory: one DMA from here
};

// The host address of a column's pages when they lie back to back in pinned
// host memory (and in `dev` the device address of their mapping, or nullptr);
// nullptr for pageable or scattered pages.
const uint8_t* pinned_base(const bj_column& hc, uint8_t*& dev);
// Copies the jobs' host pages to their device addresses; returns the bytes.
uint64_t upload_pages(bj_context* ctx, const std::vector<ColumnJob>& jobs);
// Builds the page index of every job's column (pages already on the device).
void index_columns(bj_context* ctx, std::vector<ColumnJob>& jobs, Scratch& mem);
// used[c] = 1 for every column of table `table_id` that the plan reads.
void collect_columns(const ExecPlan& ex, uint32_t table_id, uint64_t ncols, std::vector<uint8_t>& used);

// ---- Execution (engine.cpp) ----

constexpr size_t kPhaseMarks = 5;  // phase marks of a profiled call (bj_stats.phase_ms)
void phase_stats(const std::vector<cudaEvent_t>& marks, bj_stats& st);
// Shape class of a plan (log2 rows of its largest and second largest inputs,
// number of inputs) and the tuned parameters the context holds for it.
uint64_t shape_class(const ExecPlan& ex);
TuneConfig tune_for(const bj_context* ctx, const ExecPlan& ex);
// The drop-in path's guess of the probe the device sampling ranks first.
int guess_first_probe(const ExecPlan& ex, const bj_plan& plan);
// Shared tail of bj_execute / bj_execute_resident.
int execute_common(bj_context* ctx, const bj_plan* plan, bj_resident* const* resident, int flags, bj_result** out,
                   bool speculate = true);
// Runs every pipeline of `ex` over device tables into `res` (enqueued on the
// context's streams; used under stream capture). False: the result is empty.
bool run_pipelines(bj_context* ctx, const ExecPlan& ex, const std::vector<const DevTable*>& tables, bj_result& res,
                   int flags, uint64_t& pipelines);

// ---- CUDA-graph replay (graphs.cpp) ----

void destroy_graph(GraphEntry& g);
int execute_resident_graph(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, int flags,
                           bj_result** out);
// Waits for ctx's work, then drops its graphs that read table t.
void drop_graphs_using(bj_context* ctx, const bj_resident* t);

} // namespace bj

struct bj_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bj::Arena arena;
    bj::PinnedBlock stage;                 // upload staging
    std::vector<bj::PinnedBlock> pinned_free;
    std::unique_ptr<bj::ThreadPool> pool;
    std::string last_error;
    uint32_t* d_err = nullptr;         // device error word
    uint64_t* h_small = nullptr;       // pinned readback slots
    uint64_t* d_small = nullptr;       // device readback slots
    bj::GatherList gather{};               // values queued for the next read-back
    uint64_t launches = 0;
    std::atomic<uint64_t> live_results{0};
    int num_sms = 148;
    bool profile = false;
    int tape_mode = 0;               // 0 off, 1 record read-backs, 2 replay them (graph capture)
    bj::ReadbackTape* tape = nullptr;
    bool graph_output = false;       // result pages stay in the arena (graph capture)
    bool graphs = true;              // replay repeated resident queries as CUDA graphs
    std::vector<std::unique_ptr<bj::GraphEntry>> graph_cache;  // least recently used first
    static constexpr size_t kGraphCache = 1024;  // graphs kept: a batch of 256 distinct queries replays whole
    bool zero_copy = true;  // read pinned, contiguous input columns in place
    static constexpr int kSideStreams = 4;
    cudaStream_t side[kSideStreams] = {};  // independent build pipelines run here
    cudaStream_t copy = nullptr;           // host-to-HBM copies of a streamed scan
    bool stream_scans = true;              // scans of host pages copy them through HBM windows
    bool leaf_batch = true;                // leaf builds batched (one launch per pass)
    bool sideways = true;                  // batched leaf builds restricted by a smaller one's filter
    bool scan_split = true;                // allow the split scan where the tuned parameters ask for it
    // Autotuned parameters per plan shape class (key: shape_class), the
    // configuration of the running call, and an override while tuning.
    std::vector<std::pair<uint64_t, bj::TuneConfig>> tuned;
    bj::TuneConfig tune{};
    const bj::TuneConfig* tune_override = nullptr;
    // Join ordering of resident queries (bj_context_set_ordering): the
    // cardinalities the join-order program is given.
    int ordering = 0;                      // BJ_ORDER_ROWS / _SAMPLING / _LEARNED
    bj_estimator* estimator = nullptr;
    const std::vector<double>* cards_in = nullptr;  // a graph's recorded set cardinalities (capture)
    bool item_overflow = false;                     // the call's plan outgrew 32-bit item counts
    bj::PlanSpace plan_space = bj::plan_space_default();  // which plan space make_exec_plan runs
    int retry_ordering = -1;                        // after an overflow: the ordering of the rerun (-1: none)
    bool retry_rooted = false;                      // after an overflow: the rerun plans in the rooted space
    bj::PlanSpace* space_out = nullptr;             // where a first run records the plan space it ran
    const bj::PlanSpace* space_in = nullptr;        // a graph's recorded plan space
    std::vector<double>* cards_out = nullptr;       // where a first run records them
    std::vector<cudaEvent_t> pipe_events;  // one per pipeline, reused across calls
    std::vector<cudaEvent_t> window_events;  // a streamed scan's copy and release marks
    // Windows of a streamed scan whose copies began before the scan's column
    // was chosen (the drop-in path's guess; Executor::streamed_scan takes
    // them over when the guess holds).
    struct WindowPrefetch {
        const uint8_t* src = nullptr;  // mapped pages of the guessed column
        uint8_t* win[3] = {};
        uint32_t enqueued = 0;         // windows copying (their copy events recorded)
    } prefetch;
    // Asynchronous results: pinned error-word slots and completion events.
    static constexpr uint32_t kAsyncSlots = 256;
    uint32_t* async_err = nullptr;           // kAsyncSlots pinned words
    std::vector<uint32_t> free_slots;
    std::vector<cudaEvent_t> free_done;

    // `n` events without timing, created once and reused across calls.
    cudaEvent_t* events(std::vector<cudaEvent_t>& v, size_t n) {
        while (v.size() < n) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            v.push_back(e);
        }
        return v.data();
    }

    cudaEvent_t pipe_event(size_t i) {
        while (pipe_events.size() <= i) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            pipe_events.push_back(e);
        }
        return pipe_events[i];
    }
    void sync_all() {
        cudaStreamSynchronize(stream);
        for (cudaStream_t s : side)
            if (s) cudaStreamSynchronize(s);
        if (copy) cudaStreamSynchronize(copy);
    }
    std::vector<cudaEvent_t> prof_events;  // pairs around timed launches
    std::vector<cudaEvent_t> phase_events; // phase marks of the call (kPhaseMarks when complete)
    uint64_t prof_bytes = 0;

    // Memory that results give back, possibly on other threads than the one
    // running this context (a server hands results to its callers): kept
    // here under release_m and freed by the context's own next call, never
    // while one of its streams may be capturing a graph (a free enqueued on
    // a capturing stream would land in the graph).
    std::mutex release_m;
    std::vector<uint8_t*> release_dev;
    void release_device(uint8_t* p) {
        std::lock_guard<std::mutex> g(release_m);
        release_dev.push_back(p);
    }
    // On the context's own thread, outside stream capture.
    void drain_releases() {
        std::vector<uint8_t*> dev;
        std::vector<bj::PinnedBlock> excess;
        {
            std::lock_guard<std::mutex> g(release_m);
            dev.swap(release_dev);
            while (pinned_free.size() > 4) {
                excess.push_back(pinned_free.front());
                pinned_free.erase(pinned_free.begin());
            }
        }
        for (uint8_t* p : dev) cudaFreeAsync(p, stream);
        if (!excess.empty()) {
            cudaStreamSynchronize(stream);
            for (const bj::PinnedBlock& b : excess) cudaFreeHost(b.p);
        }
    }

    bj::PinnedBlock take_pinned(size_t bytes) {
        {
            std::lock_guard<std::mutex> g(release_m);
            for (size_t i = 0; i < pinned_free.size(); i++)
                if (pinned_free[i].size >= bytes) {
                    bj::PinnedBlock b = pinned_free[i];
                    pinned_free.erase(pinned_free.begin() + i);
                    return b;
                }
        }
        bj::PinnedBlock b;
        b.size = std::max<size_t>(bytes, 1 << 20);
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&b.p), b.size, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw bj::Fail{BJ_ERR_OOM, "pinned host allocation failed"};
        }
        return b;
    }
    void give_pinned(bj::PinnedBlock b) {
        if (!b.p) return;
        std::lock_guard<std::mutex> g(release_m);
        pinned_free.push_back(b);  // beyond four blocks, drain_releases frees the oldest
    }
};

struct bj_resident {
    bj::PersistentAlloc mem;
    bj::DevTable table;
    // Join-ordering statistics of the table's key columns, computed on first
    // use (estimator.cpp) and kept with the table.
    std::mutex stats_m;
    std::vector<bj::ColStats> stats;
    uint64_t base_rows = 0;  // rows before the load-time filter (0: unknown)
};

struct bj_result {
    bj_context* ctx = nullptr;
    uint64_t rows = 0;
    std::vector<int32_t> types;
    std::vector<uint64_t> npages;
    std::vector<uint64_t> page_base;
    uint64_t total_pages = 0;
    bj::PinnedBlock host;
    uint8_t* dev = nullptr;
    uint8_t* arena_pages = nullptr;  // capture only: where the graph leaves the result pages
    bool nonempty = false;
    bj_stats stats{};
    // BJ_RESULT_ASYNC: the work is in flight until `done`; the error word
    // lands in err_slot (one of the context's pinned slots).
    bool pending = false;
    cudaEvent_t done = nullptr;
    uint32_t slot = 0;
    int status = BJ_OK;
};

