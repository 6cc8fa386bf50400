// Host-side launch wrappers for the engine's kernels. Each wrapper enqueues
// its kernels on `st` and returns how many kernels it launched, so the host
// can account for every launch (bj_stats.kernel_launches).
#pragma once

#include "device.cuh"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace bj {

// Scratch allocator handed to wrappers that need temporary device memory;
// `err` is the device error word kernels launched with it report to.
struct Scratch {
    virtual void* alloc(size_t bytes) = 0;
    virtual ~Scratch() = default;
    uint32_t* err = nullptr;
};

// ---- prefix sums (k_util.cu) ----
// Exclusive scan of n values into out[0..n]; out[n] receives the total.
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, Scratch& s, cudaStream_t st);
int scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, Scratch& s, cudaStream_t st);
// The same scan with its tile status words supplied: scan_status_bytes(n)
// bytes (possibly 0) that the caller has zeroed, so no memset is issued.
// Output i goes to out[i * out_stride].
size_t scan_status_bytes(size_t n);
int scan_exclusive_u32_zeroed(const uint32_t* in, uint32_t* out, size_t n, void* status, uint32_t* err,
                              cudaStream_t st, uint32_t out_stride = 1);
// Independent exclusive scans of up to kMaxScanSegs u32 arrays of any
// lengths, in one launch (status_off is filled in by the wrapper).
constexpr int kMaxScanSegs = 64;
struct ScanSeg {
    const uint32_t* in;
    uint32_t* out;  // n + 1 entries
    uint32_t n;
};
struct ScanSegs {
    ScanSeg s[kMaxScanSegs];
    uint32_t status_off[kMaxScanSegs];
    int n;
};
int scan_exclusive_u32_segs(ScanSegs segs, Scratch& s, cudaStream_t st);
// Exclusive scans of several u64 arrays of length n (out[i][n] = total):
// one launch when n fits one tile.
constexpr int kMaxScanBatch = 32;
struct ScanBatch64 {
    const uint64_t* in[kMaxScanBatch];
    uint64_t* out[kMaxScanBatch];
    int n;
};
int scan_exclusive_u64_batch(const ScanBatch64& b, size_t n, Scratch& s, cudaStream_t st);
int fill_u32(uint32_t* p, uint32_t v, size_t n, cudaStream_t st);
// *out = the sum of n u32 values in 64 bits (one launch).
int sum_u32_wide(const uint32_t* in, size_t n, unsigned long long* out, cudaStream_t st);
// Gathers device values into dst[slot] (u32 zero-extended, or u64): the
// values a host read-back needs, in one launch.
constexpr int kMaxGather = 64;
struct GatherList {
    const void* src[kMaxGather];
    uint8_t slot[kMaxGather];
    uint8_t wide[kMaxGather];  // 1: u64, 0: u32
    int n;
};
int gather_values(const GatherList& g, uint64_t* dst, cudaStream_t st);

// ---- page index (k_pages.cu) ----
// Builds hdr / row_start / chunk_base / dense_base / page_of_blk for columns
// whose pages are device-accessible at `pages`; checks every page header.
// Pass 1 (headers, row and chunk offsets) and pass 2 (dense bases and block
// pages) each take every column of a batch in one launch (blockIdx.y =
// column); between them the host reads back row and chunk totals.
constexpr int kMaxIndexBatch = 32;
struct PageIndexCol {
    const uint8_t* pages;
    uint32_t npages;
    int32_t type;
    uint32_t* hdr;           // npages: page headers (kept)
    uint32_t* rows;          // npages (scratch)
    uint32_t* chunks;        // npages (scratch)
    uint32_t* row_start;     // npages + 1
    uint32_t* chunk_base;    // npages + 1
    uint32_t* flags;         // 1 word, zero before pass 1
    // pass 2
    uint32_t nrows;
    uint32_t* dense_base;    // chunk total
    uint32_t* page_of_blk;   // (nrows >> kBlkShift) + 2
};
struct PageIndexBatch {
    PageIndexCol c[kMaxIndexBatch];
    int n;
};
int page_index_pass1(const PageIndexBatch& b, uint32_t* err, Scratch& s, cudaStream_t st);
int page_index_pass2(const PageIndexBatch& b, cudaStream_t st);

// ---- pipelines (k_probe.cu) ----
// Items flowing through a pipeline: a row of the scanned input plus, per
// probe done so far, the index of the matching hash-table entry, and the
// product of the matched entries' multiplicities.
struct Items {
    const uint32_t* rows;                // null: implicit rows 0..count-1
    const uint32_t* ents[kMaxProbes];
    const uint64_t* mult;                // null: all 1
    uint32_t count;                      // item count, or an upper bound when dcount is set
    int nprobes;
    const uint32_t* dcount;              // device-side item count (null: `count` is exact)
};
struct ItemsOut {
    uint32_t* rows;
    uint32_t* ents[kMaxProbes];
    uint64_t* mult;
};
constexpr uint32_t kTile = 256;  // items per CTA tile in stage kernels (one per thread)
// Where a stage's probe key comes from: a column of the scanned input at the
// item's row (stage < 0), or payload slot `slot` of the entry that an earlier
// stage `stage` matched (table ht), an attribute of an input probed before.
struct KeySource {
    int32_t stage;
    uint32_t slot;
    HTView ht;
};


// Probe stage: for each item, read the key `key` at its row, probe `ht`,
// and emit one item per matching entry. mode 0 counts matches per tile into
// tile_counts; mode 1 writes items at tile_offsets (exclusive scan of counts).
// Mode 0 saturates a tile's count at 2^32 - 1 (recording kErrCapacity);
// mode 1 writes at most `capacity` items (more record kErrCapacity).
int probe_stage(const Items& in, const DevColumn& key, const HTView& ht, int mode, uint32_t* tile_counts,
                const uint32_t* tile_offsets, ItemsOut out, bool use_bloom, uint32_t* err, cudaStream_t st,
                uint32_t capacity = 0xffffffffu, KeySource src = KeySource{-1, 0, HTView{}});

// Consecutive probe stages against tables with unique keys (at most one
// match per item and stage), fused: an item probes the stages in order and
// is dropped at its first miss; survivors are appended with warp-aggregated
// atomics at *cursor, with one entry per stage after the input's. Reads the
// input count from in.dcount when set, so no host round trip is needed
// between stages. out.mult may be null when the input and every table carry
// only multiplicity 1.
constexpr int kMaxChain = 8;
struct ChainStage {
    DevColumn key;   // probe key column of the scanned input (src.stage < 0)
    HTView ht;
    int use_bloom;   // test ht.bloom (in global memory) first
    KeySource src;   // src.stage >= 0: the key is an earlier stage's payload (from an earlier launch)
};
struct ProbeChain {
    ChainStage st[kMaxChain];
    int n;
};
// dfirst (optional): the items start at index *dfirst instead of 0; dend
// (optional): receives the item count read from in.dcount, so that the next
// launch over items appended after this one can start there.
int probe_chain_unique(const Items& in, const ProbeChain& chain, ItemsOut out, uint32_t* cursor, uint32_t capacity,
                       uint32_t* err, int num_sms, cudaStream_t st, const uint32_t* dfirst = nullptr,
                       uint32_t* dend = nullptr);

// Source of one value slot: a column of the scanned input read at the item's
// row, or payload slot `slot` of the entry matched by probe `probe`.
struct SlotSource {
    int32_t kind;  // 0: column, 1: probe payload, 2: key of the entry matched by probe `probe`
    int32_t probe;
    int32_t slot;
    int32_t pad;
    DevColumn col;
};
constexpr int kMaxOut = 32;
struct SlotSources {
    SlotSource s[kMaxOut];
    int n;
};
// The tables probed so far by a pipeline, by stage.
struct ProbeSet {
    HTView ht[kMaxProbes];
};
inline ProbeSet make_probe_set(const HTView* probes, int n) {
    ProbeSet ps{};
    for (int i = 0; i < n && i < kMaxProbes; i++) ps.ht[i] = probes[i];
    return ps;
}

#if defined(__CUDACC__)
// Key of item i from a payload source (src.stage >= 0); false for NULL.
__device__ __forceinline__ bool payload_key(const KeySource& src, const uint32_t* const* ents, uint32_t i,
                                            uint64_t& v) {
    const uint32_t e = ents[src.stage][i];
    if ((src.ht.pnull[e] >> src.slot) & 1) return false;
    v = src.ht.pay[size_t(e) * src.ht.width + src.slot];
    return true;
}
__device__ __forceinline__ uint32_t item_row(const Items& in, uint32_t i) { return in.rows ? in.rows[i] : i; }
__device__ __forceinline__ uint64_t item_mult(const Items& in, uint32_t i) { return in.mult ? in.mult[i] : 1ull; }
// Value of `row` of column c as a slot carries it. A VARCHAR column without
// NULLs yields the row number, not a string handle: locating the row's page
// is left to the output, which does it for result rows only
// (StrCol::resolved), instead of every build tuple and item paying for it.
__device__ __forceinline__ bool column_value(const DevColumn& c, uint32_t row, uint64_t& v) {
    if (c.type == kVarchar && !(c.flags & kColNulls)) {
        v = row;
        return true;
    }
    return col_get(c, row, v);
}

// Value of one slot for item i (row `row`): returns false for NULL.
__device__ __forceinline__ bool slot_value(const SlotSource& s, const Items& in, uint32_t i, uint32_t row,
                                           const ProbeSet& ps, uint64_t& v) {
    if (s.kind == 0) return column_value(s.col, row, v);
    const uint32_t e = in.ents[s.probe][i];
    if (s.kind == 2) {
        v = ht_key(ps.ht[s.probe], e);
        return true;
    }
    const HTView& ht = ps.ht[s.probe];
    if ((ht.pnull[e] >> s.slot) & 1) return false;
    v = ht.pay[size_t(e) * ht.width + s.slot];
    return true;
}
#endif

// Output emit: item multiplicities are expanded; out_off[i] = first output row
// of item i (exclusive scan of multiplicities; null when every item has
// multiplicity 1, item i then being row i). Values go to flat columns.
struct FlatOut {
    uint64_t* vals[kMaxOut];
    uint8_t* valid[kMaxOut];
    int n;
};
int emit_output(const Items& in, const uint64_t* out_off, const SlotSources& src, const HTView* probes, FlatOut out,
                uint32_t* err, cudaStream_t st);
// mult of implicit/explicit items as a u64 array (for the scan of output offsets)
int items_mult(const Items& in, uint64_t* mult_out, cudaStream_t st);

// ---- scan-side probe stage (k_scan.cu) ----
// Streams the pages of `key` (a column of the scanned table) and probes `ht`,
// in work units of part of a page (scan_probe_units(npages) of them, in page
// order). mode 0: match counts per unit into page_counts; mode 1: items
// written at page_off[u] (exclusive scan of the counts, units + 1 entries);
// mode 2: items appended at *cursor (requires at most one match per row).
// bloom_smem: test ht.bloom, staged in shared memory (ignored if larger than
// scan_probe_bloom_limit()). `key` may be a window of a column's pages (its
// row_start / chunk_base / hdr advanced to the window's first page): with
// uniform pages (key.rpp) the window's first row is row_base.
size_t scan_probe_bloom_limit();
uint32_t scan_probe_units(uint32_t npages);
int scan_probe(const DevColumn& key, const HTView& ht, int mode, bool bloom_smem, uint32_t* page_counts,
               const uint32_t* page_off, uint32_t* cursor, uint32_t* out_rows, uint32_t* out_ents, uint64_t* out_mult,
               uint32_t capacity, uint32_t* err, int num_sms, cudaStream_t st, uint32_t row_base = 0);

// The same stage (mode 2: unique build keys, bloom filter present) as two
// kernels: the scan streams the key pages and appends every bloom survivor
// (key, row) to a candidate list (cand_count zero before; room for
// cand_cap, at most the column's rows), then a probe kernel probes the list
// and appends items at *cursor. The scan then carries no probe code.
int scan_probe_split(const DevColumn& key, const HTView& ht, uint32_t* cursor, uint32_t* out_rows, uint32_t* out_ents,
                     uint64_t* out_mult, uint32_t capacity, uint32_t* cand_key, uint32_t* cand_row,
                     uint32_t* cand_count, uint32_t cand_cap, uint32_t* err, int num_sms, cudaStream_t st,
                     uint32_t row_base = 0);

// ---- hash table build (k_build.cu) ----
// Tuples of a build pipeline, one per item: key from `key` (NULL key ->
// mult 0), payload from `src`, mult from the item.
struct TupleBuf {
    uint32_t* keys;
    uint32_t* keys_hi; // INT64 build keys: high halves; null for INT32
    uint64_t* mult;
    uint64_t* pay;     // count * width
    uint32_t* pnull;
    uint32_t count;
    uint32_t width;
};
// Emit, eager aggregation and bucket counts of a hash build (emit_aggregate:
// two launches, one when the build is distinct). table (1 << tlog2 words)
// and counts (one per bucket) must be zero.
struct BuildArgs {
    Items in;
    DevColumn key;       // key column of the scanned input, or (key_stage >= 0) only its type
    int32_t key_stage;   // >= 0: the key is payload slot key_slot of the entry stage key_stage matched
    uint32_t key_slot;
    SlotSources src;
    ProbeSet ps;
    TupleBuf tb;
    uint32_t* table;   // slot: index + 1 of the tuple representing it, 0 = empty
    uint32_t tlog2;
    uint32_t* is_rep;  // per tuple: 1 if it represents its distinct tuple
    uint32_t* counts;  // per bucket: representatives
    uint32_t shift;    // bucket = key_hash >> shift
    uint32_t* err;
    uint32_t distinct; // 1: no two tuples can be equal (each is its own representative; no table)
    // Sideways restriction (INT32 keys): the bloom filter (1 << rlog2w words)
    // of a table built on the same key class; a tuple whose key it cannot
    // hold is not inserted. Null: none.
    const uint32_t* rbloom;
    uint32_t rlog2w;
};
int emit_aggregate(const BuildArgs& a, cudaStream_t st);
// Scatters the representatives into their buckets' ranges (cursor: one zero
// word per bucket) and sets their bloom bits (bloom: zero, 1 << log2w words;
// null: no filter).
int scatter_bloom(TupleBuf t, const uint32_t* is_rep, uint32_t shift, uint2* buckets, uint32_t* cursor,
                  HTView ht_mut, uint32_t* bloom, uint32_t log2w, uint32_t* err, cudaStream_t st);
// The builds of inputs that probe nothing, up to kMaxLeafBuilds at a time,
// each pass one launch over all of them (k_build.cu). Each build's zero
// region (table, counts, cursor, bloom, flags) must be zero before;
// tile_sums holds tile_start[n] words.
constexpr int kMaxLeafBuilds = 6;
constexpr int kMaxLeafSlots = 4;  // leaves with more payload columns build one by one
struct LeafBuild {
    DevColumn key;                  // build key column
    DevColumn cols[kMaxLeafSlots];  // payload columns (slot j)
    int nslots;
    TupleBuf tb;
    uint32_t* table;    // aggregation table, 1 << tlog2 zero words (unused when distinct)
    uint32_t tlog2;
    uint32_t* is_rep;
    uint32_t* counts;   // nb zero words
    uint32_t shift;
    uint32_t distinct;  // see BuildArgs::distinct
    uint2* buckets;     // nb + 1: offsets written into x, first keys into y
    uint32_t nb;
    uint32_t* cursor;   // nb zero words
    uint32_t* bloom;    // zero, 1 << log2w words; null: no filter
    uint32_t log2w;
    uint32_t* dflags;   // two zero words: table flags (pass 4)
    HTView ht;          // the table's arrays to fill
    // Sideways restriction: the bloom filter (1 << rlog2w words) of another
    // table built on the same key class; a row whose key it cannot hold is
    // not inserted. Null: none.
    const uint32_t* rbloom;
    uint32_t rlog2w;
};
struct LeafBatch {
    LeafBuild l[kMaxLeafBuilds];
    int n;
    uint32_t tuple_start[kMaxLeafBuilds + 1];  // prefix of the builds' tuple counts
    uint32_t block_start[kMaxLeafBuilds + 1];  // prefix of their blocks of 256 tuples
    uint32_t tile_start[kMaxLeafBuilds + 1];   // prefix of their bucket tiles (1024 buckets each)
    uint32_t* tile_sums;
    uint32_t* err;
    int flags;          // 1: compute the table flags
};
static_assert(sizeof(LeafBatch) <= 4096, "a LeafBatch is one kernel parameter block; kept within 4 KiB");
// Returns the launches made.
int build_leaves(const LeafBatch& batch, cudaStream_t st);
constexpr uint32_t kLeafTileBuckets = 1024;

// Flags of a built table: [0] = 1 if some key repeats, [1] = 1 if some mult > 1
// (both words must be zero before). The entry count is read on the device
// from buckets[nbuckets].x.
int ht_flags(HTView ht, uint32_t nbuckets, uint32_t* flags, int num_sms, cudaStream_t st);
// Counts, for nsample evenly spaced rows of each probe's key column, how many
// hit its table: hits[p] for probe p, all probes in one launch (the role of
// the reference's 64-row join samples, engine/query/QueryPlan.cpp:719-746).
struct SampleProbe {
    DevColumn key;
    HTView ht;
};
struct SampleSet {
    SampleProbe p[kMaxProbes];
    int n;
};
int sample_probes(const SampleSet& set, uint32_t nsample, uint32_t* hits, cudaStream_t st);

// ---- join-ordering statistics (k_stats.cu) ----
// Open-addressing map from a key slot (u64) to a u64 value: keys[i] = ~0ull
// marks an empty slot; the key ~0ull itself keeps its value in vals[cap].
// cap = 1 << log2cap; keys has cap words, vals cap + 1.
struct KeyMap {
    unsigned long long* keys;
    unsigned long long* vals;
    uint32_t log2cap;
};
constexpr int kHistBins = 64;
int map_clear(const KeyMap& m, cudaStream_t st);
// Statistics of a join-key column (INT32 or INT64): hist[64] (zero before)
// counts non-null values by the top six bits of their key hash; m (cleared)
// receives key -> count; totals[0] += non-null values, totals[1] += distinct
// keys (both zero before).
int column_stats(const DevColumn& c, const KeyMap& m, uint32_t* hist, unsigned int* totals, uint32_t* err,
                 int num_sms, cudaStream_t st);
// One table of a sub-plan's exact count. For every row r: w = product over
// the children j of ch[j].map[value of ch[j].key at r] (0 when the value is
// NULL or absent); then, with has_out, out[value of pkey at r] += w (rows
// with a NULL pkey skipped), else *total += w. flags[0] |= 1 when a weight
// or the total passes 2^64 - 1.
constexpr int kMaxCountChildren = 12;
struct CountChild {
    DevColumn key;  // this table's column on the edge to the child
    KeyMap map;     // child's key -> weight
};
struct CountNode {
    CountChild ch[kMaxCountChildren];
    int nch;
    int has_out;
    DevColumn pkey;  // this table's column on the edge to its parent
    KeyMap out;
    uint32_t nrows;
    unsigned long long* total;
    unsigned int* flags;
};
int count_node(const CountNode& n, uint32_t* err, int num_sms, cudaStream_t st);
// Join samples: for directed edge d, hits[d] (zero before) = how many of
// nsample seeded rows of e[d].key have a non-null value present in e[d].map.
constexpr int kMaxSampleEdges = 24;
struct SampleEdge {
    DevColumn key;
    KeyMap map;
    uint32_t seed;
};
struct SampleEdges {
    SampleEdge e[kMaxSampleEdges];
    int n;
};
int sample_edges(const SampleEdges& e, uint32_t nsample, uint32_t* hits, cudaStream_t st);

// ---- learned cardinality estimator (k_mlp.cu) ----
// BF16 matrices are passed as raw 16-bit words. C (M x N) = A (M x K) B (K x N)
// on the tensor cores, FP32 accumulation; A(m, k) = A[m * a_rs + k * a_cs],
// B(k, n) = B[k * b_rs + n * b_cs], one stride of each being 1 and the other
// a multiple of 8. K must be a multiple of 32 and N of 64; an operand whose
// contiguous dimension is its rows (m for A, n for B) needs those rows a
// multiple of 8.
constexpr int kMlpHidden = 256;
enum GemmEpi : int {
    kEpiBiasRelu = 0,  // Cb = bf16(relu(acc + bias[n]))
    kEpiReluMask = 1,  // Cb = bf16(mask[m, n] > 0 ? acc : 0), mask laid out like C
    kEpiStoreF32 = 2,  // Cf = acc
};
struct GemmArgs {
    const uint16_t* A;
    long a_rs, a_cs;
    const uint16_t* B;
    long b_rs, b_cs;
    int M, N, K;
    int epi;
    const uint16_t* bias;
    const uint16_t* mask;
    uint16_t* Cb;
    float* Cf;
    long ldc;
};
int gemm_bf16(const GemmArgs& g, cudaStream_t st);
// Output layer (one CTA per row): y = H2 . w3 + b3; with targets t, loss +=
// (y - t)^2 and, for rows below n_real, dy = 2 (y - t) / n_real and dH2 =
// bf16(dy * w3 * [H2 > 0]) (zero for the other rows). Optional outputs may
// be null.
struct MlpHeadArgs {
    const uint16_t* H2;
    const uint16_t* w3;
    const uint16_t* b3;
    const float* t;
    float* y;
    float* loss;
    float* dy;
    uint16_t* dH2;
    int n_real;
};
int mlp_head(const MlpHeadArgs& a, int rows, cudaStream_t st);
// out[n] += sum over rows of X[m][n] (times dy[m] when dy is given).
int colsum(const uint16_t* X, const float* dy, int rows, int cols, float* out, cudaStream_t st);
int sum_f32(const float* v, int n, float* out, cudaStream_t st);
struct AdamArgs {
    float* w;
    uint16_t* wb;
    const float* grad;
    float* m;
    float* v;
    long n;
    float lr, beta1, beta2, eps, bc1, bc2;  // bc: 1 - beta^t
};
int adam_step(const AdamArgs& a, cudaStream_t st);
int f32_to_bf16(const float* in, uint16_t* out, long n, cudaStream_t st);
int gather_rows(const uint16_t* src, const float* tsrc, const uint32_t* idx, int n, int n_pad, int cols, uint16_t* dst,
                float* tdst, cudaStream_t st);

// ---- output pages (k_output.cu) ----
// Page descriptors of a VARCHAR column.
constexpr uint32_t kStrBlock = 4096;
struct StrPageDesc {
    uint64_t first_row;
    uint32_t nrows;     // rows on the page (1 for a long-string page)
    uint32_t chunk;     // long string: chunk index, else 0xffffffff
};
// Byte lengths and packing costs of the rows of every VARCHAR result column
// in one launch; stats (2 words per column, zero before): [0] largest cost,
// [1] 1 if some string is longer than PAGE_SIZE-7.
struct StrCol {
    const uint64_t* handles;  // string handles into src, or row numbers of src (see slot_value)
    uint64_t* resolved;       // non-null: handles are row numbers; their string handles go here
    const uint8_t* valid;
    // from_items: row i's value is computed here from item i (every item one
    // result row) instead of read from handles/valid, and stored to
    // vals_out (when not resolved) and valid_out.
    int from_items;
    SlotSource slot;
    uint64_t* vals_out;
    uint8_t* valid_out;
    DevColumn src;            // the source column the handles point into
    uint32_t* lens;
    uint64_t* cost;
    uint32_t* stats;
};
struct StrCols {
    StrCol c[kMaxOut];
    int n;
    Items items;  // from_items columns
    ProbeSet ps;
};
int string_len_cost(const StrCols& cols, uint64_t n, uint32_t* err, cudaStream_t st);
// Greedy page packing per block of kStrBlock rows: pass 0 counts pages per
// block, pass 1 writes page descriptors at block_page_off.
int string_pack(const uint32_t* lens, const uint8_t* valid, uint64_t n, int pass, uint32_t* block_pages,
                const uint32_t* block_page_off, StrPageDesc* descs, cudaStream_t st);
// Parallel packing: first row of each page from the exclusive scan `start`
// of the costs for page capacity cp, every floor-packed column in one launch.
constexpr uint64_t kStrPageUnits = 65496;  // eighth-bytes a page may hold
struct FloorCols {
    const uint64_t* start[kMaxOut];
    StrPageDesc* descs[kMaxOut];
    uint64_t cp[kMaxOut];
    int n;
};
int string_floor_first(const FloorCols& cols, uint64_t n, cudaStream_t st);
// Every page of the result in one launch: column k owns output pages
// [page_base, page_base + npages). Fixed width: rpp rows per page, values from
// vals/valid, or (direct) read from the items when each item is one output
// row. VARCHAR: pages from descs (floor: first rows only, row counts from the
// next page).
struct OutColumn {
    int32_t type;
    uint32_t floor;
    uint32_t direct;            // fixed width: values from `slot` of the items, not vals/valid
    SlotSource slot;
    const uint64_t* vals;       // values, or string handles into src
    const uint8_t* valid;
    const uint32_t* lens;       // VARCHAR
    const StrPageDesc* descs;   // VARCHAR
    DevColumn src;              // VARCHAR source column
    uint32_t rpp;               // fixed width: rows per page
    uint32_t page_base;
    uint32_t npages;
};
struct OutColumns {
    OutColumn c[kMaxOut];
    int n;
    uint64_t nrows;
    Items items;  // direct columns: item o is output row o
    ProbeSet ps;
    // CTA order (set by write_pages): fixed-width pages first, in rounds of
    // base_rpp rows (the smallest rows per page of those columns); round r
    // holds one CTA per fixed-width column, which writes that column's page
    // starting within the round's rows, if any. VARCHAR pages follow, column
    // by column.
    uint32_t nfixed;
    uint32_t base_rpp;
    uint32_t rounds;
    int32_t fixed_col[kMaxOut];
};
int write_pages(const OutColumns& cols, uint32_t total_pages, uint8_t* out_pages, uint32_t* err, cudaStream_t st);

} // namespace bj
