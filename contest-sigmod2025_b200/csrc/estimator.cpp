// Join ordering inputs (host side): key-column statistics of resident tables,
// exact sub-plan cardinalities, join-sample estimates, estimator features,
// and the learned cardinality estimator's training and inference.
//
// Reference counterparts: QueryPlan::computeSamples / recomputeCardinality
// (engine/query/QueryPlan.cpp:719-746, :67-72) and QueryGraph::computeCard
// (engine/query/QueryGraph.cpp:53-68) feed the join-order program
// QueryGraph::optimize (QueryGraph.cpp:107-216). The program here is the
// planner's (planner.cpp: choose_driver); this file supplies the set
// cardinalities it is given: the reference's row-count model, join samples,
// or the learned MLP (kernels in k_mlp.cu), with sampling as its fallback.
#include "engine.h"

#include <cmath>
#include <cstdio>
#include <random>

namespace bj {
namespace {

constexpr int kF = BJ_EST_FEATURES;
constexpr int kH = kMlpHidden;
constexpr int kMaxT = BJ_EST_MAX_TABLES;
constexpr long kOffW1 = 0;
constexpr long kOffB1 = kOffW1 + long(kF) * kH;
constexpr long kOffW2 = kOffB1 + kH;
constexpr long kOffB2 = kOffW2 + long(kH) * kH;
constexpr long kOffW3 = kOffB2 + kH;
constexpr long kOffB3 = kOffW3 + kH;
constexpr long kParams = kOffB3 + 8;  // b3 plus padding to 16 bytes
constexpr int kSlotFeatures = 5 + kMaxT + 2 * kHistBins;  // per table slot
static_assert(kSlotFeatures * kMaxT <= kF, "feature layout exceeds BJ_EST_FEATURES");
constexpr uint32_t kJoinSample = 64;  // rows per join sample (engine/query/QueryPlan.cpp:734)
constexpr uint32_t kMaxSubplanScans = 20;

#define EST_CK(call)                                                                                     \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw Fail{e_ == cudaErrorMemoryAllocation ? BJ_ERR_OOM : BJ_ERR_CUDA,                       \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};                              \
    } while (0)

uint16_t to_bf16(float f) {
    // Round to nearest even (NaN kept quiet).
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return uint16_t((u >> 16) | 0x40);
    u += 0x7fffu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}

// Device buffer freed with the owner.
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <typename T>
    T* alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        EST_CK(cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 256)));
        return static_cast<T*>(p);
    }
};

// Statistics of column c of a resident table, computed on first use.
ColStats& column_stats_of(bj_context* ctx, bj_resident* r, uint32_t c) {
    std::lock_guard<std::mutex> g(r->stats_m);
    if (c >= r->table.cols.size() || !r->table.present[c]) throw Fail{BJ_ERR_INVALID, "statistics of a missing column"};
    if (r->stats.size() < r->table.cols.size()) r->stats.resize(r->table.cols.size());
    ColStats& s = r->stats[c];
    if (s.ready) return s;
    const DevColumn& dc = r->table.cols[c];
    if (dc.type != kInt32 && dc.type != kInt64) throw Fail{BJ_ERR_UNSUPPORTED, "join keys must be INT32 or INT64"};
    const uint32_t log2cap = std::max<uint32_t>(4, bit_width(uint64_t(dc.nrows) * 2));
    s.map.log2cap = log2cap;
    s.map.keys = static_cast<unsigned long long*>(r->mem.alloc(sizeof(uint64_t) << log2cap));
    s.map.vals = static_cast<unsigned long long*>(r->mem.alloc(sizeof(uint64_t) * ((size_t(1) << log2cap) + 1)));
    struct Out {
        uint32_t hist[kHistBins];
        unsigned int totals[2];
    };
    Out* d = static_cast<Out*>(ctx->arena.alloc(sizeof(Out)));
    EST_CK(cudaMemsetAsync(d, 0, sizeof(Out), ctx->stream));
    EST_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
    ctx->launches += uint64_t(map_clear(s.map, ctx->stream));
    ctx->launches +=
        uint64_t(column_stats(dc, s.map, d->hist, d->totals, ctx->d_err, ctx->num_sms, ctx->stream));
    Out h{};
    uint32_t code = 0;
    EST_CK(cudaMemcpyAsync(&h, d, sizeof(Out), cudaMemcpyDeviceToHost, ctx->stream));
    EST_CK(cudaMemcpyAsync(&code, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    EST_CK(cudaStreamSynchronize(ctx->stream));
    if (code) throw Fail{BJ_ERR_INVALID, std::string("column statistics: ") + dev_error_text(code)};
    std::memcpy(s.hist, h.hist, sizeof(s.hist));
    s.nonnull = h.totals[0];
    s.distinct = h.totals[1];
    s.ready = true;
    return s;
}

// A plan's join graph with its resident tables.
struct Graph {
    PlanGraph g;
    std::vector<bj_resident*> res;  // per input
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> adj;  // per input: (neighbour, edge)

    void load(const bj_plan& plan, bj_resident* const* tables) {
        std::string err;
        int st = plan_graph(plan, g, err);
        if (st != BJ_OK) throw Fail{st, err};
        if (g.inputs.size() > kMaxSubplanScans) throw Fail{BJ_ERR_UNSUPPORTED, "sub-plans of more than 20 scans"};
        res.resize(g.inputs.size());
        for (size_t i = 0; i < g.inputs.size(); i++) {
            if (!tables || !tables[g.inputs[i].table]) throw Fail{BJ_ERR_INVALID, "missing resident table"};
            res[i] = tables[g.inputs[i].table];
        }
        adj.assign(g.inputs.size(), {});
        for (uint32_t e = 0; e < g.edges.size(); e++) {
            adj[g.edges[e].a].push_back({g.edges[e].b, e});
            adj[g.edges[e].b].push_back({g.edges[e].a, e});
        }
    }
    uint32_t n() const { return uint32_t(g.inputs.size()); }
    // Input x's column on edge e.
    uint32_t col(uint32_t x, uint32_t e) const { return g.edges[e].a == x ? g.edges[e].col_a : g.edges[e].col_b; }
    const DevColumn& dcol(uint32_t x, uint32_t e) const { return res[x]->table.cols[col(x, e)]; }
    bool connected(uint32_t mask) const {
        if (!mask) return false;
        uint32_t seen = mask & (~mask + 1), frontier = seen;
        while (frontier) {
            uint32_t next = 0;
            for (uint32_t f = frontier; f; f &= f - 1)
                for (auto [y, e] : adj[__builtin_ctz(f)]) next |= 1u << y;
            next &= mask & ~seen;
            seen |= next;
            frontier = next;
        }
        return seen == mask;
    }
    // The inputs of `mask` as a tree rooted at `root`: order (parents before
    // children), parent and parent edge per input (-1 for the root).
    void tree(uint32_t mask, uint32_t root, std::vector<uint32_t>& order, std::vector<int>& parent,
              std::vector<int>& pedge, bool larger_first) const {
        order.clear();
        parent.assign(n(), -1);
        pedge.assign(n(), -1);
        // Depth first, neighbours by descending rows (then index) when asked.
        // At most 32 inputs (masks are 32-bit), so fixed arrays hold the
        // stack and a node's children: no allocation per sub-plan.
        uint32_t stack[32];
        std::pair<uint32_t, uint32_t> kids[32];
        uint32_t top = 0;
        stack[top++] = root;
        uint32_t seen = 1u << root;
        while (top) {
            const uint32_t x = stack[--top];
            order.push_back(x);
            uint32_t nk = 0;
            for (auto [y, e] : adj[x])
                if ((mask >> y & 1) && !(seen >> y & 1)) kids[nk++] = {y, e};
            if (larger_first)
                std::sort(kids, kids + nk, [&](auto a, auto b) {
                    const uint64_t ra = g.inputs[a.first].rows, rb = g.inputs[b.first].rows;
                    return ra != rb ? ra > rb : a.first < b.first;
                });
            for (uint32_t i = nk; i-- > 0;) {
                seen |= 1u << kids[i].first;
                parent[kids[i].first] = int(x);
                pedge[kids[i].first] = int(kids[i].second);
                stack[top++] = kids[i].first;
            }
        }
    }
};

void enumerate_subplans(const Graph& G, uint32_t max_tables, std::vector<uint32_t>& out) {
    out.clear();
    const uint32_t full = (1u << G.n()) - 1;
    for (uint32_t m = 1; m <= full && m; m++)
        if (uint32_t(__builtin_popcount(m)) <= max_tables && G.connected(m)) out.push_back(m);
}

// Exact cardinalities of sub-plans (device counts by weights).
void exact_cards(bj_context* ctx, const Graph& G, const uint32_t* masks, uint64_t n, double* out) {
    DevBuf tot_buf;
    unsigned long long* tot = tot_buf.alloc<unsigned long long>(2 * n + 1);
    EST_CK(cudaMemsetAsync(tot, 0, sizeof(unsigned long long) * (2 * n + 1), ctx->stream));
    EST_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
    std::vector<uint32_t> order;
    std::vector<int> parent, pedge;
    std::vector<KeyMap> child_map(G.n());
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t mask = masks[i];
        if (!G.connected(mask)) throw Fail{BJ_ERR_INVALID, "sub-plan inputs are not connected"};
        const uint32_t root = __builtin_ctz(mask);
        G.tree(mask, root, order, parent, pedge, false);
        if (order.size() == 1) {
            out[i] = double(G.g.inputs[root].rows);  // a lone input: its rows
            continue;
        }
        // Children before parents.
        for (size_t oi = order.size(); oi-- > 0;) {
            const uint32_t x = order[oi];
            std::vector<std::pair<uint32_t, uint32_t>> kids;  // (child, edge)
            for (auto [y, e] : G.adj[x])
                if ((mask >> y & 1) && parent[y] == int(x)) kids.push_back({y, e});
            if (kids.empty()) {
                // A leaf: its key -> count map from the column statistics.
                child_map[x] = column_stats_of(ctx, G.res[x], G.col(x, uint32_t(pedge[x]))).map;
                continue;
            }
            if (kids.size() > size_t(kMaxCountChildren)) throw Fail{BJ_ERR_UNSUPPORTED, "a table with too many joins"};
            CountNode nd{};
            nd.nch = int(kids.size());
            for (size_t j = 0; j < kids.size(); j++) {
                nd.ch[j].key = G.dcol(x, kids[j].second);
                nd.ch[j].map = child_map[kids[j].first];
            }
            nd.nrows = uint32_t(G.g.inputs[x].rows);
            nd.flags = reinterpret_cast<unsigned int*>(tot + n + i);
            if (x == root) {
                nd.has_out = 0;
                nd.total = tot + i;
            } else {
                nd.has_out = 1;
                const uint32_t pc = G.col(x, uint32_t(pedge[x]));
                nd.pkey = G.res[x]->table.cols[pc];
                const ColStats& ps = column_stats_of(ctx, G.res[x], pc);
                const uint64_t keys = std::max<uint64_t>(1, std::min<uint64_t>(nd.nrows, ps.distinct + 1));
                KeyMap m{};
                m.log2cap = std::max<uint32_t>(4, bit_width(keys * 2));
                m.keys = static_cast<unsigned long long*>(ctx->arena.alloc(sizeof(uint64_t) << m.log2cap));
                m.vals = static_cast<unsigned long long*>(ctx->arena.alloc(sizeof(uint64_t) * ((size_t(1) << m.log2cap) + 1)));
                ctx->launches += uint64_t(map_clear(m, ctx->stream));
                nd.out = m;
                child_map[x] = m;
            }
            ctx->launches += uint64_t(count_node(nd, ctx->d_err, ctx->num_sms, ctx->stream));
        }
        // The maps of this sub-plan are dead once its kernels ran; the next
        // sub-plan's (stream-ordered after them) may reuse the arena.
        ctx->arena.reset();
    }
    std::vector<unsigned long long> h(2 * n);
    uint32_t code = 0;
    EST_CK(cudaMemcpyAsync(h.data(), tot, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost, ctx->stream));
    EST_CK(cudaMemcpyAsync(&code, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    EST_CK(cudaStreamSynchronize(ctx->stream));
    if (code) throw Fail{BJ_ERR_INVALID, std::string("sub-plan count: ") + dev_error_text(code)};
    for (uint64_t i = 0; i < n; i++) {
        if (__builtin_popcount(masks[i]) == 1) continue;
        out[i] = h[n + i] ? INFINITY : double(h[i]);
    }
}

// Join-sample selectivities of every directed edge: sel[2e] for a -> b (rows
// of a whose key b holds), sel[2e + 1] for b -> a.
std::vector<double> edge_samples(bj_context* ctx, const Graph& G) {
    const size_t ne = G.g.edges.size();
    std::vector<double> sel(2 * ne, 1.0);
    if (!ne) return sel;
    uint32_t* hits = static_cast<uint32_t*>(ctx->arena.alloc(sizeof(uint32_t) * 2 * ne));
    EST_CK(cudaMemsetAsync(hits, 0, sizeof(uint32_t) * 2 * ne, ctx->stream));
    std::vector<uint32_t> nsample(2 * ne);
    for (size_t e0 = 0; e0 < 2 * ne; e0 += kMaxSampleEdges) {
        SampleEdges se{};
        for (size_t d = e0; d < std::min(2 * ne, e0 + kMaxSampleEdges); d++) {
            const PlanGraph::Edge& e = G.g.edges[d / 2];
            const uint32_t src = d % 2 ? e.b : e.a, dst = d % 2 ? e.a : e.b;
            SampleEdge& s = se.e[se.n++];
            s.key = G.dcol(src, uint32_t(d / 2));
            s.map = column_stats_of(ctx, G.res[dst], G.col(dst, uint32_t(d / 2))).map;
            s.seed = uint32_t(d);
            nsample[d] = uint32_t(std::min<uint64_t>(kJoinSample, G.g.inputs[src].rows));
        }
        ctx->launches += uint64_t(sample_edges(se, kJoinSample, hits + e0, ctx->stream));
    }
    std::vector<uint32_t> h(2 * ne);
    EST_CK(cudaMemcpyAsync(h.data(), hits, sizeof(uint32_t) * 2 * ne, cudaMemcpyDeviceToHost, ctx->stream));
    EST_CK(cudaStreamSynchronize(ctx->stream));
    for (size_t d = 0; d < 2 * ne; d++) {
        // The kernel draws kJoinSample rows (with repetition on small inputs).
        sel[d] = h[d] ? double(h[d]) / kJoinSample : 1.0 / (2 * kJoinSample);
    }
    return sel;
}

// Sampling estimate of a connected set: its largest member's rows times the
// share of its sampled rows matching each neighbour in the set.
double sample_card(const Graph& G, const std::vector<double>& sel, uint32_t mask) {
    double best = 0;
    for (uint32_t m = mask; m; m &= m - 1) {
        const uint32_t i = __builtin_ctz(m);
        double c = double(G.g.inputs[i].rows);
        for (auto [y, e] : G.adj[i])
            if (mask >> y & 1) c *= sel[2 * e + (G.g.edges[e].a == i ? 0 : 1)];
        best = std::max(best, c);
    }
    return best;
}

float log_feature(double x) { return float(std::log2(x + 1.0) / 32.0); }

// A feature value as stored: FP32 for the public feature API and training,
// BF16 bits for inference (the device rounds to BF16 anyway).
inline void put_feature(float* f, size_t i, float v) { f[i] = v; }
inline void put_feature(uint16_t* f, size_t i, float v) { f[i] = to_bf16(v); }

// Feature row of one sub-plan (layout in include/b200join.h); T is float or
// BF16 bits (uint16_t). Every entry not written here is zero.
template <typename T>
void subplan_features_t(bj_context* ctx, const Graph& G, uint32_t mask, T* f) {
    std::fill(f, f + kF, T(0));
    if (__builtin_popcount(mask) > kMaxT) throw Fail{BJ_ERR_UNSUPPORTED, "sub-plan larger than the estimator's"};
    uint32_t root = __builtin_ctz(mask);
    for (uint32_t m = mask; m; m &= m - 1) {
        const uint32_t i = __builtin_ctz(m);
        if (G.g.inputs[i].rows > G.g.inputs[root].rows) root = i;
    }
    // Reused across calls (one thread plans one query at a time).
    thread_local std::vector<uint32_t> order;
    thread_local std::vector<int> parent, pedge, slot;
    G.tree(mask, root, order, parent, pedge, true);
    slot.assign(G.n(), -1);
    for (size_t k = 0; k < order.size(); k++) slot[order[k]] = int(k);
    for (size_t k = 0; k < order.size(); k++) {
        const uint32_t x = order[k];
        T* s = f + k * kSlotFeatures;
        const bj_resident* r = G.res[x];
        const double rows = double(G.g.inputs[x].rows);
        const double base = r->base_rows ? double(r->base_rows) : rows;
        put_feature(s, 0, 1.f);
        put_feature(s, 1, log_feature(rows));
        put_feature(s, 2, float(base > 0 ? std::min(1.0, rows / base) : 1.0));
        if (parent[x] < 0) continue;
        const uint32_t e = uint32_t(pedge[x]), p = uint32_t(parent[x]);
        const ColStats& own = column_stats_of(ctx, G.res[x], G.col(x, e));
        const ColStats& par = column_stats_of(ctx, G.res[p], G.col(p, e));
        put_feature(s, 3, log_feature(double(own.distinct)));
        put_feature(s, 4, log_feature(double(par.distinct)));
        put_feature(s, 5 + size_t(slot[p]), 1.f);
        for (int b = 0; b < kHistBins; b++) {
            put_feature(s, 5 + kMaxT + b, log_feature(own.hist[b]));
            put_feature(s, 5 + kMaxT + kHistBins + b, log_feature(par.hist[b]));
        }
    }
}

void subplan_features(bj_context* ctx, const Graph& G, uint32_t mask, float* f) {
    subplan_features_t(ctx, G, mask, f);
}

} // namespace

} // namespace bj

struct bj_estimator {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex m;
    bj::DevBuf w, wb, mo, vo, grad;  // fp32 master, bf16 copy, Adam moments, gradient
    long step = 0;
    // Batch scratch for up to cap rows.
    int cap = 0;
    bj::DevBuf X, H1, H2, dH2, dH1, y, t, dy, loss, idx;

    // Pinned BF16 feature rows for inference (kPredictChunk of them).
    uint16_t* hx = nullptr;

    ~bj_estimator() {
        if (stream) cudaStreamSynchronize(stream);
        if (hx) cudaFreeHost(hx);
        if (stream) cudaStreamDestroy(stream);
    }
    float* W() { return static_cast<float*>(w.p); }
    uint16_t* WB() { return static_cast<uint16_t*>(wb.p); }
    float* G() { return static_cast<float*>(grad.p); }

    void reserve(int rows) {
        if (rows <= cap) return;
        using namespace bj;
        X.alloc<uint16_t>(size_t(rows) * kF);
        H1.alloc<uint16_t>(size_t(rows) * kH);
        H2.alloc<uint16_t>(size_t(rows) * kH);
        dH2.alloc<uint16_t>(size_t(rows) * kH);
        dH1.alloc<uint16_t>(size_t(rows) * kH);
        y.alloc<float>(rows);
        t.alloc<float>(rows);
        dy.alloc<float>(rows);
        loss.alloc<float>(4);
        idx.alloc<uint32_t>(rows);
        cap = rows;
    }

    // Forward over n_pad rows of X (a multiple of 64); outputs y.
    void forward(int n_pad) {
        using namespace bj;
        GemmArgs g{};
        g.A = static_cast<uint16_t*>(X.p);
        g.a_rs = kF;
        g.a_cs = 1;
        g.B = WB() + kOffW1;
        g.b_rs = kH;
        g.b_cs = 1;
        g.M = n_pad;
        g.N = kH;
        g.K = kF;
        g.epi = kEpiBiasRelu;
        g.bias = WB() + kOffB1;
        g.Cb = static_cast<uint16_t*>(H1.p);
        g.ldc = kH;
        gemm_bf16(g, stream);
        g.A = static_cast<uint16_t*>(H1.p);
        g.a_rs = kH;
        g.B = WB() + kOffW2;
        g.K = kH;
        g.bias = WB() + kOffB2;
        g.Cb = static_cast<uint16_t*>(H2.p);
        gemm_bf16(g, stream);
    }

    // Forward, loss and gradients over a batch of n_real rows (padded to
    // n_pad) whose features are in X and targets in t.
    void forward_backward(int n_real, int n_pad) {
        using namespace bj;
        forward(n_pad);
        EST_CK(cudaMemsetAsync(grad.p, 0, sizeof(float) * kParams, stream));
        MlpHeadArgs h{};
        h.H2 = static_cast<uint16_t*>(H2.p);
        h.w3 = WB() + kOffW3;
        h.b3 = WB() + kOffB3;
        h.t = static_cast<float*>(t.p);
        h.y = static_cast<float*>(y.p);
        h.loss = static_cast<float*>(loss.p);
        h.dy = static_cast<float*>(dy.p);
        h.dH2 = static_cast<uint16_t*>(dH2.p);
        h.n_real = n_real;
        mlp_head(h, n_pad, stream);
        GemmArgs g{};
        // dW2 = H1^T dH2
        g.A = static_cast<uint16_t*>(H1.p);
        g.a_rs = 1;
        g.a_cs = kH;
        g.B = static_cast<uint16_t*>(dH2.p);
        g.b_rs = kH;
        g.b_cs = 1;
        g.M = kH;
        g.N = kH;
        g.K = n_pad;
        g.epi = kEpiStoreF32;
        g.Cf = G() + kOffW2;
        g.ldc = kH;
        gemm_bf16(g, stream);
        colsum(static_cast<uint16_t*>(dH2.p), nullptr, n_pad, kH, G() + kOffB2, stream);
        colsum(static_cast<uint16_t*>(H2.p), static_cast<float*>(dy.p), n_pad, kH, G() + kOffW3, stream);
        sum_f32(static_cast<float*>(dy.p), n_pad, G() + kOffB3, stream);
        // dH1 = (dH2 W2^T) * [H1 > 0]
        g = GemmArgs{};
        g.A = static_cast<uint16_t*>(dH2.p);
        g.a_rs = kH;
        g.a_cs = 1;
        g.B = WB() + kOffW2;
        g.b_rs = 1;
        g.b_cs = kH;
        g.M = n_pad;
        g.N = kH;
        g.K = kH;
        g.epi = kEpiReluMask;
        g.mask = static_cast<uint16_t*>(H1.p);
        g.Cb = static_cast<uint16_t*>(dH1.p);
        g.ldc = kH;
        gemm_bf16(g, stream);
        // dW1 = X^T dH1
        g = GemmArgs{};
        g.A = static_cast<uint16_t*>(X.p);
        g.a_rs = 1;
        g.a_cs = kF;
        g.B = static_cast<uint16_t*>(dH1.p);
        g.b_rs = kH;
        g.b_cs = 1;
        g.M = kF;
        g.N = kH;
        g.K = n_pad;
        g.epi = kEpiStoreF32;
        g.Cf = G() + kOffW1;
        g.ldc = kH;
        gemm_bf16(g, stream);
        colsum(static_cast<uint16_t*>(dH1.p), nullptr, n_pad, kH, G() + kOffB1, stream);
    }

    void adam(float lr) {
        using namespace bj;
        step++;
        AdamArgs a{};
        a.w = W();
        a.wb = WB();
        a.grad = G();
        a.m = static_cast<float*>(mo.p);
        a.v = static_cast<float*>(vo.p);
        a.n = kParams;
        a.lr = lr;
        a.beta1 = 0.9f;
        a.beta2 = 0.999f;
        a.eps = 1e-8f;
        a.bc1 = float(1.0 - std::pow(0.9, double(step)));
        a.bc2 = float(1.0 - std::pow(0.999, double(step)));
        adam_step(a, stream);
    }

    void upload_params(const std::vector<float>& p) {
        using namespace bj;
        EST_CK(cudaMemcpyAsync(W(), p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, stream));
        f32_to_bf16(W(), WB(), kParams, stream);
        EST_CK(cudaMemsetAsync(mo.p, 0, sizeof(float) * kParams, stream));
        EST_CK(cudaMemsetAsync(vo.p, 0, sizeof(float) * kParams, stream));
        EST_CK(cudaStreamSynchronize(stream));
        step = 0;
    }

    // Uploads n feature rows (f32 host, rounded to bf16) into X, padded with
    // zero rows to n_pad.
    void upload_features(const float* f, uint64_t n, int n_pad) {
        using namespace bj;
        std::vector<uint16_t> hb(size_t(n_pad) * kF, 0);
        for (size_t i = 0; i < size_t(n) * kF; i++) hb[i] = to_bf16(f[i]);
        EST_CK(cudaMemcpyAsync(X.p, hb.data(), hb.size() * 2, cudaMemcpyHostToDevice, stream));
        EST_CK(cudaStreamSynchronize(stream));
    }

    static constexpr int kPredictChunk = 4096;

    // Predictions for n rows whose BF16 features fill(i0, rows, dst) writes
    // into pinned staging (rows i0 .. i0 + rows - 1, row-major, kF each): one
    // copy per chunk straight from there, no FP32 rows and no conversion pass.
    template <typename Fill>
    void predict_rows(uint64_t n, float* out, Fill&& fill) {
        using namespace bj;
        reserve(kPredictChunk);
        if (!hx) {
            void* p = nullptr;
            EST_CK(cudaHostAlloc(&p, sizeof(uint16_t) * size_t(kPredictChunk) * kF, cudaHostAllocDefault));
            hx = static_cast<uint16_t*>(p);
        }
        for (uint64_t i0 = 0; i0 < n; i0 += kPredictChunk) {
            const int rows = int(std::min<uint64_t>(kPredictChunk, n - i0));
            const int pad = (rows + 63) & ~63;
            fill(i0, rows, hx);
            std::memset(hx + size_t(rows) * kF, 0, sizeof(uint16_t) * size_t(pad - rows) * kF);
            EST_CK(cudaMemcpyAsync(X.p, hx, sizeof(uint16_t) * size_t(pad) * kF, cudaMemcpyHostToDevice, stream));
            run_head(pad, rows, out + i0);
        }
    }

    // Forward and head over the pad rows in X; the first `rows` predictions to out.
    void run_head(int pad, int rows, float* out) {
        using namespace bj;
        forward(pad);
        MlpHeadArgs h{};
        h.H2 = static_cast<uint16_t*>(H2.p);
        h.w3 = WB() + kOffW3;
        h.b3 = WB() + kOffB3;
        h.y = static_cast<float*>(y.p);
        mlp_head(h, rows, stream);
        EST_CK(cudaMemcpyAsync(out, y.p, sizeof(float) * rows, cudaMemcpyDeviceToHost, stream));
        EST_CK(cudaStreamSynchronize(stream));
    }

    void predict(const float* f, uint64_t n, float* out) {
        using namespace bj;
        constexpr int kChunk = kPredictChunk;
        reserve(kChunk);
        for (uint64_t i0 = 0; i0 < n; i0 += kChunk) {
            const int rows = int(std::min<uint64_t>(kChunk, n - i0));
            const int pad = (rows + 63) & ~63;
            upload_features(f + i0 * kF, rows, pad);
            forward(pad);
            MlpHeadArgs h{};
            h.H2 = static_cast<uint16_t*>(H2.p);
            h.w3 = WB() + kOffW3;
            h.b3 = WB() + kOffB3;
            h.y = static_cast<float*>(y.p);
            mlp_head(h, rows, stream);
            EST_CK(cudaMemcpyAsync(out + i0, y.p, sizeof(float) * rows, cudaMemcpyDeviceToHost, stream));
            EST_CK(cudaStreamSynchronize(stream));
        }
    }
};

namespace bj {

void estimate_set_cards(bj_context* ctx, const bj_plan& plan, bj_resident* const* tables, std::vector<double>& cards) {
    cards.clear();
    if (ctx->ordering == BJ_ORDER_ROWS) return;
    Graph G;
    G.load(plan, tables);
    const uint32_t n = G.n();
    if (n < 2 || n > 14) return;  // the join-order program costs up to 14 inputs
    for (uint32_t i = 0; i < n; i++)
        if (G.g.inputs[i].rows == 0) return;  // empty result: nothing to order
    for (const PlanGraph::Edge& e : G.g.edges)
        if (e.type != BJ_INT32 && e.type != BJ_INT64) return;
    cards.assign(size_t(1) << n, 0.0);
    const std::vector<double> sel = edge_samples(ctx, G);
    std::vector<uint32_t> masks;
    enumerate_subplans(G, n, masks);
    for (uint32_t m : masks) cards[m] = sample_card(G, sel, m);
    if (ctx->ordering == BJ_ORDER_LEARNED && ctx->estimator && n <= uint32_t(kMaxT)) {
        std::vector<uint32_t> multi;
        for (uint32_t m : masks)
            if (__builtin_popcount(m) > 1) multi.push_back(m);
        std::vector<float> y(multi.size());
        {
            std::lock_guard<std::mutex> g(ctx->estimator->m);
            cudaSetDevice(ctx->estimator->device);
            ctx->estimator->predict_rows(multi.size(), y.data(), [&](uint64_t i0, int rows, uint16_t* dst) {
                for (int i = 0; i < rows; i++) subplan_features_t(ctx, G, multi[i0 + i], dst + size_t(i) * kF);
            });
        }
        for (size_t i = 0; i < multi.size(); i++) {
            const double c = std::exp2(double(y[i])) - 1.0;
            if (std::isfinite(c)) cards[multi[i]] = std::max(0.0, c);  // else: the sampling estimate stays
        }
    }
    ctx->arena.reset();
}

} // namespace bj

using namespace bj;

extern "C" {

BJ_API int bj_context_set_ordering(bj_context* ctx, int mode, bj_estimator* estimator) {
    if (!ctx || mode < BJ_ORDER_ROWS || mode > BJ_ORDER_LEARNED) return BJ_ERR_INVALID;
    if (mode == BJ_ORDER_LEARNED && !estimator) return BJ_ERR_INVALID;
    ctx->ordering = mode;
    ctx->estimator = estimator;
    return BJ_OK;
}

BJ_API int bj_resident_set_base_rows(bj_resident* table, uint64_t base_rows) {
    if (!table) return BJ_ERR_INVALID;
    table->base_rows = base_rows;
    return BJ_OK;
}

BJ_API int bj_subplans(const bj_plan* plan, uint32_t max_tables, uint64_t cap, uint32_t* masks, uint64_t* n) {
    if (!plan || !n || (cap && !masks)) return BJ_ERR_INVALID;
    PlanGraph pg;
    std::string err;
    int st = plan_graph(*plan, pg, err);
    if (st != BJ_OK) return st;
    if (pg.inputs.size() > kMaxSubplanScans) return BJ_ERR_UNSUPPORTED;
    Graph G;
    G.g = pg;
    G.adj.assign(pg.inputs.size(), {});
    for (uint32_t e = 0; e < pg.edges.size(); e++) {
        G.adj[pg.edges[e].a].push_back({pg.edges[e].b, e});
        G.adj[pg.edges[e].b].push_back({pg.edges[e].a, e});
    }
    std::vector<uint32_t> all;
    enumerate_subplans(G, max_tables, all);
    for (uint64_t i = 0; i < std::min<uint64_t>(cap, all.size()); i++) masks[i] = all[i];
    *n = all.size();
    return BJ_OK;
}

BJ_API int bj_subplan_cards(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, const uint32_t* masks,
                            uint64_t n, double* out) {
    if (!ctx || !plan || (n && (!masks || !out))) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    try {
        Graph G;
        G.load(*plan, tables);
        for (uint64_t i = 0; i < n; i++)
            if (masks[i] >> G.n()) throw Fail{BJ_ERR_INVALID, "sub-plan mask beyond the plan's scans"};
        exact_cards(ctx, G, masks, n, out);
        ctx->arena.reset();
    } catch (const Fail& f) {
        return fail_to_status(ctx, f);
    }
    return BJ_OK;
}

BJ_API int bj_subplan_sample_cards(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables,
                                   const uint32_t* masks, uint64_t n, double* out) {
    if (!ctx || !plan || (n && (!masks || !out))) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    try {
        Graph G;
        G.load(*plan, tables);
        const std::vector<double> sel = edge_samples(ctx, G);
        for (uint64_t i = 0; i < n; i++) {
            if (masks[i] >> G.n() || !G.connected(masks[i]))
                throw Fail{BJ_ERR_INVALID, "sub-plan mask beyond the plan's scans or not connected"};
            out[i] = sample_card(G, sel, masks[i]);
        }
        ctx->arena.reset();
    } catch (const Fail& f) {
        return fail_to_status(ctx, f);
    }
    return BJ_OK;
}

BJ_API int bj_subplan_features(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, const uint32_t* masks,
                               uint64_t n, float* out) {
    if (!ctx || !plan || (n && (!masks || !out))) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    try {
        Graph G;
        G.load(*plan, tables);
        for (uint64_t i = 0; i < n; i++) {
            if (masks[i] >> G.n() || !G.connected(masks[i]))
                throw Fail{BJ_ERR_INVALID, "sub-plan mask beyond the plan's scans or not connected"};
            subplan_features(ctx, G, masks[i], out + i * kF);
        }
        ctx->arena.reset();
    } catch (const Fail& f) {
        return fail_to_status(ctx, f);
    }
    return BJ_OK;
}

BJ_API int bj_join_order(const bj_plan* plan, const double* card, int driver_in, uint32_t* driver, double* cost) {
    if (!plan || !driver || !cost) return BJ_ERR_INVALID;
    PlanGraph pg;
    std::string err;
    int st = plan_graph(*plan, pg, err);
    if (st != BJ_OK) return st;
    if (pg.inputs.size() > 14) return BJ_ERR_UNSUPPORTED;
    if (driver_in >= int(pg.inputs.size())) return BJ_ERR_INVALID;
    std::vector<double> cards;
    if (card) cards.assign(card, card + (size_t(1) << pg.inputs.size()));
    return join_order(*plan, card ? &cards : nullptr, driver_in, *driver, *cost, err);
}

BJ_API int bj_plan_scratch_estimate(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables,
                                    uint64_t* bytes) {
    if (!ctx || !plan || !tables || !bytes) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    try {
        // Cardinalities: the context's estimator, or join samples when the
        // context orders by row counts (which say nothing about sizes).
        std::vector<double> cards;
        const int mode = ctx->ordering;
        if (mode == BJ_ORDER_ROWS) ctx->ordering = BJ_ORDER_SAMPLING;
        try {
            estimate_set_cards(ctx, *plan, tables, cards);
        } catch (...) {
            ctx->ordering = mode;
            throw;
        }
        ctx->ordering = mode;
        ExecPlan ex;
        std::string err;
        const int st = make_exec_plan(*plan, ex, err, false, cards.empty() ? nullptr : &cards);
        if (st != BJ_OK) throw Fail{st, err};
        if (ex.empty) {
            *bytes = 0;
            return BJ_OK;
        }
        auto card = [&](uint32_t m) {
            if (!cards.empty()) return cards[m];
            double c = 0;  // the row-count model: the largest input
            for (uint32_t i = 0; i < ex.inputs.size(); i++)
                if (m >> i & 1) c = std::max(c, double(ex.inputs[i].rows));
            return c;
        };
        // Pipelines run children first: each one's input set is its own input
        // plus its children's.
        std::vector<uint32_t> sub(ex.pipelines.size(), 0);
        double total = 0;
        for (size_t p = 0; p < ex.pipelines.size(); p++) {
            const PipelinePlan& pp = ex.pipelines[p];
            sub[p] = 1u << pp.input;
            for (const auto& pr : pp.probes) sub[p] |= sub[pr.child];
            const double n = card(sub[p]);
            const double w = double(pp.slots.size());
            total += 2.0 * n * (12.0 + 4.0 * double(pp.probes.size()));  // items in and out of the stages
            if (pp.build_key >= 0) {
                // tuples and table entries (key, mult, payload, NULL mask,
                // representative flag), buckets, aggregation slots
                total += n * (2.0 * (20.0 + 8.0 * w) + 8.0) + 16.0 * std::exp2(double(bit_width(uint64_t(n) + 1)));
            } else {
                total += n * 17.0 * double(ex.out_slot.size());  // flat values + result pages
            }
        }
        *bytes = uint64_t(std::min(total, 1.8e19));
        ctx->arena.reset();
    } catch (const Fail& f) {
        return fail_to_status(ctx, f);
    }
    return BJ_OK;
}

BJ_API uint64_t bj_estimator_num_params(void) { return uint64_t(kParams); }

BJ_API int bj_estimator_create(int device, uint64_t seed, bj_estimator** out) {
    if (!out) return BJ_ERR_INVALID;
    *out = nullptr;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || device < 0 || device >= nd) {
        cudaGetLastError();
        return BJ_ERR_NO_DEVICE;
    }
    try {
        cudaSetDevice(device);
        auto e = std::make_unique<bj_estimator>();
        e->device = device;
        EST_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->w.alloc<float>(kParams);
        e->wb.alloc<uint16_t>(kParams);
        e->mo.alloc<float>(kParams);
        e->vo.alloc<float>(kParams);
        e->grad.alloc<float>(kParams);
        // He-uniform weights (ReLU layers), zero biases.
        std::vector<float> p(kParams, 0.f);
        std::mt19937_64 rng(seed);
        auto fill = [&](long off, long n, int fan_in) {
            const float lim = std::sqrt(6.0f / float(fan_in));
            std::uniform_real_distribution<float> u(-lim, lim);
            for (long i = 0; i < n; i++) p[off + i] = u(rng);
        };
        fill(kOffW1, long(kF) * kH, kF);
        fill(kOffW2, long(kH) * kH, kH);
        fill(kOffW3, kH, kH);
        e->upload_params(p);
        *out = e.release();
        return BJ_OK;
    } catch (const Fail&) {
        cudaGetLastError();
        return BJ_ERR_CUDA;
    }
}

BJ_API void bj_estimator_destroy(bj_estimator* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete e;
}

BJ_API int bj_estimator_get_params(bj_estimator* e, float* out) {
    if (!e || !out) return BJ_ERR_INVALID;
    std::lock_guard<std::mutex> g(e->m);
    cudaSetDevice(e->device);
    if (cudaMemcpy(out, e->W(), sizeof(float) * kParams, cudaMemcpyDeviceToHost) != cudaSuccess) return BJ_ERR_CUDA;
    return BJ_OK;
}

BJ_API int bj_estimator_set_params(bj_estimator* e, const float* in) {
    if (!e || !in) return BJ_ERR_INVALID;
    std::lock_guard<std::mutex> g(e->m);
    cudaSetDevice(e->device);
    try {
        e->upload_params(std::vector<float>(in, in + kParams));
    } catch (const Fail&) {
        return BJ_ERR_CUDA;
    }
    return BJ_OK;
}

BJ_API int bj_estimator_train(bj_estimator* e, const float* features, const float* targets, uint64_t n,
                              uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* epoch_loss) {
    if (!e || !features || !targets || n == 0 || batch == 0 || batch > 8192 || n > (1ull << 24))
        return BJ_ERR_INVALID;
    for (uint64_t i = 0; i < n; i++)
        if (!std::isfinite(targets[i])) return BJ_ERR_INVALID;  // a NaN or infinite label would poison the fit
    std::lock_guard<std::mutex> g(e->m);
    cudaSetDevice(e->device);
    try {
        // The training set stays on the device as bf16 rows.
        DevBuf xall, tall;
        uint16_t* X = xall.alloc<uint16_t>(n * kF);
        float* T = tall.alloc<float>(n);
        {
            std::vector<uint16_t> hb(n * kF);
            for (size_t i = 0; i < n * kF; i++) hb[i] = to_bf16(features[i]);
            EST_CK(cudaMemcpyAsync(X, hb.data(), hb.size() * 2, cudaMemcpyHostToDevice, e->stream));
            EST_CK(cudaMemcpyAsync(T, targets, sizeof(float) * n, cudaMemcpyHostToDevice, e->stream));
            EST_CK(cudaStreamSynchronize(e->stream));
        }
        // Output bias starts at the mean target.
        double mean = 0;
        for (uint64_t i = 0; i < n; i++) mean += targets[i];
        mean /= double(n);
        std::vector<float> p(kParams);
        EST_CK(cudaMemcpy(p.data(), e->W(), sizeof(float) * kParams, cudaMemcpyDeviceToHost));
        if (e->step == 0) {
            p[kOffB3] = float(mean);
            e->upload_params(p);
        }
        const int bpad = int((batch + 63) & ~63u);
        e->reserve(bpad);
        DevBuf perm_buf;
        uint32_t* perm = perm_buf.alloc<uint32_t>(n);
        std::vector<uint32_t> order(n);
        std::iota(order.begin(), order.end(), 0u);
        std::mt19937_64 rng(seed);
        const uint64_t steps_per_epoch = (n + batch - 1) / batch;
        const double total = double(steps_per_epoch) * epochs;
        uint64_t done = 0;
        for (uint32_t ep = 0; ep < epochs; ep++) {
            std::shuffle(order.begin(), order.end(), rng);
            EST_CK(cudaMemcpyAsync(perm, order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, e->stream));
            EST_CK(cudaMemsetAsync(e->loss.p, 0, sizeof(float), e->stream));
            for (uint64_t b0 = 0; b0 < n; b0 += batch) {
                const int rows = int(std::min<uint64_t>(batch, n - b0));
                const int pad = (rows + 63) & ~63;
                gather_rows(X, T, perm + b0, rows, pad, kF, static_cast<uint16_t*>(e->X.p), static_cast<float*>(e->t.p),
                            e->stream);
                e->forward_backward(rows, pad);
                // Cosine decay from lr to lr / 10.
                const double frac = double(done++) / std::max(1.0, total);
                e->adam(float(lr * (0.1 + 0.9 * 0.5 * (1.0 + std::cos(M_PI * frac)))));
            }
            float l = 0;
            EST_CK(cudaMemcpyAsync(&l, e->loss.p, sizeof(float), cudaMemcpyDeviceToHost, e->stream));
            EST_CK(cudaStreamSynchronize(e->stream));
            if (epoch_loss) epoch_loss[ep] = l / float(n);
        }
    } catch (const Fail&) {
        cudaGetLastError();
        return BJ_ERR_CUDA;
    }
    return BJ_OK;
}

BJ_API int bj_estimator_predict(bj_estimator* e, const float* features, uint64_t n, float* out) {
    if (!e || (n && (!features || !out))) return BJ_ERR_INVALID;
    std::lock_guard<std::mutex> g(e->m);
    cudaSetDevice(e->device);
    try {
        e->predict(features, n, out);
    } catch (const Fail&) {
        cudaGetLastError();
        return BJ_ERR_CUDA;
    }
    return BJ_OK;
}

BJ_API int bj_estimator_gradients(bj_estimator* e, const float* features, const float* targets, uint64_t n,
                                  float* loss, float* grads) {
    if (!e || !features || !targets || !loss || !grads || n == 0 || n > 4096) return BJ_ERR_INVALID;
    std::lock_guard<std::mutex> g(e->m);
    cudaSetDevice(e->device);
    try {
        const int pad = int((n + 63) & ~63ull);
        e->reserve(pad);
        e->upload_features(features, n, pad);
        std::vector<float> t(pad, 0.f);
        std::copy(targets, targets + n, t.begin());
        EST_CK(cudaMemcpyAsync(e->t.p, t.data(), sizeof(float) * pad, cudaMemcpyHostToDevice, e->stream));
        EST_CK(cudaMemsetAsync(e->loss.p, 0, sizeof(float), e->stream));
        e->forward_backward(int(n), pad);
        EST_CK(cudaMemcpyAsync(grads, e->G(), sizeof(float) * kParams, cudaMemcpyDeviceToHost, e->stream));
        EST_CK(cudaMemcpyAsync(loss, e->loss.p, sizeof(float), cudaMemcpyDeviceToHost, e->stream));
        EST_CK(cudaStreamSynchronize(e->stream));
        *loss /= float(n);
    } catch (const Fail&) {
        cudaGetLastError();
        return BJ_ERR_CUDA;
    }
    return BJ_OK;
}

namespace {
constexpr char kEstMagic[8] = {'B', 'J', 'M', 'L', 'P', '0', '0', '1'};
}

BJ_API int bj_estimator_save(bj_estimator* e, const char* path) {
    if (!e || !path) return BJ_ERR_INVALID;
    std::vector<float> p(kParams);
    int st = bj_estimator_get_params(e, p.data());
    if (st != BJ_OK) return st;
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return BJ_ERR_INVALID;
    const uint64_t np = kParams, nf = kF;
    bool ok = std::fwrite(kEstMagic, 1, 8, f) == 8 && std::fwrite(&nf, 8, 1, f) == 1 && std::fwrite(&np, 8, 1, f) == 1 &&
              std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? BJ_OK : BJ_ERR_INVALID;
}

BJ_API int bj_estimator_load(int device, const char* path, bj_estimator** out) {
    if (!path || !out) return BJ_ERR_INVALID;
    *out = nullptr;
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return BJ_ERR_INVALID;
    char magic[8];
    uint64_t nf = 0, np = 0;
    std::vector<float> p(kParams);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kEstMagic, 8) == 0 && std::fread(&nf, 8, 1, f) == 1 &&
              std::fread(&np, 8, 1, f) == 1 && nf == uint64_t(kF) && np == uint64_t(kParams) &&
              std::fread(p.data(), sizeof(float), p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) return BJ_ERR_INVALID;
    bj_estimator* e = nullptr;
    int st = bj_estimator_create(device, 0, &e);
    if (st != BJ_OK) return st;
    st = bj_estimator_set_params(e, p.data());
    if (st != BJ_OK) {
        bj_estimator_destroy(e);
        return st;
    }
    *out = e;
    return BJ_OK;
}

} // extern "C"
