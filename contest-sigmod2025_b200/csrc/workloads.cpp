// Seeded synthetic workloads for the join engine's tests and benchmark.
// See workloads.h for the shapes. All randomness comes from xoshiro256**
// streams seeded through splitmix64 (Blackman & Vigna), one stream per
// (seed, table, column, block) so generation is parallel and deterministic.
#include "workloads.h"

#include "../../include/contest/pages.h"
#include "../../include/contest/plan_io.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <memory>
#include <vector>

namespace {

uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (auto& v : s) v = splitmix64(seed);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    // Uniform in [0, n) by multiply-shift (Lemire); the tiny bias is irrelevant here.
    uint64_t below(uint64_t n) { return uint64_t((__uint128_t(next()) * n) >> 64); }
    double unit() { return double(next() >> 11) * 0x1.0p-53; }
};

uint64_t stream_seed(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t x = seed ^ (a * 0x100000001B3ull) ^ (b << 20) ^ (c << 40);
    splitmix64(x);
    return splitmix64(x);
}

template <typename Fn>
void parallel_for(size_t n, Fn&& fn) {
    size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 32));
    nt = std::min(nt, std::max<size_t>(n, 1));
    std::atomic<size_t> next{0};
    std::exception_ptr err;
    std::atomic<bool> failed{false};
    auto worker = [&] {
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= n || failed.load()) return;
            try {
                fn(i);
            } catch (...) {
                if (!failed.exchange(true)) err = std::current_exception();
            }
        }
    };
    std::vector<std::thread> ts;
    for (size_t t = 1; t < nt; t++) ts.emplace_back(worker);
    worker();
    for (auto& t : ts) t.join();
    if (err) std::rethrow_exception(err);
}

// Fisher-Yates shuffle of 0..n-1.
std::vector<int32_t> permutation(uint64_t n, uint64_t seed) {
    std::vector<int32_t> p(n);
    for (uint64_t i = 0; i < n; i++) p[i] = int32_t(i);
    Rng r(seed);
    for (uint64_t i = n; i > 1; i--) std::swap(p[i - 1], p[r.below(i)]);
    return p;
}

// Zipf(s) over ranks 1..n by rejection-inversion (W. Hörmann, G. Derflinger,
// "Rejection-inversion to generate variates from monotone discrete
// distributions", ACM TOMACS 6(3), 1996). Constant expected time per sample.
class Zipf {
    public:
    Zipf(uint64_t n, double s) : n_(double(n)), s_(s) {
        h_x1_ = H(1.5) - 1.0;
        h_n_ = H(n_ + 0.5);
        cut_ = 2.0 - Hinv(H(2.5) - h(2.0));
    }
    uint64_t sample(Rng& r) const {
        for (;;) {
            double u = h_n_ + r.unit() * (h_x1_ - h_n_);
            double x = Hinv(u);
            double k = std::floor(x + 0.5);
            if (k < 1) k = 1;
            if (k > n_) k = n_;
            if (k - x <= cut_ || u >= H(k + 0.5) - h(k)) return uint64_t(k);
        }
    }

    private:
    // log1p(x)/x and expm1(x)/x, continuous at 0.
    static double log1p_over(double x) { return std::fabs(x) > 1e-8 ? std::log1p(x) / x : 1.0 - x / 2.0; }
    static double expm1_over(double x) { return std::fabs(x) > 1e-8 ? std::expm1(x) / x : 1.0 + x / 2.0; }
    double h(double x) const { return std::exp(-s_ * std::log(x)); }
    // Antiderivative of h: (x^(1-s) - 1) / (1-s).
    double H(double x) const {
        double lx = std::log(x);
        return expm1_over((1.0 - s_) * lx) * lx;
    }
    double Hinv(double y) const {
        double t = y * (1.0 - s_);
        if (t < -1.0) t = -1.0;
        return std::exp(log1p_over(t) * y);
    }
    double n_, s_, h_x1_, h_n_, cut_;
};

struct PageBuf {
    std::vector<uint8_t> bytes;
    Page* alloc() {
        size_t off = bytes.size();
        bytes.resize(off + PAGE_SIZE);
        return reinterpret_cast<Page*>(bytes.data() + off);
    }
};

// Dense fixed-width column without NULLs: every page but the last is full, so
// pages are independent and encoded in parallel.
void encode_dense(plan_io::OwnedColumn& col, int32_t type, const void* values, uint64_t n) {
    size_t width = type == BJ_INT32 ? 4 : 8;
    size_t per = contest_pages::full_page_rows(width);
    size_t npages = (n + per - 1) / per;
    col.type = type;
    col.bytes.assign(npages * PAGE_SIZE, 0);
    const uint8_t* src = static_cast<const uint8_t*>(values);
    parallel_for((npages + 63) / 64, [&](size_t blk) {
        for (size_t p = blk * 64; p < std::min(npages, blk * 64 + 64); p++) {
            uint8_t* page = col.bytes.data() + p * PAGE_SIZE;
            size_t r0 = p * per, rows = std::min<size_t>(per, n - r0);
            uint16_t r16 = uint16_t(rows);
            std::memcpy(page, &r16, 2);
            std::memcpy(page + 2, &r16, 2);
            std::memcpy(page + contest_pages::value_begin(width), src + r0 * width, rows * width);
            size_t nb = (rows + 7) / 8;
            uint8_t* bm = page + PAGE_SIZE - nb;
            std::memset(bm, 0xff, nb);
            if (rows % 8) bm[nb - 1] = uint8_t((1u << (rows % 8)) - 1);
        }
    });
}

void encode_general(plan_io::OwnedColumn& col, int32_t type, uint64_t n, const void* values,
                    const uint8_t* valid, const uint64_t* str_off, const char* str_bytes) {
    PageBuf buf;
    auto alloc = [&buf] { return buf.alloc(); };
    col.type = type;
    if (type == BJ_VARCHAR) {
        contest_pages::StringWriter w(alloc);
        for (uint64_t i = 0; i < n; i++) {
            if (valid && !valid[i])
                w.append_null();
            else
                w.append(std::string_view(str_bytes + str_off[i], str_off[i + 1] - str_off[i]));
        }
        w.finish();
    } else {
        size_t width = type == BJ_INT32 ? 4 : 8;
        contest_pages::FixedWriter w(width, alloc);
        const uint8_t* src = static_cast<const uint8_t*>(values);
        for (uint64_t i = 0; i < n; i++) {
            if (valid && !valid[i])
                w.append_null();
            else
                w.append(src + i * width);
        }
        w.finish();
    }
    col.bytes = std::move(buf.bytes);
}

void encode_any(plan_io::OwnedColumn& col, int32_t type, uint64_t n, const void* values,
                const uint8_t* valid, const uint64_t* str_off, const char* str_bytes) {
    if (type != BJ_VARCHAR && !valid)
        encode_dense(col, type, values, n);
    else
        encode_general(col, type, n, values, valid, str_off, str_bytes);
}

bj_node scan_node(uint64_t table) {
    bj_node n{};
    n.kind = BJ_NODE_SCAN;
    n.base_table_id = table;
    return n;
}

bj_node join_node(uint64_t left, uint64_t right, uint64_t la, uint64_t ra, bool build_left) {
    bj_node n{};
    n.kind = BJ_NODE_JOIN;
    n.build_left = build_left;
    n.left = left;
    n.right = right;
    n.left_attr = la;
    n.right_attr = ra;
    return n;
}

void add_node(plan_io::OwnedPlan& p, bj_node n, std::vector<bj_attr> attrs) {
    p.nodes.push_back(n);
    p.attrs.push_back(std::move(attrs));
}

uint64_t scaled(double base, double scale) { return std::max<uint64_t>(1, uint64_t(std::llround(base * scale))); }

void make_join2(plan_io::OwnedPlan& p, uint64_t seed, double scale) {
    uint64_t nr = scaled(1e6, scale), ns = scaled(8e6, scale);
    p.tables.resize(2);
    // R
    {
        auto keys = permutation(nr, stream_seed(seed, 1, 0, 0));
        std::vector<int64_t> pay(nr);
        const uint64_t blk = 1 << 20;
        parallel_for((nr + blk - 1) / blk, [&](size_t b) {
            Rng r(stream_seed(seed, 1, 1, b));
            for (uint64_t i = b * blk; i < std::min(nr, (b + 1) * blk); i++) pay[i] = int64_t(r.below(1ull << 40));
        });
        auto& t = p.tables[0];
        t.num_rows = nr;
        t.columns.resize(2);
        encode_any(t.columns[0], BJ_INT32, nr, keys.data(), nullptr, nullptr, nullptr);
        encode_any(t.columns[1], BJ_INT64, nr, pay.data(), nullptr, nullptr, nullptr);
    }
    // S
    {
        std::vector<int32_t> fk(ns), pay(ns);
        std::vector<uint8_t> valid(ns);
        const uint64_t blk = 1 << 20;
        parallel_for((ns + blk - 1) / blk, [&](size_t b) {
            Rng r(stream_seed(seed, 2, 0, b));
            for (uint64_t i = b * blk; i < std::min(ns, (b + 1) * blk); i++) {
                valid[i] = r.below(10) != 0;
                fk[i] = int32_t(r.below(nr));
                pay[i] = int32_t(r.below(1000000));
            }
        });
        auto& t = p.tables[1];
        t.num_rows = ns;
        t.columns.resize(2);
        encode_any(t.columns[0], BJ_INT32, ns, fk.data(), valid.data(), nullptr, nullptr);
        encode_any(t.columns[1], BJ_INT32, ns, pay.data(), nullptr, nullptr, nullptr);
    }
    add_node(p, scan_node(0), {{0, BJ_INT32, 0}, {1, BJ_INT64, 0}});
    add_node(p, scan_node(1), {{0, BJ_INT32, 0}, {1, BJ_INT32, 0}});
    add_node(p, join_node(0, 1, 0, 0, true), {{1, BJ_INT64, 0}, {3, BJ_INT32, 0}, {2, BJ_INT32, 0}});
    p.root = 2;
}

void make_snowflake(plan_io::OwnedPlan& p, uint64_t seed, double scale) {
    const double dim_rows[4] = {5e6, 1e6, 2e5, 2e4};
    const int32_t thresholds[4] = {10, 50, 300, 600};
    uint64_t nf = scaled(50e6, scale);
    p.tables.resize(5);
    std::vector<std::vector<int32_t>> rank_to_key(4);
    for (int d = 0; d < 4; d++) {
        uint64_t nd = scaled(dim_rows[d], scale);
        auto keys = permutation(nd, stream_seed(seed, 10 + d, 0, 0));
        rank_to_key[d] = permutation(nd, stream_seed(seed, 10 + d, 1, 0));
        // Attributes and strings of all rows, then the load-time filter.
        std::vector<int32_t> attr(nd);
        std::vector<uint8_t> len(nd);
        const uint64_t blk = 1 << 18;
        parallel_for((nd + blk - 1) / blk, [&](size_t b) {
            Rng r(stream_seed(seed, 10 + d, 2, b));
            for (uint64_t i = b * blk; i < std::min(nd, (b + 1) * blk); i++) {
                attr[i] = int32_t(r.below(1000));
                len[i] = uint8_t(1 + r.below(64));
            }
        });
        std::vector<int32_t> fkey, fattr;
        std::vector<uint64_t> off{0};
        std::string bytes;
        Rng sr(stream_seed(seed, 10 + d, 3, 0));
        for (uint64_t i = 0; i < nd; i++) {
            if (attr[i] >= thresholds[d]) continue;
            fkey.push_back(keys[i]);
            fattr.push_back(attr[i]);
            for (int c = 0; c < len[i]; c++) bytes.push_back(char(32 + sr.below(95)));
            off.push_back(bytes.size());
        }
        auto& t = p.tables[1 + d];
        t.num_rows = fkey.size();
        t.columns.resize(3);
        encode_any(t.columns[0], BJ_INT32, fkey.size(), fkey.data(), nullptr, nullptr, nullptr);
        encode_any(t.columns[1], BJ_INT32, fattr.size(), fattr.data(), nullptr, nullptr, nullptr);
        encode_any(t.columns[2], BJ_VARCHAR, fkey.size(), nullptr, nullptr, off.data(), bytes.data());
    }
    // Fact: four Zipf(1.1) foreign keys.
    {
        auto& t = p.tables[0];
        t.num_rows = nf;
        t.columns.resize(4);
        std::vector<int32_t> fk(nf);
        for (int d = 0; d < 4; d++) {
            Zipf z(rank_to_key[d].size(), 1.1);
            const uint64_t blk = 1 << 20;
            parallel_for((nf + blk - 1) / blk, [&](size_t b) {
                Rng r(stream_seed(seed, 20 + d, 0, b));
                for (uint64_t i = b * blk; i < std::min(nf, (b + 1) * blk); i++)
                    fk[i] = rank_to_key[d][z.sample(r) - 1];
            });
            encode_any(t.columns[d], BJ_INT32, nf, fk.data(), nullptr, nullptr, nullptr);
        }
    }
    // Scans: fact {fk0..fk3}; dim d {key, name}.
    add_node(p, scan_node(0), {{0, BJ_INT32, 0}, {1, BJ_INT32, 0}, {2, BJ_INT32, 0}, {3, BJ_INT32, 0}});
    for (int d = 0; d < 4; d++) add_node(p, scan_node(1 + d), {{0, BJ_INT32, 0}, {2, BJ_VARCHAR, 0}});
    // ((((F J D0) J D1) J D2) J D3), each joining F.fk_d = D_d.key.
    // Node 5: F(0..3) + D0(key 4, name 5) -> keep fk0..fk3, name0.
    add_node(p, join_node(1, 0, 0, 0, true),
             {{2, BJ_INT32, 0}, {3, BJ_INT32, 0}, {4, BJ_INT32, 0}, {5, BJ_INT32, 0}, {1, BJ_VARCHAR, 0}});
    // Node 6: (fk0..fk3, name0) + D1(key 5, name 6) on fk1 -> fk1..fk3, name0.
    add_node(p, join_node(5, 2, 1, 0, false),
             {{1, BJ_INT32, 0}, {2, BJ_INT32, 0}, {3, BJ_INT32, 0}, {4, BJ_VARCHAR, 0}});
    // Node 7: (fk1, fk2, fk3, name0) + D2(key 4, name 5) on fk2 -> fk1, fk2, fk3, name0.
    add_node(p, join_node(6, 3, 1, 0, false),
             {{0, BJ_INT32, 0}, {1, BJ_INT32, 0}, {2, BJ_INT32, 0}, {3, BJ_VARCHAR, 0}});
    // Node 8: + D3(key 4, name 5) on fk3 -> name0, name3, fk1, fk2.
    add_node(p, join_node(7, 4, 2, 0, false),
             {{3, BJ_VARCHAR, 0}, {5, BJ_VARCHAR, 0}, {0, BJ_INT32, 0}, {1, BJ_INT32, 0}});
    p.root = 8;
}

} // namespace

// A plan over a prefix of a workload's tables (page arrays shared, not copied).
struct VariantPlan {
    std::vector<bj_table> tables;
    std::vector<std::vector<bj_attr>> attrs;
    std::vector<bj_node> nodes;
    bj_plan view{};
};

struct bjw_workload {
    plan_io::OwnedPlan plan;
    bj_plan view{};
    std::string name;
    std::vector<std::unique_ptr<VariantPlan>> variants;  // by dimension count
};

struct bjw_pages {
    plan_io::OwnedColumn col;
};

extern "C" {

int bjw_workload_create(const char* name, uint64_t seed, double scale, bjw_workload** out) {
    try {
        auto w = std::make_unique<bjw_workload>();
        std::string n(name ? name : "");
        w->name = n;
        if (n == "join2")
            make_join2(w->plan, seed, scale);
        else if (n == "snowflake")
            make_snowflake(w->plan, seed, scale);
        else
            return BJ_ERR_INVALID;
        w->view = w->plan.view();
        *out = w.release();
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INTERNAL;
    }
}

int bjw_workload_load(const char* path, bjw_workload** out) {
    try {
        auto w = std::make_unique<bjw_workload>();
        plan_io::Reader r(path);
        r.plan(w->plan);
        w->view = w->plan.view();
        *out = w.release();
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INVALID;
    }
}

const bj_plan* bjw_workload_plan(bjw_workload* w) { return &w->view; }

const bj_plan* bjw_workload_variant(bjw_workload* w, int dims) {
    if (!w || w->name != "snowflake" || dims < 1 || dims > 4) return nullptr;
    if (w->variants.size() <= size_t(dims)) w->variants.resize(dims + 1);
    auto& v = w->variants[dims];
    if (!v) {
        v = std::make_unique<VariantPlan>();
        for (int t = 0; t <= dims; t++) v->tables.push_back(w->view.inputs[t]);
        auto add = [&](bj_node n, std::vector<bj_attr> a) {
            v->nodes.push_back(n);
            v->attrs.push_back(std::move(a));
        };
        // Scans: fact {fk0..fk3}; dimension d {key, name}.
        add(scan_node(0), {{0, BJ_INT32, 0}, {1, BJ_INT32, 0}, {2, BJ_INT32, 0}, {3, BJ_INT32, 0}});
        for (int d = 0; d < dims; d++) add(scan_node(1 + d), {{0, BJ_INT32, 0}, {2, BJ_VARCHAR, 0}});
        // Join d keeps fk0..fk3 and the names so far, and adds dimension d's
        // name: left has 4 + d attributes, the right's name is 4 + d + 1.
        uint64_t left = 0;
        for (int d = 0; d < dims; d++) {
            std::vector<bj_attr> out;
            for (uint32_t a = 0; a < uint32_t(4 + d); a++) out.push_back({a, a < 4 ? BJ_INT32 : BJ_VARCHAR, 0});
            out.push_back({uint32_t(4 + d + 1), BJ_VARCHAR, 0});
            add(join_node(left, uint64_t(1 + d), uint64_t(d), 0, false), std::move(out));
            left = v->nodes.size() - 1;
        }
        for (size_t i = 0; i < v->nodes.size(); i++) {
            v->nodes[i].num_output_attrs = v->attrs[i].size();
            v->nodes[i].output_attrs = v->attrs[i].data();
        }
        v->view = bj_plan{v->nodes.size(), v->nodes.data(), v->tables.size(), v->tables.data(), left};
    }
    return &v->view;
}

uint64_t bjw_workload_scan_bytes(bjw_workload* w) {
    // Pages of every column a scan node names (each base column counted once).
    const bj_plan& p = w->view;
    std::vector<std::vector<bool>> used(p.num_inputs);
    for (uint64_t i = 0; i < p.num_inputs; i++) used[i].assign(p.inputs[i].num_columns, false);
    for (uint64_t n = 0; n < p.num_nodes; n++) {
        const bj_node& node = p.nodes[n];
        if (node.kind != BJ_NODE_SCAN) continue;
        for (uint64_t a = 0; a < node.num_output_attrs; a++)
            if (node.output_attrs[a].index < used[node.base_table_id].size())
                used[node.base_table_id][node.output_attrs[a].index] = true;
    }
    uint64_t bytes = 0;
    for (uint64_t i = 0; i < p.num_inputs; i++)
        for (uint64_t c = 0; c < p.inputs[i].num_columns; c++)
            if (used[i][c]) bytes += p.inputs[i].columns[c].num_pages * BJ_PAGE_SIZE;
    return bytes;
}

void bjw_workload_free(bjw_workload* w) { delete w; }

int bjw_save_plan(const char* path, const bj_plan* plan) {
    try {
        plan_io::Writer wr(path);
        wr.plan(*plan);
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INVALID;
    }
}

int bjw_save_table(const char* path, const bj_table* table) {
    try {
        plan_io::save_table(path, *table);
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INVALID;
    }
}

int bjw_encode_column(int32_t type, uint64_t n, const void* values, const uint8_t* valid,
                      const uint64_t* str_offsets, const char* str_bytes, bjw_pages** out) {
    if (type < BJ_INT32 || type > BJ_VARCHAR || !out) return BJ_ERR_INVALID;
    if (type == BJ_VARCHAR && n && !str_offsets) return BJ_ERR_INVALID;
    if (type != BJ_VARCHAR && n && !values) return BJ_ERR_INVALID;
    try {
        auto p = std::make_unique<bjw_pages>();
        encode_any(p->col, type, n, values, valid, str_offsets, str_bytes);
        p->col.index();
        *out = p.release();
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INTERNAL;
    }
}

uint64_t bjw_pages_count(const bjw_pages* p) { return p->col.ptrs.size(); }
const void* const* bjw_pages_ptrs(const bjw_pages* p) { return p->col.ptrs.data(); }
void bjw_pages_free(bjw_pages* p) { delete p; }

} // extern "C"
