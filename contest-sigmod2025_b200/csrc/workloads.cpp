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

// "schema20": 20 tables in a random PK-FK tree and a batch of random acyclic
// join queries over them (the batched-workload shape: 2-12 tables per query,
// tables of 10K-40M rows before their filter, per-table filter selectivity
// log-uniform in [0.1%, 100%], PK-FK edges uniform or Zipf(0.8-1.5)).
// Table t: c0 INT32 primary key (a permutation of the unfiltered rows), c1
// INT32 foreign key to its parent's c0 (table 0: uniform values), c2 INT32
// uniform in [0, 1e6), c3 FP64 uniform in [0, 1), c4 VARCHAR of 1-32
// printable characters. The filter keeps a row when a seeded draw falls under
// the table's selectivity (applied at load time, as the contest does).
struct QuerySpec {
    std::vector<uint32_t> tables;  // in join order: each after a neighbour
    std::vector<uint32_t> via;     // via[i]: the earlier table tables[i] joins (i >= 1)
    std::vector<uint32_t> payload; // per table: the payload column its scan outputs (2, 3 or 4)
    std::vector<std::pair<uint32_t, uint32_t>> out;  // (position in tables, 0 key / 1 payload)
};

constexpr uint32_t kSchemaTables = 20;

constexpr uint32_t kNoRow = 0xffffffffu;

// The exact result size of a query: a count over the join tree, children
// before parents (a table joins one added before it, so reverse order works).
// prow[t][r]: the parent row that row r of table t references (kNoRow: none).
double schema20_count(const QuerySpec& q, const std::vector<uint32_t>& parent,
                      const std::vector<std::vector<uint32_t>>& prow) {
    const size_t m = q.tables.size();
    std::vector<std::vector<double>> w(m);
    for (size_t i = 0; i < m; i++) w[i].assign(prow[q.tables[i]].size(), 1.0);
    for (size_t i = m; i-- > 1;) {
        const uint32_t t = q.tables[i], v = q.via[i];
        size_t j = 0;
        while (q.tables[j] != v) j++;
        if (parent[t] == v && t != v) {  // t is v's child: sum t's weights into the rows they reference
            std::vector<double> agg(w[j].size(), 0.0);
            for (size_t r = 0; r < w[i].size(); r++)
                if (prow[t][r] != kNoRow) agg[prow[t][r]] += w[i][r];
            for (size_t r = 0; r < w[j].size(); r++) w[j][r] *= agg[r];
        } else {                         // t is v's parent: each row of v takes the weight of its row of t
            for (size_t r = 0; r < w[j].size(); r++)
                w[j][r] *= prow[v][r] == kNoRow ? 0.0 : w[i][prow[v][r]];
        }
    }
    double total = 0;
    for (double x : w[0]) total += x;
    return total;
}

// With wide keys, every other table (odd ids) keys its rows by INT64 values
// whose low 32 bits are the INT32 key's and whose high half is a small
// signed number that varies per row (so low halves repeat across keys), and
// its children's foreign keys are INT64 too (no reference counterpart: the
// reference reads join keys as 32 bits).
constexpr int64_t wide_key(int32_t k) {
    const int64_t hi = int64_t((uint32_t(k) * 2654435761u) >> 29) - 4;  // -4 .. 3
    return int64_t(uint64_t(hi) << 32 | uint32_t(k));
}

void make_schema20(plan_io::OwnedPlan& p, uint64_t seed, double scale, uint32_t nqueries,
                   std::vector<uint32_t>& parent, std::vector<QuerySpec>& queries, std::vector<uint64_t>& rows,
                   const std::vector<uint8_t>& wide) {
    std::vector<std::vector<uint32_t>> prow;
    Rng g(stream_seed(seed, 200, 0, 0));
    rows.assign(kSchemaTables, 0);
    std::vector<double> sel(kSchemaTables), skew(kSchemaTables);
    parent.assign(kSchemaTables, 0);
    for (uint32_t t = 0; t < kSchemaTables; t++) {
        rows[t] = scaled(std::exp(std::log(1e4) + g.unit() * (std::log(4e7) - std::log(1e4))), scale);
        sel[t] = std::exp(std::log(1e-3) + g.unit() * (0.0 - std::log(1e-3)));
        skew[t] = g.unit() < 0.5 ? 0.0 : 0.8 + 0.7 * g.unit();  // 0: uniform FK
        parent[t] = t ? uint32_t(g.below(t)) : 0u;
    }
    // Tables in order (a parent precedes its children): a foreign key draws a
    // rank over the parent's rows that passed its filter (uniform or Zipf),
    // mapped to a row by a seeded permutation, so every edge joins.
    std::vector<std::vector<uint32_t>> ranked(kSchemaTables);  // per table: its rows in rank order
    std::vector<std::vector<int32_t>> key(kSchemaTables);      // per table: c0 of its rows
    prow.assign(kSchemaTables, {});
    p.tables.resize(kSchemaTables);
    auto make_table = [&](uint32_t t) {
        const uint64_t n = rows[t];
        const auto keys = permutation(n, stream_seed(seed, 202, t, 0));
        Rng r(stream_seed(seed, 203, t, 0));
        const std::vector<uint32_t>& pr = ranked[parent[t]];
        std::unique_ptr<Zipf> z;
        if (t && skew[t] > 0 && !pr.empty()) z = std::make_unique<Zipf>(pr.size(), skew[t]);
        std::vector<int32_t>& c0 = key[t];
        std::vector<int32_t> c1, c2;
        std::vector<double> c3;
        std::vector<uint64_t> off{0};
        std::string bytes;
        for (uint64_t i = 0; i < n; i++) {
            int32_t fk;
            uint32_t to = kNoRow;
            if (!t || pr.empty()) {
                fk = int32_t(r.below(1000000));
            } else {
                to = z ? pr[z->sample(r) - 1] : pr[r.below(pr.size())];
                fk = key[parent[t]][to];
            }
            const int32_t a = int32_t(r.below(1000000));
            const double d = r.unit();
            const uint32_t len = 1 + uint32_t(r.below(32));
            const bool keep = r.unit() < sel[t];
            if (!keep) {
                for (uint32_t c = 0; c < len; c++) r.next();
                continue;
            }
            c0.push_back(keys[i]);
            c1.push_back(fk);
            prow[t].push_back(to);
            c2.push_back(a);
            c3.push_back(d);
            for (uint32_t c = 0; c < len; c++) bytes.push_back(char(32 + r.below(95)));
            off.push_back(bytes.size());
        }
        // The kept rows in a seeded order (the rank -> row map of the FKs).
        ranked[t].resize(c0.size());
        for (uint32_t i = 0; i < c0.size(); i++) ranked[t][i] = i;
        Rng sh(stream_seed(seed, 201, t, 0));
        for (uint64_t i = ranked[t].size(); i > 1; i--) std::swap(ranked[t][i - 1], ranked[t][sh.below(i)]);
        auto& tab = p.tables[t];
        tab.num_rows = c0.size();
        tab.columns.resize(5);
        auto encode_key = [&](plan_io::OwnedColumn& col, const std::vector<int32_t>& v, bool w64) {
            if (!w64) {
                encode_any(col, BJ_INT32, v.size(), v.data(), nullptr, nullptr, nullptr);
                return;
            }
            std::vector<int64_t> v64(v.size());
            for (size_t i = 0; i < v.size(); i++) v64[i] = wide_key(v[i]);
            encode_any(col, BJ_INT64, v64.size(), v64.data(), nullptr, nullptr, nullptr);
        };
        encode_key(tab.columns[0], c0, wide[t]);
        encode_key(tab.columns[1], c1, t && wide[parent[t]]);
        encode_any(tab.columns[2], BJ_INT32, c2.size(), c2.data(), nullptr, nullptr, nullptr);
        encode_any(tab.columns[3], BJ_FP64, c3.size(), c3.data(), nullptr, nullptr, nullptr);
        encode_any(tab.columns[4], BJ_VARCHAR, c0.size(), nullptr, nullptr, off.data(), bytes.data());
    };
    // A table needs its parent's rows: tables are made level by level of the
    // tree, the tables of one level in parallel (each from its own streams).
    std::vector<uint8_t> made(kSchemaTables, 0);
    for (size_t left = kSchemaTables; left;) {
        std::vector<uint32_t> level;
        for (uint32_t t = 0; t < kSchemaTables; t++)
            if (!made[t] && (t == 0 || made[parent[t]])) level.push_back(t);
        parallel_for(level.size(), [&](size_t i) { make_table(level[i]); });
        for (uint32_t t : level) made[t] = 1;
        left -= level.size();
    }
    // Queries: a random connected set of 2-12 tables grown from a random table.
    std::vector<std::vector<uint32_t>> nbr(kSchemaTables);
    for (uint32_t t = 1; t < kSchemaTables; t++) {
        nbr[t].push_back(parent[t]);
        nbr[parent[t]].push_back(t);
    }
    queries.assign(nqueries, QuerySpec{});
    parallel_for(nqueries, [&](size_t k) {
        Rng q(stream_seed(seed, 204, k, 0));
        const uint32_t want = 2 + uint32_t(q.below(11));
        QuerySpec spec;
        std::vector<uint8_t> in(kSchemaTables, 0);
        const uint32_t start = uint32_t(q.below(kSchemaTables));
        spec.tables.push_back(start);
        spec.via.push_back(start);
        in[start] = 1;
        // A table joins only when the result of the tables so far stays within
        // the largest of them (no many-to-many blow-up through a shared parent
        // under skew); the plan joins in this order, so every intermediate
        // result is bounded the same way.
        uint64_t largest = p.tables[start].num_rows;
        while (spec.tables.size() < want) {
            std::vector<std::pair<uint32_t, uint32_t>> frontier;  // (new table, its neighbour in the set)
            for (uint32_t x : spec.tables)
                for (uint32_t y : nbr[x])
                    if (!in[y]) frontier.push_back({y, x});
            bool added = false;
            while (!frontier.empty() && !added) {
                const size_t at = q.below(frontier.size());
                const auto pick = frontier[at];
                spec.tables.push_back(pick.first);
                spec.via.push_back(pick.second);
                const uint64_t cap = std::max<uint64_t>(largest, p.tables[pick.first].num_rows);
                if (spec.tables.size() == 2 || schema20_count(spec, parent, prow) <= double(cap)) {
                    in[pick.first] = 1;
                    largest = cap;
                    added = true;
                } else {
                    spec.tables.pop_back();
                    spec.via.pop_back();
                    frontier.erase(frontier.begin() + at);
                }
            }
            if (!added) break;
        }
        for (size_t i = 0; i < spec.tables.size(); i++) spec.payload.push_back(2 + uint32_t(q.below(3)));
        const uint32_t nout = 1 + uint32_t(q.below(4));
        for (uint32_t o = 0; o < nout; o++)
            spec.out.push_back({uint32_t(q.below(spec.tables.size())), q.below(4) == 0 ? 0u : 1u});
        queries[k] = std::move(spec);
    });
}

// The plan of one schema20 query: scans output (c0, c1, payload) per table;
// each join appends a table joined on its edge to an earlier one (child's c1
// = parent's c0) and keeps every attribute; the root projects the query's
// outputs.
void schema20_plan(const QuerySpec& q, const std::vector<uint32_t>& parent, const std::vector<uint8_t>& wide,
                   std::vector<bj_node>& nodes, std::vector<std::vector<bj_attr>>& attrs, uint64_t& root) {
    nodes.clear();
    attrs.clear();
    auto kt = [&](bool w) { return w ? BJ_INT64 : BJ_INT32; };
    auto type_of = [](uint32_t c) { return c == 3 ? BJ_FP64 : c == 4 ? BJ_VARCHAR : BJ_INT32; };
    std::vector<uint32_t> base;  // attribute index of each table's c0 in the growing join output
    std::vector<bj_attr> acc;    // the growing join output
    uint64_t left = 0;
    for (size_t i = 0; i < q.tables.size(); i++) {
        const uint32_t t = q.tables[i];
        nodes.push_back(scan_node(t));
        attrs.push_back({{0, kt(wide[t]), 0}, {1, kt(t && wide[parent[t]]), 0}, {q.payload[i], type_of(q.payload[i]), 0}});
        const uint64_t scan = nodes.size() - 1;
        if (i == 0) {
            left = scan;
            base.push_back(0);
            acc = attrs.back();
            for (uint32_t a = 0; a < 3; a++) acc[a].index = a;
            continue;
        }
        // Join the new table with its neighbour v (position j): child.c1 = parent.c0.
        const uint32_t v = q.via[i];
        size_t j = 0;
        while (q.tables[j] != v) j++;
        uint64_t la, ra;
        if (parent[t] == v && t != v) {  // t is v's child
            la = base[j] + 0;            // v.c0
            ra = 1;                      // t.c1
        } else {                         // t is v's parent
            la = base[j] + 1;            // v.c1
            ra = 0;                      // t.c0
        }
        std::vector<bj_attr> out;
        const uint32_t width = uint32_t(acc.size());
        for (uint32_t a = 0; a < width + 3; a++) {
            const int32_t ty = a < width ? acc[a].type : attrs[scan][a - width].type;
            out.push_back({a, ty, 0});
        }
        nodes.push_back(join_node(left, scan, la, ra, true));
        attrs.push_back(out);
        base.push_back(width);
        acc = out;
        left = nodes.size() - 1;
    }
    // Root: the outputs (a table's key, or its payload).
    std::vector<bj_attr> out;
    for (const auto& [pos, what] : q.out) {
        const uint32_t a = base[pos] + (what == 0 ? 0u : 2u);
        out.push_back({a, acc[a].type, 0});
    }
    attrs[left] = out;  // the last join (queries have two tables or more) projects the outputs
    root = left;
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
    std::vector<uint64_t> base_rows;  // schema20: rows of each table before its filter
    std::vector<std::unique_ptr<VariantPlan>> variants;  // by dimension count
    std::vector<std::unique_ptr<VariantPlan>> queries;   // schema20: every query over the shared tables
};

struct bjw_pages {
    plan_io::OwnedColumn col;
};

extern "C" {

int bjw_workload_create(const char* name, uint64_t seed, double scale, bjw_workload** out) {
    return bjw_workload_create_queries(name, seed, scale, 256, out);
}

int bjw_workload_create_queries(const char* name, uint64_t seed, double scale, uint64_t nqueries,
                                bjw_workload** out) {
    try {
        auto w = std::make_unique<bjw_workload>();
        std::string n(name ? name : "");
        w->name = n;
        if (n == "join2") {
            make_join2(w->plan, seed, scale);
        } else if (n == "snowflake") {
            make_snowflake(w->plan, seed, scale);
        } else if (n == "schema20" || n == "schema20w") {
            std::vector<uint32_t> parent;
            std::vector<QuerySpec> specs;
            std::vector<uint8_t> wide(kSchemaTables, 0);
            if (n == "schema20w")
                for (uint32_t t = 1; t < kSchemaTables; t += 2) wide[t] = 1;
            if (nqueries < 1 || nqueries > (1u << 20)) return BJ_ERR_INVALID;
            make_schema20(w->plan, seed, scale, uint32_t(nqueries), parent, specs, w->base_rows, wide);
            // Query 0 is the workload's own plan; every query is also a plan
            // over the shared tables.
            schema20_plan(specs[0], parent, wide, w->plan.nodes, w->plan.attrs, w->plan.root);
            w->view = w->plan.view();
            for (const QuerySpec& q : specs) {
                auto v = std::make_unique<VariantPlan>();
                v->tables.assign(w->view.inputs, w->view.inputs + w->view.num_inputs);
                uint64_t root = 0;
                schema20_plan(q, parent, wide, v->nodes, v->attrs, root);
                for (size_t i = 0; i < v->nodes.size(); i++) {
                    v->nodes[i].num_output_attrs = v->attrs[i].size();
                    v->nodes[i].output_attrs = v->attrs[i].data();
                }
                v->view = bj_plan{v->nodes.size(), v->nodes.data(), v->tables.size(), v->tables.data(), root};
                w->queries.push_back(std::move(v));
            }
            *out = w.release();
            return BJ_OK;
        } else {
            return BJ_ERR_INVALID;
        }
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

uint64_t bjw_workload_base_rows(bjw_workload* w, uint64_t table) {
    if (!w || table >= w->view.num_inputs) return 0;
    return table < w->base_rows.size() ? w->base_rows[table] : w->view.inputs[table].num_rows;
}

uint64_t bjw_workload_num_queries(bjw_workload* w) { return w ? (w->queries.empty() ? 1 : w->queries.size()) : 0; }

const bj_plan* bjw_workload_query(bjw_workload* w, uint64_t k) {
    if (!w) return nullptr;
    if (w->queries.empty()) return k == 0 ? &w->view : nullptr;
    return k < w->queries.size() ? &w->queries[k]->view : nullptr;
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
