// CPU oracle for the join engine -- TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// What the reference computes, restated plainly:
//  * A plan is a tree of Scan and HashJoin nodes; a join node's output
//    attributes index the concatenation of its left and right children's
//    outputs (engine/query/PlanImport.cpp:24-41 follows the same indexing to
//    build attribute equivalence classes).
//  * Every join attribute is restricted to NOT NULL, so a NULL key never
//    matches (engine/query/QueryPlan.cpp:749-753).
//  * Join keys compare by value; the reference reads them as 32-bit integers
//    (engine/op/TableScan.cpp:328, engine/op/Hashtable.hpp:34-39).
//  * The result is the multiset of joined rows projected on the root's output
//    attributes, in any order (tests/read_sql.cpp:1208-1213 sorts both sides
//    before comparing); build sides and join order do not change it (the
//    reference ignores both, engine/query/QueryPlan.cpp:748-782).
// The oracle evaluates the tree bottom-up with sort-based equi-joins over
// row-id tuples, then writes the projected rows as contest pages with the
// same packing rules the contest's converter uses (src/build_table.cpp:456).
#include "oracle.h"

#include "../include/contest/pages.h"

#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct Fail : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void set_err(char* err, uint64_t len, const std::string& msg) {
    if (err && len) {
        std::snprintf(err, len, "%s", msg.c_str());
    }
}

const Page* const* page_ptrs(const bj_column& c) { return reinterpret_cast<const Page* const*>(c.pages); }

// A fully decoded column.
struct DecodedColumn {
    int32_t type = 0;
    std::vector<uint64_t> bits;     // INT32 sign-extended, INT64, FP64 bit pattern
    std::vector<std::string> strs;  // VARCHAR
    std::vector<uint8_t> valid;
};

DecodedColumn decode(const bj_column& c, uint64_t num_rows) {
    DecodedColumn d;
    d.type = c.type;
    d.valid.assign(num_rows, 0);
    if (c.type == BJ_VARCHAR)
        d.strs.resize(num_rows);
    else
        d.bits.assign(num_rows, 0);
    uint64_t seen = 0;
    contest_pages::decode_column(DataType(c.type), page_ptrs(c), c.num_pages,
                                 [&](size_t row, const contest_pages::Cell& cell) {
                                     if (row >= num_rows) throw Fail("column has more rows than the table");
                                     seen = row + 1;
                                     if (cell.kind < 0) return;
                                     d.valid[row] = 1;
                                     if (c.type == BJ_VARCHAR)
                                         d.strs[row] = cell.str;
                                     else
                                         d.bits[row] = cell.bits;
                                 });
    if (seen != num_rows) throw Fail("column has fewer rows than the table");
    return d;
}

struct AttrRef {
    uint32_t slot;    // position of the scan in the relation's row-id tuple
    uint32_t input;   // base table
    uint32_t column;  // base column
    int32_t type;
};

struct Relation {
    uint32_t width = 0;             // number of scans in the subtree
    std::vector<uint32_t> rids;     // rows * width base row ids
    std::vector<AttrRef> attrs;
    uint64_t rows() const { return width ? rids.size() / width : 0; }
};

class Evaluator {
    public:
    explicit Evaluator(const bj_plan& p) : plan_(p), cols_(p.num_inputs) {
        for (uint64_t i = 0; i < p.num_inputs; i++) cols_[i].resize(p.inputs[i].num_columns);
    }

    Relation eval(uint64_t node_id, int depth = 0) {
        if (node_id >= plan_.num_nodes) throw Fail("node index out of range");
        if (depth > 4096) throw Fail("plan is not a tree");
        const bj_node& n = plan_.nodes[node_id];
        if (n.kind == BJ_NODE_SCAN) return scan(n);
        if (n.kind != BJ_NODE_JOIN) throw Fail("unknown node kind");
        Relation l = eval(n.left, depth + 1);
        Relation r = eval(n.right, depth + 1);
        return join(n, l, r);
    }

    const DecodedColumn& column(uint32_t input, uint32_t col) {
        auto& slot = cols_[input][col];
        if (!slot) {
            const bj_table& t = plan_.inputs[input];
            slot = std::make_unique<DecodedColumn>(decode(t.columns[col], t.num_rows));
        }
        return *slot;
    }

    private:
    Relation scan(const bj_node& n) {
        if (n.base_table_id >= plan_.num_inputs) throw Fail("scan of a missing input");
        const bj_table& t = plan_.inputs[n.base_table_id];
        Relation rel;
        rel.width = 1;
        rel.rids.resize(t.num_rows);
        std::iota(rel.rids.begin(), rel.rids.end(), 0u);
        for (uint64_t a = 0; a < n.num_output_attrs; a++) {
            const bj_attr& at = n.output_attrs[a];
            if (t.num_rows && at.index >= t.num_columns) throw Fail("scan attribute out of range");
            if (t.num_rows && t.columns[at.index].type != at.type) throw Fail("scan attribute type mismatch");
            rel.attrs.push_back(AttrRef{0, uint32_t(n.base_table_id), uint32_t(at.index), at.type});
        }
        return rel;
    }

    // Sort key of one side's join attribute: non-null rows only.
    struct KeyRow {
        uint64_t key;
        uint32_t row;
    };

    std::vector<KeyRow> keyed(const Relation& rel, const AttrRef& a) {
        std::vector<KeyRow> out;
        if (rel.rows() == 0) return out;
        const DecodedColumn& c = column(a.input, a.column);
        out.reserve(rel.rows());
        for (uint64_t i = 0; i < rel.rows(); i++) {
            uint32_t rid = rel.rids[i * rel.width + a.slot];
            if (!c.valid[rid]) continue;
            out.push_back(KeyRow{c.bits[rid], uint32_t(i)});
        }
        std::sort(out.begin(), out.end(), [](const KeyRow& x, const KeyRow& y) {
            return x.key != y.key ? x.key < y.key : x.row < y.row;
        });
        return out;
    }

    Relation join(const bj_node& n, const Relation& l, const Relation& r) {
        if (n.left_attr >= l.attrs.size() || n.right_attr >= r.attrs.size()) throw Fail("join attribute out of range");
        const AttrRef& la = l.attrs[n.left_attr];
        const AttrRef& ra = r.attrs[n.right_attr];
        if (la.type == BJ_VARCHAR || ra.type == BJ_VARCHAR) throw Fail("VARCHAR join keys are not supported");
        if (la.type == BJ_FP64 || ra.type == BJ_FP64) throw Fail("FP64 join keys are not supported");
        Relation out;
        out.width = l.width + r.width;
        std::vector<AttrRef> both = l.attrs;
        for (AttrRef a : r.attrs) {
            a.slot += l.width;
            both.push_back(a);
        }
        for (uint64_t i = 0; i < n.num_output_attrs; i++) {
            if (n.output_attrs[i].index >= both.size()) throw Fail("join output attribute out of range");
            AttrRef a = both[n.output_attrs[i].index];
            if (a.type != n.output_attrs[i].type) throw Fail("join output attribute type mismatch");
            out.attrs.push_back(a);
        }
        // Merge join over the two sorted key lists.
        std::vector<KeyRow> lk = keyed(l, la), rk = keyed(r, ra);
        size_t i = 0, j = 0;
        while (i < lk.size() && j < rk.size()) {
            if (lk[i].key < rk[j].key) {
                i++;
            } else if (rk[j].key < lk[i].key) {
                j++;
            } else {
                size_t i2 = i, j2 = j;
                while (i2 < lk.size() && lk[i2].key == lk[i].key) i2++;
                while (j2 < rk.size() && rk[j2].key == rk[j].key) j2++;
                for (size_t x = i; x < i2; x++)
                    for (size_t y = j; y < j2; y++) {
                        const uint32_t* lr = &l.rids[size_t(lk[x].row) * l.width];
                        const uint32_t* rr = &r.rids[size_t(rk[y].row) * r.width];
                        out.rids.insert(out.rids.end(), lr, lr + l.width);
                        out.rids.insert(out.rids.end(), rr, rr + r.width);
                    }
                i = i2;
                j = j2;
            }
        }
        return out;
    }

    const bj_plan& plan_;
    std::vector<std::vector<std::unique_ptr<DecodedColumn>>> cols_;
};

struct PageStore {
    std::vector<std::unique_ptr<Page>> pages;
    Page* alloc() {
        pages.push_back(std::make_unique<Page>());
        return pages.back().get();
    }
};

} // namespace

struct oracle_table {
    std::vector<PageStore> stores;
    std::vector<std::vector<const void*>> ptrs;
    std::vector<bj_column> cols;
    bj_table view{};
};

struct oracle_rows {
    std::vector<int32_t> types;
    std::vector<uint8_t> bytes;      // canonical encodings, back to back
    std::vector<uint64_t> offsets;   // rows + 1
    std::vector<uint64_t> hashes;    // per row
    std::vector<uint32_t> order;     // sorted row order
};

namespace {

uint64_t hash_bytes(const uint8_t* p, size_t n) {
    uint64_t h = 0x6A09E667F3BCC909ull ^ (n * 0x9E3779B97F4A7C15ull);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = (h ^ w) * 0xD6E8FEB86659FD93ull;
        h ^= h >> 32;
    }
    uint64_t tail = 0;
    std::memcpy(&tail, p + i, n - i);
    h = (h ^ tail ^ (uint64_t(n - i) << 56)) * 0xD6E8FEB86659FD93ull;
    h ^= h >> 29;
    h *= 0x9FB21C651E98DF25ull;
    return h ^ (h >> 32);
}

void append_cell(std::vector<uint8_t>& out, int32_t type, bool valid, uint64_t bits, const std::string* s) {
    out.push_back(valid ? 1 : 0);
    if (!valid) return;
    switch (type) {
    case BJ_INT32: {
        uint32_t v = uint32_t(bits);
        out.insert(out.end(), reinterpret_cast<uint8_t*>(&v), reinterpret_cast<uint8_t*>(&v) + 4);
        break;
    }
    case BJ_INT64:
    case BJ_FP64:
        out.insert(out.end(), reinterpret_cast<uint8_t*>(&bits), reinterpret_cast<uint8_t*>(&bits) + 8);
        break;
    default: {
        uint32_t len = uint32_t(s->size());
        out.insert(out.end(), reinterpret_cast<uint8_t*>(&len), reinterpret_cast<uint8_t*>(&len) + 4);
        out.insert(out.end(), s->begin(), s->end());
    }
    }
}

std::string validate(const bj_table& t) {
    char buf[256];
    for (uint64_t c = 0; c < t.num_columns; c++) {
        const bj_column& col = t.columns[c];
        if (col.type < BJ_INT32 || col.type > BJ_VARCHAR) return "bad column type";
        uint64_t rows = 0;
        for (uint64_t p = 0; p < col.num_pages; p++) {
            const uint8_t* pg = static_cast<const uint8_t*>(col.pages[p]);
            uint16_t n, nv;
            std::memcpy(&n, pg, 2);
            std::memcpy(&nv, pg + 2, 2);
            if (col.type == BJ_VARCHAR && n >= 0xfffe) {
                if (nv > PAGE_SIZE - 4) return "long-string chunk too long";
                if (n == 0xfffe && p == 0) return "continuation page first";
                if (n == 0xfffe) {
                    uint16_t prev;
                    std::memcpy(&prev, col.pages[p - 1], 2);
                    if (prev < 0xfffe) return "continuation page after a short-string page";
                }
                if (n == 0xffff) rows++;
                continue;
            }
            // A page with no rows is valid (the reference's writers emit them).
            size_t nb = (n + 7) / 8;
            const uint8_t* bm = pg + PAGE_SIZE - nb;
            uint64_t pop = 0;
            for (size_t i = 0; i < n; i++) pop += (bm[i / 8] >> (i % 8)) & 1;
            if (pop != nv) {
                std::snprintf(buf, sizeof buf, "column %" PRIu64 " page %" PRIu64 ": %u non-null in header, %" PRIu64 " in bitmap", c, p, nv, pop);
                return buf;
            }
            if (col.type == BJ_VARCHAR) {
                uint16_t prev = 0;
                for (size_t i = 0; i < nv; i++) {
                    uint16_t e;
                    std::memcpy(&e, pg + 4 + 2 * i, 2);
                    if (e < prev) return "string offsets decrease";
                    prev = e;
                }
                if (4 + 2 * size_t(nv) + prev > PAGE_SIZE - nb) {
                    std::snprintf(buf, sizeof buf, "column %" PRIu64 " page %" PRIu64 ": strings overlap the bitmap", c, p);
                    return buf;
                }
            } else {
                size_t w = col.type == BJ_INT32 ? 4 : 8;
                if (contest_pages::value_begin(w) + nv * w > PAGE_SIZE - nb) {
                    std::snprintf(buf, sizeof buf, "column %" PRIu64 " page %" PRIu64 ": values overlap the bitmap", c, p);
                    return buf;
                }
            }
            rows += n;
        }
        if (rows != t.num_rows) {
            std::snprintf(buf, sizeof buf, "column %" PRIu64 " holds %" PRIu64 " rows, table says %" PRIu64, c, rows, t.num_rows);
            return buf;
        }
    }
    return "";
}

} // namespace

extern "C" {

int oracle_execute(const bj_plan* plan, oracle_table** out, char* err, uint64_t err_len) {
    try {
        if (!plan || !out) throw Fail("null argument");
        Evaluator ev(*plan);
        Relation rel = ev.eval(plan->root);
        auto res = std::make_unique<oracle_table>();
        size_t ncols = rel.attrs.size();
        res->stores.resize(ncols);
        res->ptrs.resize(ncols);
        res->cols.resize(ncols);
        uint64_t rows = rel.rows();
        for (size_t c = 0; c < ncols; c++) {
            const AttrRef& a = rel.attrs[c];
            PageStore& st = res->stores[c];
            auto alloc = [&st] { return st.alloc(); };
            if (rows) {
                const DecodedColumn& src = ev.column(a.input, a.column);
                if (a.type == BJ_VARCHAR) {
                    contest_pages::StringWriter w(alloc);
                    for (uint64_t i = 0; i < rows; i++) {
                        uint32_t rid = rel.rids[i * rel.width + a.slot];
                        if (src.valid[rid])
                            w.append(src.strs[rid]);
                        else
                            w.append_null();
                    }
                    w.finish();
                } else {
                    contest_pages::FixedWriter w(a.type == BJ_INT32 ? 4 : 8, alloc);
                    for (uint64_t i = 0; i < rows; i++) {
                        uint32_t rid = rel.rids[i * rel.width + a.slot];
                        if (src.valid[rid])
                            w.append(&src.bits[rid]);  // little-endian: low 4 bytes for INT32
                        else
                            w.append_null();
                    }
                    w.finish();
                }
            }
            for (auto& p : st.pages) res->ptrs[c].push_back(p.get());
            res->cols[c] = bj_column{a.type, 0, res->ptrs[c].size(), res->ptrs[c].data()};
        }
        res->view = bj_table{rows, ncols, res->cols.data()};
        *out = res.release();
        return BJ_OK;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return BJ_ERR_INVALID;
    }
}

const bj_table* oracle_table_view(const oracle_table* t) { return &t->view; }
void oracle_table_free(oracle_table* t) { delete t; }

int oracle_validate_table(const bj_table* t, char* err, uint64_t err_len) {
    std::string msg = validate(*t);
    if (msg.empty()) return 0;
    set_err(err, err_len, msg);
    return 1;
}

int oracle_rows_from_table(const bj_table* t, oracle_rows** out, char* err, uint64_t err_len) {
    try {
        std::string msg = validate(*t);
        if (!msg.empty()) throw Fail(msg);
        auto r = std::make_unique<oracle_rows>();
        std::vector<DecodedColumn> cols;
        for (uint64_t c = 0; c < t->num_columns; c++) {
            r->types.push_back(t->columns[c].type);
            cols.push_back(decode(t->columns[c], t->num_rows));
        }
        r->offsets.push_back(0);
        for (uint64_t i = 0; i < t->num_rows; i++) {
            for (uint64_t c = 0; c < cols.size(); c++) {
                const DecodedColumn& d = cols[c];
                append_cell(r->bytes, d.type, d.valid[i], d.type == BJ_VARCHAR ? 0 : d.bits[i],
                            d.type == BJ_VARCHAR ? &d.strs[i] : nullptr);
            }
            r->offsets.push_back(r->bytes.size());
        }
        uint64_t n = t->num_rows;
        r->hashes.resize(n);
        for (uint64_t i = 0; i < n; i++)
            r->hashes[i] = hash_bytes(r->bytes.data() + r->offsets[i], r->offsets[i + 1] - r->offsets[i]);
        r->order.resize(n);
        std::iota(r->order.begin(), r->order.end(), 0u);
        const oracle_rows* rp = r.get();
        std::sort(r->order.begin(), r->order.end(), [rp](uint32_t a, uint32_t b) {
            if (rp->hashes[a] != rp->hashes[b]) return rp->hashes[a] < rp->hashes[b];
            size_t la = rp->offsets[a + 1] - rp->offsets[a], lb = rp->offsets[b + 1] - rp->offsets[b];
            int c = std::memcmp(rp->bytes.data() + rp->offsets[a], rp->bytes.data() + rp->offsets[b], std::min(la, lb));
            return c != 0 ? c < 0 : la < lb;
        });
        *out = r.release();
        return BJ_OK;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return BJ_ERR_INVALID;
    }
}

uint64_t oracle_rows_count(const oracle_rows* r) { return r->order.size(); }

int oracle_rows_equal(const oracle_rows* a, const oracle_rows* b, uint64_t* first_diff) {
    uint64_t n = std::min(a->order.size(), b->order.size());
    if (a->types != b->types) {
        if (first_diff) *first_diff = 0;
        return 0;
    }
    for (uint64_t i = 0; i < n; i++) {
        uint32_t x = a->order[i], y = b->order[i];
        size_t lx = a->offsets[x + 1] - a->offsets[x], ly = b->offsets[y + 1] - b->offsets[y];
        if (a->hashes[x] != b->hashes[y] || lx != ly ||
            std::memcmp(a->bytes.data() + a->offsets[x], b->bytes.data() + b->offsets[y], lx) != 0) {
            if (first_diff) *first_diff = i;
            return 0;
        }
    }
    if (a->order.size() != b->order.size()) {
        if (first_diff) *first_diff = n;
        return 0;
    }
    return 1;
}

void oracle_rows_digest(const oracle_rows* r, uint64_t out[3]) {
    uint64_t s = 0, x = 0;
    for (uint64_t h : r->hashes) {
        s += h;
        x ^= h;
    }
    out[0] = r->order.size();
    out[1] = s;
    out[2] = x;
}

int oracle_rows_format(const oracle_rows* r, uint64_t i, char* buf, uint64_t len) {
    if (i >= r->order.size() || !buf || !len) return 1;
    uint32_t row = r->order[i];
    const uint8_t* p = r->bytes.data() + r->offsets[row];
    std::string s = "(";
    char tmp[64];
    for (size_t c = 0; c < r->types.size(); c++) {
        if (c) s += ", ";
        bool valid = *p++;
        if (!valid) {
            s += "NULL";
            continue;
        }
        switch (r->types[c]) {
        case BJ_INT32: {
            int32_t v;
            std::memcpy(&v, p, 4);
            p += 4;
            std::snprintf(tmp, sizeof tmp, "%d", v);
            s += tmp;
            break;
        }
        case BJ_INT64: {
            int64_t v;
            std::memcpy(&v, p, 8);
            p += 8;
            std::snprintf(tmp, sizeof tmp, "%" PRId64, v);
            s += tmp;
            break;
        }
        case BJ_FP64: {
            double v;
            std::memcpy(&v, p, 8);
            p += 8;
            std::snprintf(tmp, sizeof tmp, "%.17g", v);
            s += tmp;
            break;
        }
        default: {
            uint32_t l;
            std::memcpy(&l, p, 4);
            p += 4;
            s += "'";
            s.append(reinterpret_cast<const char*>(p), l);
            s += "'";
            p += l;
        }
        }
    }
    s += ")";
    std::snprintf(buf, len, "%s", s.c_str());
    return 0;
}

void oracle_rows_free(oracle_rows* r) { delete r; }

} // extern "C"
