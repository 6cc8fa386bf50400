// Binary files for plans and tables (header-only, host side).
//
// Used to hand the same plan and pages to separate processes (the reference
// engine's runner, the test suite, the benchmark) without re-generating data.
// Layout, all little-endian:
//   table : u64 num_rows, u64 num_columns, per column { i32 type, u32 0,
//           u64 num_pages, num_pages * 8192 page bytes }
//   plan  : "BJPLAN01", u64 num_inputs, tables..., u64 num_nodes, per node
//           { i32 kind, i32 build_left, u64 base_table_id, u64 left, u64 right,
//             u64 left_attr, u64 right_attr, u64 num_attrs,
//             num_attrs * { u64 index, i32 type, u32 0 } }, u64 root
//   result: "BJTABL01", one table
// The in-memory form is `OwnedPlan`: pages in one buffer plus a `bj_plan` view.
#pragma once

#include "../b200join.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace plan_io {

struct OwnedColumn {
    int32_t type = 0;
    std::vector<uint8_t> bytes;     // num_pages * BJ_PAGE_SIZE
    std::vector<const void*> ptrs;  // page pointers into bytes
    void index() {
        ptrs.resize(bytes.size() / BJ_PAGE_SIZE);
        for (size_t i = 0; i < ptrs.size(); i++) ptrs[i] = bytes.data() + i * BJ_PAGE_SIZE;
    }
};

struct OwnedTable {
    uint64_t num_rows = 0;
    std::vector<OwnedColumn> columns;
    std::vector<bj_column> view_cols;
    bj_table view() {
        view_cols.resize(columns.size());
        for (size_t i = 0; i < columns.size(); i++) {
            columns[i].index();
            view_cols[i] = bj_column{columns[i].type, 0, columns[i].ptrs.size(), columns[i].ptrs.data()};
        }
        return bj_table{num_rows, columns.size(), view_cols.data()};
    }
};

struct OwnedPlan {
    std::vector<OwnedTable> tables;
    std::vector<bj_table> table_views;
    std::vector<std::vector<bj_attr>> attrs;
    std::vector<bj_node> nodes;
    uint64_t root = 0;
    bj_plan view() {
        table_views.resize(tables.size());
        for (size_t i = 0; i < tables.size(); i++) table_views[i] = tables[i].view();
        for (size_t i = 0; i < nodes.size(); i++) {
            nodes[i].num_output_attrs = attrs[i].size();
            nodes[i].output_attrs = attrs[i].data();
        }
        return bj_plan{nodes.size(), nodes.data(), table_views.size(), table_views.data(), root};
    }
};

class Writer {
    public:
    explicit Writer(const std::string& path) : f_(std::fopen(path.c_str(), "wb")) {
        if (!f_) throw std::runtime_error("cannot open " + path);
    }
    ~Writer() {
        if (f_) std::fclose(f_);
    }
    void raw(const void* p, size_t n) {
        if (n && std::fwrite(p, 1, n, f_) != n) throw std::runtime_error("short write");
    }
    template <typename T>
    void pod(const T& v) { raw(&v, sizeof(T)); }
    void table(const bj_table& t) {
        pod<uint64_t>(t.num_rows);
        pod<uint64_t>(t.num_columns);
        for (uint64_t c = 0; c < t.num_columns; c++) {
            const bj_column& col = t.columns[c];
            pod<int32_t>(col.type);
            pod<uint32_t>(0);
            pod<uint64_t>(col.num_pages);
            for (uint64_t p = 0; p < col.num_pages; p++) raw(col.pages[p], BJ_PAGE_SIZE);
        }
    }
    void plan(const bj_plan& p) {
        raw("BJPLAN01", 8);
        pod<uint64_t>(p.num_inputs);
        for (uint64_t i = 0; i < p.num_inputs; i++) table(p.inputs[i]);
        pod<uint64_t>(p.num_nodes);
        for (uint64_t i = 0; i < p.num_nodes; i++) {
            const bj_node& n = p.nodes[i];
            pod<int32_t>(n.kind);
            pod<int32_t>(n.build_left);
            pod<uint64_t>(n.base_table_id);
            pod<uint64_t>(n.left);
            pod<uint64_t>(n.right);
            pod<uint64_t>(n.left_attr);
            pod<uint64_t>(n.right_attr);
            pod<uint64_t>(n.num_output_attrs);
            for (uint64_t a = 0; a < n.num_output_attrs; a++) {
                pod<uint64_t>(n.output_attrs[a].index);
                pod<int32_t>(n.output_attrs[a].type);
                pod<uint32_t>(0);
            }
        }
        pod<uint64_t>(p.root);
    }

    private:
    FILE* f_;
};

class Reader {
    public:
    explicit Reader(const std::string& path) : f_(std::fopen(path.c_str(), "rb")) {
        if (!f_) throw std::runtime_error("cannot open " + path);
    }
    ~Reader() {
        if (f_) std::fclose(f_);
    }
    void raw(void* p, size_t n) {
        if (n && std::fread(p, 1, n, f_) != n) throw std::runtime_error("truncated file");
    }
    template <typename T>
    T pod() {
        T v;
        raw(&v, sizeof(T));
        return v;
    }
    void magic(const char* m) {
        char buf[8];
        raw(buf, 8);
        if (std::memcmp(buf, m, 8) != 0) throw std::runtime_error(std::string("bad magic, want ") + m);
    }
    void table(OwnedTable& t) {
        t.num_rows = pod<uint64_t>();
        uint64_t nc = pod<uint64_t>();
        if (nc > (1u << 20)) throw std::runtime_error("implausible column count");
        t.columns.resize(nc);
        for (auto& c : t.columns) {
            c.type = pod<int32_t>();
            pod<uint32_t>();
            uint64_t np = pod<uint64_t>();
            c.bytes.resize(np * BJ_PAGE_SIZE);
            raw(c.bytes.data(), c.bytes.size());
        }
    }
    void plan(OwnedPlan& p) {
        magic("BJPLAN01");
        uint64_t ni = pod<uint64_t>();
        p.tables.resize(ni);
        for (auto& t : p.tables) table(t);
        uint64_t nn = pod<uint64_t>();
        p.nodes.resize(nn);
        p.attrs.resize(nn);
        for (uint64_t i = 0; i < nn; i++) {
            bj_node& n = p.nodes[i];
            n.kind = pod<int32_t>();
            n.build_left = pod<int32_t>();
            n.base_table_id = pod<uint64_t>();
            n.left = pod<uint64_t>();
            n.right = pod<uint64_t>();
            n.left_attr = pod<uint64_t>();
            n.right_attr = pod<uint64_t>();
            uint64_t na = pod<uint64_t>();
            p.attrs[i].resize(na);
            for (auto& a : p.attrs[i]) {
                a.index = pod<uint64_t>();
                a.type = pod<int32_t>();
                a.reserved = pod<uint32_t>();
            }
        }
        p.root = pod<uint64_t>();
    }

    private:
    FILE* f_;
};

inline void save_table(const std::string& path, const bj_table& t) {
    Writer w(path);
    w.raw("BJTABL01", 8);
    w.table(t);
}

inline void load_table(const std::string& path, OwnedTable& t) {
    Reader r(path);
    r.magic("BJTABL01");
    r.table(t);
}

} // namespace plan_io
