// Contest API types, restated for the B200 join engine.
//
// This header re-declares the SIGMOD 2025 contest interface that the reference
// engine implements (include/plan.h:24-149 and :337-344 of the contest
// repository, attribute.h:8-13 for DataType). The declarations must stay
// layout-compatible with that header so that a caller compiled against it can
// link against libcontest_b200.so instead of the reference engine: the same
// enums in the same order, the same struct members in the same order, and the
// same `Contest::` function signatures.
//
// Page format (the contest's 8 KiB column pages):
//   * fixed-width types: u16 row count at +0, u16 non-null count at +2, the
//     non-null values packed densely from +4 (INT32) or +8 (INT64 / FP64), and a
//     null bitmap (bit i set = row i is not null) in the last ceil(rows/8)
//     bytes of the page;
//   * VARCHAR: u16 row count, u16 non-null count, then one u16 end offset per
//     non-null string at +4, the string bytes right after the offsets, and the
//     same trailing bitmap;
//   * a string longer than PAGE_SIZE - 7 bytes occupies its own run of pages:
//     the first has row count 0xffff, the continuations 0xfffe, each with the
//     byte count of its chunk at +2 and the bytes from +4.
#pragma once

#include <cstddef>
#include <cstdint>
#include <tuple>
#include <variant>
#include <vector>

enum class DataType {
    INT32,
    INT64,
    FP64,
    VARCHAR,
};

enum class NodeType {
    HashJoin,
    Scan,
};

struct ScanNode {
    size_t base_table_id;
};

struct JoinNode {
    bool build_left;
    size_t left;
    size_t right;
    size_t left_attr;
    size_t right_attr;
};

struct PlanNode {
    std::variant<ScanNode, JoinNode> data;
    std::vector<std::tuple<size_t, DataType>> output_attrs;

    PlanNode(std::variant<ScanNode, JoinNode> node_data,
             std::vector<std::tuple<size_t, DataType>> attrs)
        : data(std::move(node_data)), output_attrs(std::move(attrs)) {}
};

constexpr size_t PAGE_SIZE = 8192;

struct alignas(8) Page {
    std::byte data[PAGE_SIZE];
};

// A column owns its pages: they are released with `delete` when the column dies.
struct Column {
    DataType type;
    std::vector<Page*> pages;

    explicit Column(DataType t) : type(t), pages() {}
    Column(Column&& other) noexcept : type(other.type), pages(std::move(other.pages)) {
        other.pages.clear();
    }
    Column& operator=(Column&& other) noexcept {
        if (this != &other) {
            release();
            type = other.type;
            pages = std::move(other.pages);
            other.pages.clear();
        }
        return *this;
    }
    Column(const Column&) = delete;
    Column& operator=(const Column&) = delete;
    ~Column() { release(); }

    Page* new_page() {
        Page* p = new Page;
        pages.push_back(p);
        return p;
    }

    private:
    void release() {
        for (Page* p : pages) delete p;
        pages.clear();
    }
};

struct ColumnarTable {
    size_t num_rows{0};
    std::vector<Column> columns;
};

struct Plan {
    std::vector<PlanNode> nodes;
    std::vector<ColumnarTable> inputs;
    size_t root;

    size_t new_join_node(bool build_left, size_t left, size_t right, size_t left_attr,
                         size_t right_attr, std::vector<std::tuple<size_t, DataType>> output_attrs) {
        JoinNode j{build_left, left, right, left_attr, right_attr};
        nodes.emplace_back(j, std::move(output_attrs));
        return nodes.size() - 1;
    }
    size_t new_scan_node(size_t base_table_id,
                         std::vector<std::tuple<size_t, DataType>> output_attrs) {
        ScanNode s{base_table_id};
        nodes.emplace_back(s, std::move(output_attrs));
        return nodes.size() - 1;
    }
    size_t new_input(ColumnarTable input) {
        inputs.emplace_back(std::move(input));
        return inputs.size() - 1;
    }
};

namespace Contest {
void* build_context();
void destroy_context(void* context);
ColumnarTable execute(const Plan& plan, void* context);
} // namespace Contest
