// Test driver for the C++ drop-in (libcontest_b200.so): reads a plan file,
// builds a contest `Plan` that owns its pages (new Page, as the contest's
// loaders do), calls Contest::build_context / execute / destroy_context the
// way the contest harness does (tests/read_sql.cpp:1254-1256 of the contest
// repository), and writes the returned ColumnarTable to a result file.
//
//   contest_dropin <plan.bjplan> <out.bjtable> [repeat]
#include "../../include/contest/plan.h"
#include "../../include/contest/plan_io.h"

#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: contest_dropin <plan> <out> [repeat]\n");
        return 2;
    }
    int repeat = argc > 3 ? std::atoi(argv[3]) : 1;
    try {
        plan_io::OwnedPlan op;
        plan_io::Reader rd(argv[1]);
        rd.plan(op);
        Plan plan;
        for (auto& t : op.tables) {
            ColumnarTable ct;
            ct.num_rows = t.num_rows;
            for (auto& c : t.columns) {
                Column col{DataType(c.type)};
                for (size_t p = 0; p < c.bytes.size() / PAGE_SIZE; p++)
                    std::memcpy(col.new_page()->data, c.bytes.data() + p * PAGE_SIZE, PAGE_SIZE);
                ct.columns.push_back(std::move(col));
            }
            plan.new_input(std::move(ct));
        }
        for (size_t n = 0; n < op.nodes.size(); n++) {
            std::vector<std::tuple<size_t, DataType>> attrs;
            for (auto& a : op.attrs[n]) attrs.emplace_back(size_t(a.index), DataType(a.type));
            const bj_node& nd = op.nodes[n];
            if (nd.kind == BJ_NODE_SCAN)
                plan.new_scan_node(nd.base_table_id, std::move(attrs));
            else
                plan.new_join_node(nd.build_left != 0, nd.left, nd.right, nd.left_attr, nd.right_attr, std::move(attrs));
        }
        plan.root = op.root;
        void* ctx = Contest::build_context();
        ColumnarTable result;
        for (int i = 0; i < repeat; i++) result = Contest::execute(plan, ctx);
        Contest::destroy_context(ctx);
        std::vector<std::vector<const void*>> ptrs(result.columns.size());
        std::vector<bj_column> cols(result.columns.size());
        for (size_t c = 0; c < result.columns.size(); c++) {
            for (Page* p : result.columns[c].pages) ptrs[c].push_back(p);
            cols[c] = bj_column{int32_t(result.columns[c].type), 0, ptrs[c].size(), ptrs[c].data()};
        }
        bj_table t{result.num_rows, cols.size(), cols.data()};
        plan_io::save_table(argv[2], t);
        // `result` deletes its pages here, through Column's destructor.
    } catch (const std::exception& e) {
        std::fprintf(stderr, "contest_dropin: %s\n", e.what());
        return 1;
    }
    return 0;
}
