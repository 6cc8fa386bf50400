// Runner for the reference CPU engine -- TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile from the reference's own sources (nothing of them
// is copied into this repository) into oracle/_ref/ref_runner. It drives the
// reference through its public API exactly as the contest harness does
// (tests/read_sql.cpp:1254-1256, 1301-1306): Contest::build_context once, then
// Contest::execute(plan, ctx) per query.
//
//   ref_runner run   <plan.bjplan> <out.bjtable>
//       execute once, write the result table.
//   ref_runner bench <workload> <seed> <scale> <warmup> <steps> [out.bjtable]
//       generate a workload (libb200join_workloads.so), time execute() with
//       wall clock: `warmup` untimed calls, then `steps` timed calls; print
//       one JSON line.
//   ref_runner benchfile <plan.bjplan> <warmup> <steps>
//       same timing on a plan file.
//   ref_runner batch <workload> <seed> <scale> <passes>
//       every query of a batched workload ("schema20") once per pass, one
//       context for all; print queries/s and per-query latency as JSON.
#include <plan.h>

#include "../contest-sigmod2025_b200/csrc/workloads.h"
#include "../include/contest/plan_io.h"

#include <sched.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

// Builds a reference `Plan` whose pages point into the caller's buffers.
// `release` must run before the Plan dies: Column's destructor deletes pages.
struct BorrowedPlan {
    Plan plan;
    explicit BorrowedPlan(const bj_plan& p) {
        for (uint64_t i = 0; i < p.num_inputs; i++) {
            const bj_table& t = p.inputs[i];
            ColumnarTable ct;
            ct.num_rows = t.num_rows;
            for (uint64_t c = 0; c < t.num_columns; c++) {
                ct.columns.emplace_back(DataType(t.columns[c].type));
                for (uint64_t pg = 0; pg < t.columns[c].num_pages; pg++)
                    ct.columns.back().pages.push_back(const_cast<Page*>(static_cast<const Page*>(t.columns[c].pages[pg])));
            }
            plan.inputs.emplace_back(std::move(ct));
        }
        for (uint64_t n = 0; n < p.num_nodes; n++) {
            const bj_node& node = p.nodes[n];
            std::vector<std::tuple<size_t, DataType>> attrs;
            for (uint64_t a = 0; a < node.num_output_attrs; a++)
                attrs.emplace_back(size_t(node.output_attrs[a].index), DataType(node.output_attrs[a].type));
            if (node.kind == BJ_NODE_SCAN)
                plan.new_scan_node(node.base_table_id, std::move(attrs));
            else
                plan.new_join_node(node.build_left != 0, node.left, node.right, node.left_attr, node.right_attr,
                                   std::move(attrs));
        }
        plan.root = p.root;
    }
    ~BorrowedPlan() {
        for (auto& t : plan.inputs)
            for (auto& c : t.columns) c.pages.clear();
    }
};

void write_result(const std::string& path, const ColumnarTable& r) {
    std::vector<std::vector<const void*>> ptrs(r.columns.size());
    std::vector<bj_column> cols(r.columns.size());
    for (size_t c = 0; c < r.columns.size(); c++) {
        for (auto* p : r.columns[c].pages) ptrs[c].push_back(p);
        cols[c] = bj_column{int32_t(r.columns[c].type), 0, ptrs[c].size(), ptrs[c].data()};
    }
    bj_table t{r.num_rows, cols.size(), cols.data()};
    plan_io::save_table(path, t);
}

int cores() {
    cpu_set_t set;
    CPU_ZERO(&set);
    if (sched_getaffinity(0, sizeof(set), &set) != 0) return 1;
    return CPU_COUNT(&set);
}

int bench(const bj_plan& p, int warmup, int steps, const char* out_path, const char* label) {
    BorrowedPlan bp(p);
    void* ctx = Contest::build_context();
    std::vector<double> ms;
    uint64_t rows = 0;
    for (int i = 0; i < warmup + steps; i++) {
        auto t0 = std::chrono::steady_clock::now();
        ColumnarTable r = Contest::execute(bp.plan, ctx);
        auto t1 = std::chrono::steady_clock::now();
        rows = r.num_rows;
        if (i >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        if (out_path && i == warmup + steps - 1) write_result(out_path, r);
    }
    Contest::destroy_context(ctx);
    std::vector<double> sorted = ms;
    std::sort(sorted.begin(), sorted.end());
    double med = sorted.empty() ? 0 : sorted[sorted.size() / 2];
    double mean = 0;
    for (double v : ms) mean += v;
    mean = ms.empty() ? 0 : mean / ms.size();
    std::printf("{\"workload\": \"%s\", \"threads\": %d, \"rows\": %llu, \"median_ms\": %.4f, \"mean_ms\": %.4f, \"times_ms\": [",
                label, cores(), (unsigned long long)rows, med, mean);
    for (size_t i = 0; i < ms.size(); i++) std::printf("%s%.4f", i ? ", " : "", ms[i]);
    std::printf("]}\n");
    return 0;
}

int batch(bjw_workload* w, int passes, const char* label) {
    const uint64_t n = bjw_workload_num_queries(w);
    std::vector<std::unique_ptr<BorrowedPlan>> plans;
    for (uint64_t k = 0; k < n; k++) plans.push_back(std::make_unique<BorrowedPlan>(*bjw_workload_query(w, k)));
    void* ctx = Contest::build_context();
    std::vector<double> ms;
    uint64_t rows = 0;
    const auto start = std::chrono::steady_clock::now();
    for (int pass = 0; pass < passes; pass++)
        for (auto& bp : plans) {
            auto t0 = std::chrono::steady_clock::now();
            ColumnarTable r = Contest::execute(bp->plan, ctx);
            auto t1 = std::chrono::steady_clock::now();
            rows += r.num_rows;
            ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        }
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    Contest::destroy_context(ctx);
    std::vector<double> sorted = ms;
    std::sort(sorted.begin(), sorted.end());
    auto at = [&](double q) { return sorted.empty() ? 0.0 : sorted[std::min(sorted.size() - 1, size_t(q * sorted.size()))]; };
    std::printf("{\"workload\": \"%s\", \"threads\": %d, \"queries\": %zu, \"rows\": %llu, \"seconds\": %.4f, "
                "\"queries_per_s\": %.2f, \"p50_ms\": %.4f, \"p99_ms\": %.4f}\n",
                label, cores(), ms.size(), (unsigned long long)rows, total, total > 0 ? ms.size() / total : 0.0,
                at(0.5), at(0.99));
    return 0;
}

} // namespace

int main(int argc, char** argv) {
    try {
        if (argc >= 4 && std::string(argv[1]) == "run") {
            plan_io::OwnedPlan op;
            plan_io::Reader rd(argv[2]);
            rd.plan(op);
            bj_plan p = op.view();
            BorrowedPlan bp(p);
            void* ctx = Contest::build_context();
            {
                ColumnarTable r = Contest::execute(bp.plan, ctx);
                write_result(argv[3], r);
            }
            Contest::destroy_context(ctx);
            return 0;
        }
        if (argc >= 7 && std::string(argv[1]) == "bench") {
            bjw_workload* w = nullptr;
            if (bjw_workload_create(argv[2], std::stoull(argv[3]), std::stod(argv[4]), &w) != 0) {
                std::fprintf(stderr, "cannot build workload %s\n", argv[2]);
                return 2;
            }
            int rc = bench(*bjw_workload_plan(w), std::stoi(argv[5]), std::stoi(argv[6]), argc > 7 ? argv[7] : nullptr, argv[2]);
            bjw_workload_free(w);
            return rc;
        }
        if (argc >= 6 && std::string(argv[1]) == "batch") {
            bjw_workload* w = nullptr;
            if (bjw_workload_create(argv[2], std::stoull(argv[3]), std::stod(argv[4]), &w) != 0) {
                std::fprintf(stderr, "cannot build workload %s\n", argv[2]);
                return 2;
            }
            int rc = batch(w, std::stoi(argv[5]), argv[2]);
            bjw_workload_free(w);
            return rc;
        }
        if (argc >= 5 && std::string(argv[1]) == "benchfile") {
            plan_io::OwnedPlan op;
            plan_io::Reader rd(argv[2]);
            rd.plan(op);
            bj_plan p = op.view();
            return bench(p, std::stoi(argv[3]), std::stoi(argv[4]), nullptr, argv[2]);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_runner: %s\n", e.what());
        return 3;
    }
    std::fprintf(stderr, "usage: ref_runner run <plan> <out> | bench <workload> <seed> <scale> <warmup> <steps> [out] | benchfile <plan> <warmup> <steps> | batch <workload> <seed> <scale> <passes>\n");
    return 1;
}
