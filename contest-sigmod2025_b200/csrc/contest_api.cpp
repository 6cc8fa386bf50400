// Drop-in implementation of the contest API (include/contest/plan.h) on top of
// the C ABI. A program written against the contest's plan.h links
// libcontest_b200.so in place of the reference engine (engine/Execute.cpp:
// 28-48): build_context creates the device context, execute flattens the
// Plan into a bj_plan (page pointers are passed through, not copied),
// runs it, and turns the result into a ColumnarTable whose pages come from
// plain `new Page`, so Column's destructor can delete them (plan.h's
// ownership rule; the reference needs global operator new/delete overrides
// for the same purpose, engine/infra/PageMemory.cpp:138-203).
// Failures surface as std::runtime_error, as in the reference.
#include "../../include/contest/plan.h"
#include "../../include/b200join.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

int device_from_env() {
    const char* s = std::getenv("B200JOIN_DEVICE");
    return s ? std::atoi(s) : 0;
}

[[noreturn]] void raise(bj_context* ctx, int status, const char* what) {
    std::string msg = std::string("b200join: ") + what + " failed (status " + std::to_string(status) + ")";
    if (ctx && *bj_last_error(ctx)) msg += ": " + std::string(bj_last_error(ctx));
    throw std::runtime_error(msg);
}

void copy_pages_out(bj_result* r, uint64_t c, Column& col) {
    uint64_t n = bj_result_column_num_pages(r, c);
    col.pages.reserve(n);
    for (uint64_t p = 0; p < n; p++) col.pages.push_back(new Page);
    auto work = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t p = lo; p < hi; p++) {
            const void* src = bj_result_page(r, c, p);
            std::memcpy(col.pages[p]->data, src, PAGE_SIZE);
        }
    };
    unsigned nt = n > 2048 ? std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1u;
    if (nt == 1) {
        work(0, n);
        return;
    }
    std::vector<std::thread> ts;
    uint64_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        uint64_t lo = t * per, hi = std::min(n, lo + per);
        if (lo < hi) ts.emplace_back(work, lo, hi);
    }
    for (auto& t : ts) t.join();
}

} // namespace

namespace Contest {

void* build_context() {
    bj_context* ctx = nullptr;
    int st = bj_context_create(device_from_env(), &ctx);
    if (st != BJ_OK) raise(nullptr, st, "build_context");
    return ctx;
}

void destroy_context(void* context) { bj_context_destroy(static_cast<bj_context*>(context)); }

ColumnarTable execute(const Plan& plan, void* context) {
    bj_context* ctx = static_cast<bj_context*>(context);
    bool own = false;
    if (!ctx) {
        ctx = static_cast<bj_context*>(build_context());
        own = true;
    }
    // Flatten the plan: page pointer arrays are borrowed from the Plan.
    static_assert(sizeof(Page*) == sizeof(const void*), "page pointers are passed through as void*");
    std::vector<std::vector<bj_column>> cols(plan.inputs.size());
    std::vector<bj_table> tables(plan.inputs.size());
    for (size_t i = 0; i < plan.inputs.size(); i++) {
        const ColumnarTable& t = plan.inputs[i];
        for (const Column& c : t.columns)
            cols[i].push_back(bj_column{int32_t(c.type), 0, c.pages.size(),
                                        reinterpret_cast<const void* const*>(c.pages.data())});
        tables[i] = bj_table{t.num_rows, cols[i].size(), cols[i].data()};
    }
    std::vector<std::vector<bj_attr>> attrs(plan.nodes.size());
    std::vector<bj_node> nodes(plan.nodes.size());
    for (size_t n = 0; n < plan.nodes.size(); n++) {
        const PlanNode& pn = plan.nodes[n];
        for (auto& [idx, type] : pn.output_attrs) attrs[n].push_back(bj_attr{uint64_t(idx), int32_t(type), 0});
        bj_node& b = nodes[n];
        b = bj_node{};
        if (auto* s = std::get_if<ScanNode>(&pn.data)) {
            b.kind = BJ_NODE_SCAN;
            b.base_table_id = s->base_table_id;
        } else {
            const JoinNode& j = std::get<JoinNode>(pn.data);
            b.kind = BJ_NODE_JOIN;
            b.build_left = j.build_left;
            b.left = j.left;
            b.right = j.right;
            b.left_attr = j.left_attr;
            b.right_attr = j.right_attr;
        }
        b.num_output_attrs = attrs[n].size();
        b.output_attrs = attrs[n].data();
    }
    bj_plan bp{nodes.size(), nodes.data(), tables.size(), tables.data(), plan.root};
    bj_result* r = nullptr;
    int st = bj_execute(ctx, &bp, &r);
    if (st != BJ_OK) {
        std::string msg = bj_last_error(ctx);
        if (own) bj_context_destroy(ctx);
        throw std::runtime_error("b200join: execute failed (status " + std::to_string(st) + "): " + msg);
    }
    ColumnarTable out;
    out.num_rows = bj_result_num_rows(r);
    try {
        for (uint64_t c = 0; c < bj_result_num_columns(r); c++) {
            out.columns.emplace_back(DataType(bj_result_column_type(r, c)));
            copy_pages_out(r, c, out.columns.back());
        }
    } catch (...) {
        bj_result_free(r);
        if (own) bj_context_destroy(ctx);
        throw;
    }
    bj_result_free(r);
    if (own) bj_context_destroy(ctx);
    return out;
}

} // namespace Contest
