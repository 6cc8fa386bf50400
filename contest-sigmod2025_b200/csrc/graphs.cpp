// CUDA-graph replay of repeated resident queries: the graph cache of a
// context, capture under a recorded read-back tape, and replay.
#include "engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

namespace bj {

// ---------------------------------------------------------------------------
// CUDA-graph replay of repeated resident queries.
//
// A serving process runs the same query shapes over the same resident tables
// again and again. The first run of a (plan, tables, flags) key executes
// normally and records every host read-back (probe hit rates, table flags,
// counts) on a tape. The second run executes the same host logic under
// stream capture, answering read-backs from the tape instead of
// synchronising, so every kernel, copy and cross-stream dependency of the
// query lands in one CUDA graph. Later runs launch that graph -- all kernels
// run again, on the same resident inputs -- and copy the result pages out.
// The tables are immutable once resident, so the recorded counts stay exact;
// freeing a table drops the graphs that read it.

std::vector<uint64_t> graph_key(const bj_plan& plan, bj_resident* const* tables, int flags, bool profile) {
    std::vector<uint64_t> k{plan.num_nodes, plan.num_inputs, plan.root, uint64_t(flags), uint64_t(profile)};
    for (uint64_t i = 0; i < plan.num_nodes; i++) {
        const bj_node& n = plan.nodes[i];
        k.insert(k.end(), {uint64_t(n.kind), uint64_t(n.build_left), n.base_table_id, n.left, n.right, n.left_attr,
                           n.right_attr, n.num_output_attrs});
        for (uint64_t a = 0; a < n.num_output_attrs; a++) {
            k.push_back(n.output_attrs[a].index);
            k.push_back(uint64_t(uint32_t(n.output_attrs[a].type)));
        }
    }
    for (uint64_t i = 0; i < plan.num_inputs; i++) k.push_back(reinterpret_cast<uint64_t>(tables[i]));
    return k;
}

void destroy_graph(GraphEntry& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    for (cudaEvent_t e : g.prof) cudaEventDestroy(e);
    g.prof.clear();
    for (cudaEvent_t e : g.phase) cudaEventDestroy(e);
    g.phase.clear();
}

bool capture_graph(bj_context* ctx, GraphEntry& g, const bj_plan* plan, bj_resident* const* resident, int flags) {
    bool capturing = false;
    bj_result res;
    res.ctx = ctx;
    uint64_t launches0 = ctx->launches;
    try {
        ExecPlan ex;
        std::string err;
        if (make_exec_plan(*plan, ex, err, false, g.cards.empty() ? nullptr : &g.cards, g.space) != BJ_OK ||
            ex.empty)
            return false;
        ctx->tune = tune_for(ctx, ex);
        std::vector<const DevTable*> tables(plan->num_inputs);
        for (uint64_t i = 0; i < plan->num_inputs; i++) tables[i] = &resident[i]->table;
        g.tape.pos = 0;
        ctx->tape = &g.tape;
        ctx->tape_mode = 2;
        ctx->graph_output = true;
        BJ_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        capturing = true;
        // The graph clears the device error word first and copies it to the
        // pinned read-back slot last, so a replay needs no other call.
        BJ_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
        uint64_t pipelines = 0;
        const bool nonempty = run_pipelines(ctx, ex, tables, res, flags, pipelines);
        BJ_CK(cudaMemcpyAsync(&ctx->h_small[63], ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        capturing = false;
        cudaGraph_t graph = nullptr;
        BJ_CK(cudaStreamEndCapture(ctx->stream, &graph));
        ctx->tape_mode = 0;
        ctx->tape = nullptr;
        ctx->graph_output = false;
        // The recording ends with the call's final error check, not replayed here.
        if (!graph || g.tape.pos + 1 != g.tape.slots.size()) {
            if (graph) cudaGraphDestroy(graph);
            throw Fail{BJ_ERR_INTERNAL, "graph capture diverged from its recording"};
        }
        cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) throw Fail{BJ_ERR_CUDA, "cudaGraphInstantiate failed"};
        g.out_types = ex.out_types;
        if (nonempty) {
            g.rows = res.rows;
            g.npages = res.npages;
            g.page_base = res.page_base;
            g.total_pages = res.total_pages;
            g.pages = res.arena_pages;
        } else {
            g.rows = 0;
            g.npages.assign(ex.out_types.size(), 0);
            g.page_base.assign(ex.out_types.size(), 0);
            g.total_pages = 0;
            g.pages = nullptr;
        }
        g.stats = bj_stats{};
        g.stats.kernel_launches = ctx->launches - launches0;
        g.stats.pipelines = pipelines;
        g.stats.arena_bytes = ctx->arena.used_total();
        for (uint64_t i = 0; i < plan->num_inputs; i++) {
            std::vector<uint8_t> used;
            collect_columns(ex, uint32_t(i), tables[i]->cols.size(), used);
            for (size_t c = 0; c < used.size(); c++)
                if (used[c]) g.stats.input_pages += tables[i]->cols[c].npages;
        }
        g.prof = ctx->prof_events;
        g.phase = ctx->phase_events;
        g.prof_bytes = ctx->prof_bytes;
        ctx->prof_events.clear();
        ctx->phase_events.clear();
        ctx->prof_bytes = 0;
        ctx->arena.reset();
        return true;
    } catch (const Fail&) {
        if (capturing) {
            cudaGraph_t gr = nullptr;
            cudaStreamEndCapture(ctx->stream, &gr);
            if (gr) cudaGraphDestroy(gr);
        }
        cudaGetLastError();
        ctx->gather.n = 0;
        ctx->tape_mode = 0;
        ctx->tape = nullptr;
        ctx->graph_output = false;
        for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
        ctx->prof_events.clear();
        for (cudaEvent_t e : ctx->phase_events) cudaEventDestroy(e);
        ctx->phase_events.clear();
        ctx->prof_bytes = 0;
        ctx->sync_all();
        ctx->arena.reset();
        return false;
    }
}

int replay_graph(bj_context* ctx, GraphEntry& g, const std::vector<int32_t>& types, int flags, bj_result** out) {
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<bj_result> res(new bj_result);
    res->ctx = ctx;
    try {
        res->types = types;
        ctx->h_small[63] = 0;  // the graph's last node writes the low half
        BJ_CK(cudaEventRecord(ctx->ev0, ctx->stream));
        BJ_CK(cudaGraphLaunch(g.exec, ctx->stream));
        res->rows = g.rows;
        res->npages = g.npages;
        res->page_base = g.page_base;
        res->total_pages = g.total_pages;
        size_t bytes = g.total_pages * kPageSize;
        if (bytes && (flags & BJ_RESULT_DEVICE)) {
            BJ_CK(cudaMallocAsync(reinterpret_cast<void**>(&res->dev), bytes, ctx->stream));
            BJ_CK(cudaMemcpyAsync(res->dev, g.pages, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        } else if (bytes) {
            res->host = ctx->take_pinned(bytes);
            BJ_CK(cudaMemcpyAsync(res->host.p, g.pages, bytes, cudaMemcpyDeviceToHost, ctx->stream));
            res->stats.d2h_bytes = bytes;
        }
        BJ_CK(cudaEventRecord(ctx->ev1, ctx->stream));
        bool async = (flags & BJ_RESULT_ASYNC) && ctx->async_err && g.prof.empty() && g.phase.empty();
        if (async) {
            // The error word of this query goes to its own slot; the result
            // completes in bj_result_wait (device_ms is not measured).
            {
                std::lock_guard<std::mutex> lk(ctx->release_m);
                async = !ctx->free_slots.empty();
                if (async) {
                    res->slot = ctx->free_slots.back();
                    ctx->free_slots.pop_back();
                    if (!ctx->free_done.empty()) {
                        res->done = ctx->free_done.back();
                        ctx->free_done.pop_back();
                    }
                }
            }
            if (async && !res->done && cudaEventCreateWithFlags(&res->done, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                std::lock_guard<std::mutex> lk(ctx->release_m);
                ctx->free_slots.push_back(res->slot);
                throw Fail{BJ_ERR_CUDA, "event creation failed"};
            }
        }
        if (async) {
            ctx->async_err[res->slot] = 0;
            res->pending = true;
            BJ_CK(cudaMemcpyAsync(ctx->async_err + res->slot, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  ctx->stream));
            BJ_CK(cudaEventRecord(res->done, ctx->stream));
        } else {
            BJ_CK(cudaStreamSynchronize(ctx->stream));
            if (uint32_t code = uint32_t(ctx->h_small[63]))
                throw Fail{BJ_ERR_INVALID, std::string("device check failed: ") + dev_error_text(code)};
            float ms = 0;
            BJ_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            res->stats.device_ms = ms;
        }
        for (size_t i = 0; i + 1 < g.prof.size(); i += 2) {
            float k = 0;
            BJ_CK(cudaEventElapsedTime(&k, g.prof[i], g.prof[i + 1]));
            res->stats.scan_kernel_ms += k;
            res->stats.scan_kernel_launches++;
        }
        phase_stats(g.phase, res->stats);
        res->stats.scan_kernel_bytes = g.prof_bytes;
        res->stats.kernel_launches = g.stats.kernel_launches;
        res->stats.pipelines = g.stats.pipelines;
        res->stats.arena_bytes = g.stats.arena_bytes;
        res->stats.input_pages = g.stats.input_pages;
        res->stats.output_pages = g.total_pages;
        ctx->launches += g.stats.kernel_launches;
    } catch (const Fail& f) {
        int st = fail_to_status(ctx, f);  // waits for the stream
        if (res->pending) {
            std::lock_guard<std::mutex> lk(ctx->release_m);
            ctx->free_slots.push_back(res->slot);
            ctx->free_done.push_back(res->done);
            res->pending = false;
        }
        if (res->dev) cudaFree(res->dev);
        res->dev = nullptr;
        ctx->give_pinned(res->host);
        res->host = PinnedBlock{};
        return st;
    }
    res->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->live_results++;
    ctx->last_error.clear();
    *out = res.release();
    return BJ_OK;
}

int execute_resident_graph(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, int flags,
                           bj_result** out) {
    ctx->drain_releases();
    std::vector<uint64_t> key = graph_key(*plan, tables, flags & ~BJ_RESULT_ASYNC, ctx->profile);
    key.push_back(uint64_t(ctx->ordering));
    key.push_back(reinterpret_cast<uint64_t>(ctx->estimator));
    key.push_back(uint64_t(ctx->plan_space));
    uint64_t hash = 0x9e3779b97f4a7c15ull;
    for (uint64_t v : key) hash = (hash ^ v) * 0x100000001b3ull + (hash >> 29);
    GraphEntry* g = nullptr;
    auto& gc = ctx->graph_cache;
    for (size_t i = gc.size(); i-- > 0;)
        if (gc[i]->hash == hash && gc[i]->key == key) {
            // Most recently used goes last.
            std::rotate(gc.begin() + i, gc.begin() + i + 1, gc.end());
            g = gc.back().get();
            break;
        }
    if (!g) {
        auto e = std::make_unique<GraphEntry>();
        e->key = std::move(key);
        e->hash = hash;
        e->tables.assign(tables, tables + plan->num_inputs);
        ctx->tape = &e->tape;
        ctx->tape_mode = 1;
        ctx->cards_out = &e->cards;
        ctx->space_out = &e->space;
        int st = execute_common(ctx, plan, tables, flags, out);
        ctx->cards_out = nullptr;
        ctx->space_out = nullptr;
        ctx->tape_mode = 0;
        ctx->tape = nullptr;
        if (st == BJ_OK) {
            if (gc.size() >= bj_context::kGraphCache) {
                destroy_graph(*gc.front());
                gc.erase(gc.begin());
            }
            gc.push_back(std::move(e));
        }
        return st;
    }
    if (!g->failed && !g->exec && !capture_graph(ctx, *g, plan, tables, flags)) g->failed = true;
    if (g->failed) {
        ctx->cards_in = &g->cards;  // plan as the first run did
        ctx->space_in = &g->space;
        int st = execute_common(ctx, plan, tables, flags, out);
        ctx->cards_in = nullptr;
        ctx->space_in = nullptr;
        return st;
    }
    return replay_graph(ctx, *g, g->out_types, flags, out);
}

// Waits for ctx's work, then drops its graphs that read table t.
void drop_graphs_using(bj_context* ctx, const bj_resident* t) {
    ctx->sync_all();
    auto& gc = ctx->graph_cache;
    for (size_t i = 0; i < gc.size();) {
        const auto& tabs = gc[i]->tables;
        if (std::find(tabs.begin(), tabs.end(), t) != tabs.end()) {
            destroy_graph(*gc[i]);
            gc.erase(gc.begin() + i);
        } else {
            i++;
        }
    }
}

} // namespace bj
