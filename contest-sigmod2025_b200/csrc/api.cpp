// The C ABI of include/b200join.h around the executor: plan explanation,
// context life cycle and settings, the execute entry points and results.
#include "engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace bj;

extern "C" {

BJ_API const char* bj_version(void) { return "b200join 0.1 (sm_100a)"; }

BJ_API int bj_plan_explain(const bj_plan* plan, char* buf, uint64_t cap, uint64_t* len) {
    if (!plan || !len || (cap && !buf)) return BJ_ERR_INVALID;
    try {
        ExecPlan ex;
        std::string err;
        int st = make_exec_plan(*plan, ex, err, true);
        if (st != BJ_OK) return st;
        std::string out;
        char line[256];
        auto input_text = [&](uint32_t i) {
            char t[96];
            std::snprintf(t, sizeof t, "input %u (table %u, %llu rows)", i, ex.inputs[i].table,
                          static_cast<unsigned long long>(ex.inputs[i].rows));
            return std::string(t);
        };
        if (ex.empty) {
            out = "empty: an input has no rows\n";
        } else {
            out = "driver: " + input_text(ex.driver);
            if (ex.est_cost >= 0) {
                std::snprintf(line, sizeof line, "; estimated cost %.4g (result card + 10 x hashed card per join)",
                              ex.est_cost);
                out += line;
            }
            if (ex.ref_cost >= 0) {
                std::snprintf(line, sizeof line, "; the reference's plan space at best %.4g", ex.ref_cost);
                out += line;
            }
            out += "\n";
            for (size_t p = 0; p < ex.pipelines.size(); p++) {
                const PipelinePlan& pp = ex.pipelines[p];
                std::snprintf(line, sizeof line, "pipeline %zu: scan ", p);
                out += line;
                out += input_text(pp.input);
                for (size_t k = 0; k < pp.probes.size(); k++) {
                    std::snprintf(line, sizeof line, "%s pipeline %u on attr %u", k ? "," : ", probe", pp.probes[k].child,
                                  pp.probes[k].probe_attr);
                    out += line;
                    if (pp.probes[k].key_probe >= 0) {
                        std::snprintf(line, sizeof line, " (payload of pipeline %u)",
                                      pp.probes[size_t(pp.probes[k].key_probe)].child);
                        out += line;
                    }
                }
                if (pp.build_key >= 0) {
                    std::snprintf(line, sizeof line, " -> hash table on attr %lld", static_cast<long long>(pp.build_key));
                    out += line;
                    if (pp.build_key_probe >= 0) {
                        std::snprintf(line, sizeof line, " (payload of pipeline %u)",
                                      pp.probes[size_t(pp.build_key_probe)].child);
                        out += line;
                    }
                    if (pp.restrict_by >= 0) {
                        std::snprintf(line, sizeof line, ", rows restricted by pipeline %d's filter", pp.restrict_by);
                        out += line;
                    }
                } else {
                    out += " -> result";
                }
                out += "\n";
            }
            if (!ex.ref_plan.empty()) out += "reference plan space, cheapest: " + ex.ref_plan + "\n";
            if (ex.rooted_cost >= 0) {
                std::snprintf(line, sizeof line, "rooted plan space, cheapest: driver input %u, cost %.4g\n",
                              ex.rooted_driver, ex.rooted_cost);
                out += line;
            }
            out += ex.reference_space ? "runs: the reference space's plan\n" : "runs: the rooted plan\n";
            // The drop-in path's guess of the probe scanned first (it starts
            // copying that column's pages before the device sampling decides).
            const int g = guess_first_probe(ex, *plan);
            if (g >= 0) {
                const PipelinePlan& root = ex.pipelines.back();
                std::snprintf(line, sizeof line, "scan guess: pipeline %u on attr %u\n", root.probes[size_t(g)].child,
                              root.probes[size_t(g)].probe_attr);
                out += line;
            }
        }
        *len = out.size();
        if (cap) {
            const size_t n = std::min<size_t>(out.size(), cap - 1);
            std::memcpy(buf, out.data(), n);
            buf[n] = '\0';
        }
        return BJ_OK;
    } catch (...) {
        return BJ_ERR_INTERNAL;
    }
}

BJ_API int bj_context_create(int device, bj_context** out) {
    if (!out) return BJ_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return BJ_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return BJ_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return BJ_ERR_CUDA;
    auto ctx = std::make_unique<bj_context>();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return BJ_ERR_CUDA;
    for (auto& s : ctx->side)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return BJ_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking) != cudaSuccess) return BJ_ERR_CUDA;
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) return BJ_ERR_CUDA;
    if (cudaMalloc(&ctx->d_err, 256) != cudaSuccess) return BJ_ERR_OOM;
    ctx->arena.err = ctx->d_err;
    if (cudaMalloc(&ctx->d_small, sizeof(uint64_t) * 64) != cudaSuccess) return BJ_ERR_OOM;
    if (cudaHostAlloc(reinterpret_cast<void**>(&ctx->h_small), sizeof(uint64_t) * 64, cudaHostAllocDefault) != cudaSuccess)
        return BJ_ERR_OOM;
    cudaMemset(ctx->d_err, 0, 256);
    cudaMemset(ctx->d_small, 0, sizeof(uint64_t) * 64);
    if (cudaHostAlloc(reinterpret_cast<void**>(&ctx->async_err), sizeof(uint32_t) * bj_context::kAsyncSlots,
                      cudaHostAllocDefault) != cudaSuccess)
        return BJ_ERR_OOM;
    for (uint32_t i = bj_context::kAsyncSlots; i > 0; i--) ctx->free_slots.push_back(i - 1);
    // Keep freed result buffers cached in the stream-ordered pool.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t threshold = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (const char* zc = std::getenv("B200JOIN_ZERO_COPY")) ctx->zero_copy = std::atoi(zc) != 0;
    if (const char* gr = std::getenv("B200JOIN_GRAPHS")) ctx->graphs = std::atoi(gr) != 0;
    if (const char* sp = std::getenv("B200JOIN_SCAN_SPLIT")) ctx->scan_split = std::atoi(sp) != 0;
    if (const char* ss = std::getenv("B200JOIN_STREAM_SCAN")) ctx->stream_scans = std::atoi(ss) != 0;
    if (const char* lb = std::getenv("B200JOIN_LEAF_BATCH")) ctx->leaf_batch = std::atoi(lb) != 0;
    if (const char* sw = std::getenv("B200JOIN_SIDEWAYS")) ctx->sideways = std::atoi(sw) != 0;
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    ctx->pool = std::make_unique<ThreadPool>(std::min(hw, 16u) - 1);
    *out = ctx.release();
    return BJ_OK;
}

BJ_API void bj_context_destroy(bj_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    ctx->sync_all();
    for (auto& g : ctx->graph_cache) destroy_graph(*g);
    ctx->graph_cache.clear();
    for (cudaEvent_t e : ctx->pipe_events) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->window_events) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->free_done) cudaEventDestroy(e);
    if (ctx->async_err) cudaFreeHost(ctx->async_err);
    for (uint8_t* p : ctx->release_dev) cudaFree(p);
    for (cudaStream_t s : ctx->side)
        if (s) cudaStreamDestroy(s);
    if (ctx->copy) cudaStreamDestroy(ctx->copy);
    for (auto& b : ctx->pinned_free) cudaFreeHost(b.p);
    if (ctx->stage.p) cudaFreeHost(ctx->stage.p);
    if (ctx->h_small) cudaFreeHost(ctx->h_small);
    if (ctx->d_small) cudaFree(ctx->d_small);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

BJ_API const char* bj_last_error(const bj_context* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

BJ_API void* bj_context_stream(bj_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

BJ_API int bj_context_autotune(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, int repeats,
                               char* report, uint64_t cap, uint64_t* len) {
    if (!ctx || !plan || !tables || repeats < 1) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    ExecPlan ex;
    std::string err;
    int st = make_exec_plan(*plan, ex, err);
    if (st != BJ_OK) {
        ctx->last_error = err;
        return st;
    }
    const uint64_t key = shape_class(ex);
    std::string text = "shape class " + std::to_string(key >> 16) + "/" + std::to_string((key >> 8) & 255) + "/" +
                       std::to_string(key & 255) + " (log2 rows of the largest and second largest input / inputs)\n";
    const bool graphs = ctx->graphs;
    ctx->graphs = false;  // every run executes (no replay)
    TuneConfig best{};
    double best_ms = -1;
    int64_t rows = -1;  // every parameter set must return the same row count
    for (uint8_t split : {uint8_t(1), uint8_t(0)})
        for (uint8_t bits : {uint8_t(8), uint8_t(16), uint8_t(32)})
            for (uint8_t extra : {uint8_t(0), uint8_t(1)}) {
                TuneConfig c{split, bits, extra};
                ctx->tune_override = &c;
                std::vector<double> ms;
                for (int r = 0; r <= repeats && st == BJ_OK; r++) {
                    bj_result* res = nullptr;
                    st = bj_execute_resident(ctx, plan, tables, BJ_RESULT_DEVICE, &res);
                    if (st != BJ_OK) break;
                    bj_stats s{};
                    bj_result_stats(res, &s);
                    const int64_t n = int64_t(bj_result_num_rows(res));
                    bj_result_free(res);
                    if (rows >= 0 && n != rows) {
                        ctx->last_error = "autotune: parameter sets returned different row counts";
                        st = BJ_ERR_INTERNAL;
                        break;
                    }
                    rows = n;
                    if (r > 0) ms.push_back(s.device_ms);  // the first run warms up
                }
                ctx->tune_override = nullptr;
                if (st != BJ_OK) break;
                std::sort(ms.begin(), ms.end());
                const double med = ms[ms.size() / 2];
                char line[160];
                std::snprintf(line, sizeof(line), "scan %s, bloom %2u bits/key, buckets x%u: %.4f ms\n",
                              split ? "split" : "fused", unsigned(bits), 1u << extra, med);
                text += line;
                if (best_ms < 0 || med < best_ms) {
                    best_ms = med;
                    best = c;
                }
            }
    ctx->graphs = graphs;
    if (st != BJ_OK) return st;
    bool found = false;
    for (auto& [k, c] : ctx->tuned)
        if (k == key) {
            c = best;
            found = true;
        }
    if (!found) ctx->tuned.push_back({key, best});
    // Graphs captured under other parameters are dropped.
    ctx->sync_all();
    for (auto& g : ctx->graph_cache) destroy_graph(*g);
    ctx->graph_cache.clear();
    char line[160];
    std::snprintf(line, sizeof(line), "chosen: scan %s, bloom %u bits/key, buckets x%u (%.4f ms)\n",
                  best.scan_split ? "split" : "fused", unsigned(best.bloom_bits), 1u << best.bucket_extra, best_ms);
    text += line;
    if (len) *len = text.size();
    if (report && cap) {
        const size_t n = std::min<size_t>(cap - 1, text.size());
        std::memcpy(report, text.data(), n);
        report[n] = 0;
    }
    return BJ_OK;
}

BJ_API int bj_context_set_plan_space(bj_context* ctx, int space) {
    if (!ctx || space < 0 || space > 2) return BJ_ERR_INVALID;
    ctx->plan_space = PlanSpace(space);
    return BJ_OK;
}

BJ_API void bj_context_set_graphs(bj_context* ctx, int on) {
    if (!ctx) return;
    if (!on) {
        // Graphs already captured stay valid but are no longer used.
        ctx->sync_all();
    }
    ctx->graphs = on != 0;
}

BJ_API void bj_context_profile(bj_context* ctx, int on) {
    if (ctx) ctx->profile = on != 0;
}

BJ_API int bj_execute(bj_context* ctx, const bj_plan* plan, bj_result** out) {
    if (!ctx) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    return execute_common(ctx, plan, nullptr, BJ_RESULT_HOST, out);
}

BJ_API int bj_execute_resident(bj_context* ctx, const bj_plan* plan, bj_resident* const* tables, int flags,
                               bj_result** out) {
    if (!ctx || !tables) return BJ_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->graphs && plan) return execute_resident_graph(ctx, plan, tables, flags, out);
    return execute_common(ctx, plan, tables, flags, out);
}


BJ_API uint64_t bj_result_num_rows(const bj_result* r) { return r ? r->rows : 0; }
BJ_API uint64_t bj_result_num_columns(const bj_result* r) { return r ? r->types.size() : 0; }
BJ_API int32_t bj_result_column_type(const bj_result* r, uint64_t c) {
    return r && c < r->types.size() ? r->types[c] : -1;
}
BJ_API uint64_t bj_result_column_num_pages(const bj_result* r, uint64_t c) {
    return r && c < r->npages.size() ? r->npages[c] : 0;
}
BJ_API int bj_result_wait(bj_result* r) {
    if (!r) return BJ_ERR_INVALID;
    if (!r->pending) return r->status;
    bj_context* ctx = r->ctx;
    const cudaError_t e = cudaEventSynchronize(r->done);
    const uint32_t code = *reinterpret_cast<volatile uint32_t*>(ctx->async_err + r->slot);
    {
        std::lock_guard<std::mutex> lk(ctx->release_m);
        ctx->free_slots.push_back(r->slot);
        ctx->free_done.push_back(r->done);
    }
    r->done = nullptr;
    r->pending = false;
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->last_error = std::string("CUDA error: ") + cudaGetErrorString(e);
        r->status = BJ_ERR_CUDA;
    } else if (code) {
        ctx->last_error = std::string("device check failed: ") + dev_error_text(code);
        r->status = BJ_ERR_INVALID;
    }
    return r->status;
}

// The data accessors complete an asynchronous result first.
static bool result_ready(const bj_result* r) { return r && bj_result_wait(const_cast<bj_result*>(r)) == BJ_OK; }

BJ_API const void* bj_result_page(const bj_result* r, uint64_t c, uint64_t p) {
    if (!result_ready(r) || !r->host.p || c >= r->npages.size() || p >= r->npages[c]) return nullptr;
    return r->host.p + (r->page_base[c] + p) * kPageSize;
}
BJ_API const void* bj_result_device_page(const bj_result* r, uint64_t c, uint64_t p) {
    if (!result_ready(r) || !r->dev || c >= r->npages.size() || p >= r->npages[c]) return nullptr;
    return r->dev + (r->page_base[c] + p) * kPageSize;
}
BJ_API int bj_result_copy_pages(const bj_result* r, uint64_t c, void* const* dst) {
    if (!r || c >= r->npages.size() || (r->npages[c] && !dst)) return BJ_ERR_INVALID;
    if (const int st = bj_result_wait(const_cast<bj_result*>(r))) return st;
    for (uint64_t p = 0; p < r->npages[c]; p++) {
        if (!dst[p]) return BJ_ERR_INVALID;
        if (r->host.p) {
            std::memcpy(dst[p], r->host.p + (r->page_base[c] + p) * kPageSize, kPageSize);
        } else if (r->dev) {
            if (cudaMemcpy(dst[p], r->dev + (r->page_base[c] + p) * kPageSize, kPageSize, cudaMemcpyDeviceToHost) !=
                cudaSuccess)
                return BJ_ERR_CUDA;
        } else {
            return BJ_ERR_INVALID;
        }
    }
    return BJ_OK;
}
BJ_API int bj_result_stats(const bj_result* r, bj_stats* out) {
    if (!r || !out) return BJ_ERR_INVALID;
    if (const int st = bj_result_wait(const_cast<bj_result*>(r))) return st;
    *out = r->stats;
    return BJ_OK;
}
BJ_API void bj_result_free(bj_result* r) {
    if (!r) return;
    bj_result_wait(r);
    if (r->ctx) {
        if (r->dev) {
            r->ctx->release_device(r->dev);
            r->dev = nullptr;
        }
        if (r->host.p) r->ctx->give_pinned(r->host);
        r->ctx->live_results--;
    }
    delete r;
}

} // extern "C"

