// Host planner: turns a contest plan into device pipelines.
//
// The reference imports the plan into attribute equivalence classes
// (engine/query/PlanImport.cpp:24-89), ignores the given join order and build
// sides, and re-plans incrementally with DPccp over sampled cardinalities,
// running at most three operators per pipeline (engine/query/QueryPlan.cpp:
// 748-794, QueryGraph.cpp:107-216). Here the same equivalence classes are
// built, then the join tree over the scans is rooted at the driver of the
// cheapest plan under the reference's cost model (a dynamic program over
// connected sets of inputs and their drivers, planner.cpp: choose_driver):
// every other input becomes one build pipeline whose hash table
// is keyed on the class that links it to its parent, carrying the payload
// columns its ancestors still need; the driver's pipeline probes its children
// and writes the result. A pipeline may probe any number of children (the
// GPU has no reason to cap it at two) and the probe order inside a pipeline
// is chosen at run time from sampled hit rates (engine/query/QueryPlan.cpp:
// 719-746 samples 64 rows per table for the same purpose).
#pragma once

#include "../../include/b200join.h"

#include <cstdint>
#include <string>
#include <vector>

namespace bj {

struct PlanAttr {
    uint32_t input;   // scan index
    uint32_t column;  // base column
    int32_t type;
    uint32_t eq;      // equivalence class
};

struct PlanInput {
    uint32_t table;                // base table id
    uint64_t rows;
    std::vector<uint32_t> attrs;   // global attribute ids of this scan
};

// One value slot of a pipeline: a column of the scanned input, or a payload
// slot of a probed child's hash table.
struct SlotPlan {
    int kind;         // 0: attr of the scanned input, 1: child payload
    uint32_t attr;    // source attribute (global id), for both kinds
    uint32_t probe;   // kind 1: index into Pipeline::probes
    uint32_t slot;    // kind 1: slot in that child's table
};

struct PipelinePlan {
    uint32_t input;
    int64_t build_key = -1;  // attr id of the hash key; -1 for the output pipeline
    // The build key comes from payload slot build_key_slot of probe
    // build_key_probe when that is >= 0 (an attribute of an input this
    // pipeline probed), else from the scanned input's column.
    int32_t build_key_probe = -1;
    uint32_t build_key_slot = 0;
    struct Probe {
        uint32_t child;       // pipeline index of the child
        uint32_t probe_attr;  // attr whose values probe the child's table
        // key_probe >= 0: probe_attr is carried as payload slot key_slot of
        // the table probed by probes[key_probe] (which must run earlier);
        // otherwise it is a column of `input`.
        int32_t key_probe = -1;
        uint32_t key_slot = 0;
    };
    std::vector<Probe> probes;
    std::vector<SlotPlan> slots;  // payload (build) or output sources (root)
    // A sideways restriction (sideways_restrictions): the pipeline of a much
    // smaller build that probes nothing, keyed on the same equivalence class
    // as this build and not below it, whose bloom filter drops this build's
    // tuples with keys it cannot hold; -1: none.
    int32_t restrict_by = -1;
};

struct ExecPlan {
    std::vector<PlanInput> inputs;
    std::vector<PlanAttr> attrs;
    std::vector<PipelinePlan> pipelines;  // children before parents; last = root
    std::vector<uint32_t> out_slot;       // result column -> slot of the root pipeline
    std::vector<int32_t> out_types;
    bool empty = false;                   // some input has no rows
    uint32_t driver = 0;                  // input scanned by the output pipeline
    double est_cost = -1;                 // cost of the chosen plan (-1: not costed)
    double rooted_cost = -1;              // the cheapest rooted plan's cost, and its driver
    uint32_t rooted_driver = 0;
    double ref_cost = -1;                 // the cheapest plan of the reference's plan space, same cost model
    std::string ref_plan;                 // that plan, as probe(R, hash(L)) over input indices
    // The pipelines run are the reference space's plan (probes and builds
    // may be keyed on an earlier probe's payload) rather than a rooted tree.
    bool reference_space = false;
};

// Sideways restrictions (the reference installs a finished table's Join
// restriction on every later scan of another input of its key class,
// engine/query/QueryPlan.cpp:620-624, :670-676; buildScan applies it,
// :113-126). A tuple of a build whose key a table of the same class cannot
// hold joins no result row, so a build is restricted by the bloom filter of
// a smaller input that probes nothing (a leaf, built before every pipeline
// that probes), built on that class and not below the restricted build.
// The provider is small enough to carry a filter (kSidewaysMaxFilterRows
// rows at most) and has at most a quarter of the restricted input's rows;
// both keys INT32; the leaf is batched (kLeafBatchMaxSlots payload columns
// at most). A restricted leaf costs a second batch of leaf builds, so leaves
// are restricted only from kSidewaysMinRows rows on; a build fed by probes
// runs after every leaf anyway and pays one filter test per tuple.
constexpr uint64_t kSidewaysMinRows = uint64_t(1) << 18;
constexpr uint64_t kSidewaysMaxFilterRows = uint64_t(1) << 17;
constexpr size_t kLeafBatchMaxSlots = 4;
void sideways_restrictions(ExecPlan& ex);

// Which plan space make_exec_plan runs: the cheaper of the two (auto), or
// one of them (for tests and measurements; B200JOIN_PLAN_SPACE=rooted /
// reference overrides auto).
enum class PlanSpace { Auto = 0, Rooted = 1, Reference = 2 };
PlanSpace plan_space_default();

// Builds the execution plan; returns BJ_OK or a status with `err` set.
// reference_cost: also cost the reference's plan space (ExecPlan::ref_cost;
// for bj_plan_explain, not needed to run the plan).
// set_card (optional): estimated cardinality of every set of inputs, indexed
// by the bit mask of its inputs (inputs numbered in scan order, see
// PlanGraph), 2^n entries; entries of sets that are not connected are never
// read. Without it, a set's cardinality is its largest input's row count
// (the reference's model, engine/query/QueryGraph.cpp:53-68).
int make_exec_plan(const bj_plan& plan, ExecPlan& out, std::string& err, bool reference_cost = false,
                   const std::vector<double>* set_card = nullptr, PlanSpace space = plan_space_default());

// The join graph of a plan: its scans (inputs, numbered in the order a
// depth-first walk from the root reaches them, left child first) and one
// edge per join node. A plan's joins always form a tree over its scans.
struct PlanGraph {
    struct Input {
        uint32_t table;  // base table id
        uint64_t rows;
    };
    struct Edge {
        uint32_t a, b;          // inputs
        uint32_t col_a, col_b;  // base columns of a and b joined
        int32_t type;           // key type (both sides)
    };
    std::vector<Input> inputs;
    std::vector<Edge> edges;
};
int plan_graph(const bj_plan& plan, PlanGraph& g, std::string& err);

// Join order under the given set cardinalities (as make_exec_plan's
// set_card; null: the reference's row-count model): the executor's cheapest
// driver and its cost. With `forced_driver` >= 0, the cost of the cheapest
// plan that driver roots instead. Plans of more than 14 inputs are not
// costed (cost -1, the largest input drives).
int join_order(const bj_plan& plan, const std::vector<double>* set_card, int forced_driver, uint32_t& driver,
               double& cost, std::string& err);

} // namespace bj
