// Host planner (see planner.h).
#include "planner.h"

#include <algorithm>
#include <cstdlib>
#include <functional>
#include <limits>
#include <numeric>
#include <queue>

namespace bj {
namespace {

struct UnionFind {
    std::vector<uint32_t> p;
    uint32_t add() {
        p.push_back(uint32_t(p.size()));
        return p.back();
    }
    uint32_t find(uint32_t x) {
        while (p[x] != x) x = p[x] = p[p[x]];
        return x;
    }
    void merge(uint32_t a, uint32_t b) { p[find(a)] = find(b); }
};

struct Edge {
    uint32_t a, b;            // inputs
    uint32_t attr_a, attr_b;  // attrs of a and b
};

struct Importer {
    const bj_plan& plan;
    ExecPlan& ex;
    UnionFind uf;
    std::vector<Edge> edges;
    std::string err;
    int status = BJ_OK;

    bool fail(int st, std::string msg) {
        if (status == BJ_OK) {
            status = st;
            err = std::move(msg);
        }
        return false;
    }

    // Output attribute list of a node, as global attr ids
    // (engine/query/PlanImport.cpp:24-57 walks the tree the same way).
    bool rec(uint64_t id, std::vector<uint32_t>& out, int depth) {
        if (id >= plan.num_nodes) return fail(BJ_ERR_INVALID, "plan node index out of range");
        if (depth > 1024) return fail(BJ_ERR_INVALID, "plan is too deep or cyclic");
        const bj_node& n = plan.nodes[id];
        if (n.num_output_attrs && !n.output_attrs) return fail(BJ_ERR_INVALID, "missing output attributes");
        if (n.kind == BJ_NODE_SCAN) {
            if (n.base_table_id >= plan.num_inputs) return fail(BJ_ERR_INVALID, "scan of a missing input table");
            const bj_table& t = plan.inputs[n.base_table_id];
            if (t.num_rows >= (1ull << 32) - 2) return fail(BJ_ERR_UNSUPPORTED, "tables are limited to 2^32-2 rows");
            uint32_t in = uint32_t(ex.inputs.size());
            ex.inputs.push_back(PlanInput{uint32_t(n.base_table_id), t.num_rows, {}});
            for (uint64_t a = 0; a < n.num_output_attrs; a++) {
                const bj_attr& at = n.output_attrs[a];
                if (at.type < BJ_INT32 || at.type > BJ_VARCHAR) return fail(BJ_ERR_INVALID, "unknown attribute type");
                if (t.num_rows) {
                    if (at.index >= t.num_columns) return fail(BJ_ERR_INVALID, "scan attribute beyond the table's columns");
                    if (t.columns[at.index].type != at.type)
                        return fail(BJ_ERR_INVALID, "scan attribute type differs from the column type");
                }
                uint32_t gid = uint32_t(ex.attrs.size());
                ex.attrs.push_back(PlanAttr{in, uint32_t(at.index), at.type, uf.add()});
                ex.inputs[in].attrs.push_back(gid);
                out.push_back(gid);
            }
            return true;
        }
        if (n.kind != BJ_NODE_JOIN) return fail(BJ_ERR_INVALID, "unknown plan node kind");
        std::vector<uint32_t> l, r;
        if (!rec(n.left, l, depth + 1) || !rec(n.right, r, depth + 1)) return false;
        if (n.left_attr >= l.size() || n.right_attr >= r.size()) return fail(BJ_ERR_INVALID, "join attribute out of range");
        uint32_t la = l[n.left_attr], ra = r[n.right_attr];
        // Join keys are 32-bit integers in the reference (engine/op/TableScan.cpp:328,
        // engine/op/Hashtable.hpp:35-39), which misreads any other type. Here
        // INT64 keys are joined by their full 64-bit value too (no reference
        // counterpart); both sides of a join must have the same key type.
        const int32_t lt = ex.attrs[la].type, rt = ex.attrs[ra].type;
        if (lt != rt || (lt != BJ_INT32 && lt != BJ_INT64))
            return fail(BJ_ERR_UNSUPPORTED, "join keys must be INT32 or INT64, the same type on both sides");
        uf.merge(la, ra);
        edges.push_back(Edge{ex.attrs[la].input, ex.attrs[ra].input, la, ra});
        for (uint64_t a = 0; a < n.num_output_attrs; a++) {
            uint64_t idx = n.output_attrs[a].index;
            if (idx >= l.size() + r.size()) return fail(BJ_ERR_INVALID, "join output attribute out of range");
            uint32_t g = idx < l.size() ? l[idx] : r[idx - l.size()];
            if (ex.attrs[g].type != n.output_attrs[a].type)
                return fail(BJ_ERR_INVALID, "join output attribute type mismatch");
            out.push_back(g);
        }
        return true;
    }
};

// Join order over the plan's join tree, with the reference's cost model
// (engine/query/QueryGraph.cpp:62-66, 70-87, 120-145: a join costs the
// cardinality of its result plus 10 x the cardinality of the side hashed,
// and a result's cardinality is the largest of its inputs'). The plans
// enumerated are the ones the executor runs: every pipeline is driven by a
// scan, probes only with its own columns, and builds its table keyed on one
// of its own columns, so a plan for a connected set S of inputs is fixed by
// its driver d and the order in which d's pipeline joins the branches
// hanging off d. cost[S][d] = card(d) for S = {d}; otherwise the minimum over
// the neighbours v of d in S of
//     cost[S \ L][d] + cost[L][v] + card(S) + 10 card(L),
// L being the branch of S behind the edge d-v (joined last, built with
// driver v). Subsets come in increasing numeric order, so both parts of a
// split are done before S. The reference enumerates the same connected
// pairs with DPccp (engine/query/DPccp.hpp:16-56) over equivalence-class
// neighbourhoods and caps a pipeline at two probes (QueryGraph.hpp:39); the
// executor probes any number of tables per pipeline, so there is no cap.
// Returns the driver of the cheapest full plan (ties: the larger input,
// then the lower index); `cost` receives its cost. Plans over more than
// kMaxDpInputs inputs take the largest input.
constexpr uint32_t kMaxDpInputs = 14;

uint32_t choose_driver(const std::vector<double>& card, const std::vector<Edge>& edges, double& cost,
                       const std::vector<double>* set_card = nullptr, int forced_driver = -1) {
    const uint32_t n = uint32_t(card.size());
    uint32_t largest = 0;
    for (uint32_t i = 1; i < n; i++)
        if (card[i] > card[largest]) largest = i;
    cost = -1;
    if (n == 1 || n > kMaxDpInputs) return forced_driver >= 0 ? uint32_t(forced_driver) : largest;
    std::vector<uint32_t> nbr(n, 0);
    for (const Edge& e : edges) {
        nbr[e.a] |= 1u << e.b;
        nbr[e.b] |= 1u << e.a;
    }
    // Vertices reachable from `v` inside `set`.
    auto reach = [&](uint32_t v, uint32_t set) {
        uint32_t seen = 1u << v, frontier = seen;
        while (frontier) {
            uint32_t next = 0;
            for (uint32_t f = frontier; f; f &= f - 1) next |= nbr[__builtin_ctz(f)];
            next &= set & ~seen;
            seen |= next;
            frontier = next;
        }
        return seen;
    };
    const uint32_t full = n == 32 ? ~0u : (1u << n) - 1;
    const double inf = std::numeric_limits<double>::infinity();
    std::vector<double> best(size_t(full + 1) * n, inf);
    std::vector<double> setcard(full + 1, 0.0);
    for (uint32_t S = 1; S <= full; S++) {
        const uint32_t low = __builtin_ctz(S);
        setcard[S] = std::max(setcard[S & (S - 1)], card[low]);
        if (S == (1u << low)) {
            best[size_t(S) * n + low] = set_card ? (*set_card)[S] : card[low];
            if (set_card) setcard[S] = (*set_card)[S];
            continue;
        }
        if (reach(low, S) != S) continue;  // not connected
        if (set_card) setcard[S] = (*set_card)[S];
        for (uint32_t ds = S; ds; ds &= ds - 1) {
            const uint32_t d = __builtin_ctz(ds);
            double c = inf;
            for (uint32_t vs = nbr[d] & S; vs; vs &= vs - 1) {
                const uint32_t v = __builtin_ctz(vs);
                const uint32_t L = reach(v, S & ~(1u << d));
                const uint32_t R = S & ~L;
                const double cr = best[size_t(R) * n + d], cl = best[size_t(L) * n + v];
                if (cr == inf || cl == inf) continue;
                c = std::min(c, cr + cl + setcard[S] + 10.0 * setcard[L]);
            }
            best[size_t(S) * n + d] = c;
        }
    }
    uint32_t driver = largest;
    for (uint32_t d = 0; d < n; d++) {
        const double c = best[size_t(full) * n + d], cb = best[size_t(full) * n + driver];
        if (c < cb || (c == cb && (card[d] > card[driver] || (card[d] == card[driver] && d < driver)))) driver = d;
    }
    if (forced_driver >= 0 && uint32_t(forced_driver) < n) driver = uint32_t(forced_driver);
    cost = best[size_t(full) * n + driver];
    return driver;
}

// The reference's own dynamic program over its plan space, for comparison
// (engine/query/QueryGraph.cpp:107-216 with DPccp, DPccp.hpp:16-56): a plan for
// a connected set of inputs and a count of probes in its top pipeline (0-2,
// maxPipelineLength = 3, QueryGraph.hpp:39); joining `left` as a hash table into
// the pipeline of `right` adds card(left + right) + 10 card(left) and one probe
// (consider, QueryGraph.cpp:90-108). Its pipelines may probe with an earlier
// probe's payload, which the executor does not run, and probe at most twice,
// which the executor does not need. On a tree of join edges, the pairs DPccp
// enumerates are the two sides of each edge of a connected set. Returns the
// cheapest full plan's cost, or -1 above kMaxDpInputs inputs.
// `plan_text` (optional) receives the cheapest plan in the notation
// probe(R, hash(L)): input R's pipeline (or the pipeline of plan R) probes the
// hash table built from plan L. `tree` (optional) receives it as nodes: a
// base input (probes == 0) or probe(right, hash(left)); node 0 is the root.
// `set_card` (optional) gives every connected set's cardinality, as for
// choose_driver.
struct RefNode {
    uint32_t set;
    int probes;          // probes in this node's top pipeline; 0: a base input
    int32_t left = -1;   // hashed plan
    int32_t right = -1;  // plan whose pipeline continues
};

double reference_dp_cost(const std::vector<double>& card, const std::vector<Edge>& edges,
                         std::string* plan_text = nullptr, const std::vector<double>* set_card = nullptr,
                         std::vector<RefNode>* tree = nullptr) {
    const uint32_t n = uint32_t(card.size());
    if (n == 0 || n > kMaxDpInputs) return -1;
    if (n == 1) {
        if (plan_text) *plan_text = "input 0";
        if (tree) *tree = {RefNode{1u, 0, -1, -1}};
        return card[0];
    }
    std::vector<uint32_t> nbr(n, 0);
    for (const Edge& e : edges) {
        nbr[e.a] |= 1u << e.b;
        nbr[e.b] |= 1u << e.a;
    }
    auto reach = [&](uint32_t v, uint32_t set) {
        uint32_t seen = 1u << v, frontier = seen;
        while (frontier) {
            uint32_t next = 0;
            for (uint32_t f = frontier; f; f &= f - 1) next |= nbr[__builtin_ctz(f)];
            next &= set & ~seen;
            seen |= next;
            frontier = next;
        }
        return seen;
    };
    constexpr int kPipes = 3;
    const uint32_t full = (1u << n) - 1;
    const double inf = std::numeric_limits<double>::infinity();
    std::vector<double> best(size_t(full + 1) * kPipes, inf), setcard(full + 1, 0.0);
    struct Choice {
        uint32_t left = 0, right = 0;
        int lpipes = 0, rpipes = 0;
    };
    std::vector<Choice> how(plan_text || tree ? size_t(full + 1) * kPipes : 0);
    for (uint32_t S = 1; S <= full; S++) {
        const uint32_t low = __builtin_ctz(S);
        setcard[S] = std::max(setcard[S & (S - 1)], card[low]);
        if (S == (1u << low)) {
            if (set_card) setcard[S] = (*set_card)[S];
            best[size_t(S) * kPipes] = setcard[S];  // a base relation costs its cardinality
            continue;
        }
        if (reach(low, S) != S) continue;
        if (set_card) setcard[S] = (*set_card)[S];
        // Each edge of S splits it into two connected sides; either side can
        // be the hash table joined into the other's pipeline.
        for (uint32_t us = S; us; us &= us - 1) {
            const uint32_t u = __builtin_ctz(us);
            for (uint32_t vs = nbr[u] & S; vs; vs &= vs - 1) {
                const uint32_t v = __builtin_ctz(vs);
                if (v < u) continue;  // each edge once
                const uint32_t A = reach(v, S & ~(1u << u)), B = S & ~A;
                for (int side = 0; side < 2; side++) {
                    const uint32_t left = side ? B : A, right = side ? A : B;
                    const double base = setcard[S] + 10.0 * setcard[left];
                    double lbest = inf;
                    int lpick = 0;
                    for (int lp = 0; lp < kPipes; lp++)
                        if (best[size_t(left) * kPipes + lp] < lbest) {
                            lbest = best[size_t(left) * kPipes + lp];
                            lpick = lp;
                        }
                    for (int rp = 0; rp + 1 < kPipes; rp++) {
                        const double c = lbest + best[size_t(right) * kPipes + rp] + base;
                        double& t = best[size_t(S) * kPipes + rp + 1];
                        if (c < t) {
                            t = c;
                            if (plan_text || tree) how[size_t(S) * kPipes + rp + 1] = Choice{left, right, lpick, rp};
                        }
                    }
                }
            }
        }
    }
    double r = inf;
    int rp = 0;
    for (int p = 0; p < kPipes; p++)
        if (best[size_t(full) * kPipes + p] < r) {
            r = best[size_t(full) * kPipes + p];
            rp = p;
        }
    if (plan_text && r < inf) {
        std::function<std::string(uint32_t, int)> show = [&](uint32_t S, int p) -> std::string {
            if (p == 0) return "input " + std::to_string(__builtin_ctz(S));
            const Choice& c = how[size_t(S) * kPipes + p];
            return "probe(" + show(c.right, c.rpipes) + ", hash(" + show(c.left, c.lpipes) + "))";
        };
        *plan_text = show(full, rp);
    }
    if (tree && r < inf) {
        tree->clear();
        std::function<int32_t(uint32_t, int)> add = [&](uint32_t S, int p) -> int32_t {
            const int32_t id = int32_t(tree->size());
            tree->push_back(RefNode{S, p, -1, -1});
            if (p > 0) {
                const Choice& c = how[size_t(S) * kPipes + p];
                const int32_t l = add(c.left, c.lpipes);
                const int32_t rr = add(c.right, c.rpipes);
                (*tree)[size_t(id)].left = l;
                (*tree)[size_t(id)].right = rr;
            }
            return id;
        };
        add(full, rp);
    }
    return r;
}

// Pipelines of a plan of the reference's space (tree from reference_dp_cost).
// A node's pipeline scans the base input at the bottom of its right spine and
// probes, bottom up, the tables hashed from the left plans along the spine.
// A hashed plan's pipeline carries, as payload, every attribute of its
// inputs that is a result column or the endpoint of a join edge leaving its
// set; its build key is its endpoint of the edge to the rest of its parent's
// set. A probe's or build's key is the scanned input's column when its input
// is scanned, else the payload of the earlier probe whose set holds it.
bool reference_pipelines(ExecPlan& ex, const std::vector<Edge>& edges, const std::vector<RefNode>& tree,
                         const std::vector<uint32_t>& out_src, std::string& err) {
    std::vector<uint8_t> is_out(ex.attrs.size(), 0);
    for (uint32_t a : out_src) is_out[a] = 1;
    // The output pipeline carries each distinct result attribute once.
    std::vector<uint32_t> root_carry = out_src;
    std::sort(root_carry.begin(), root_carry.end());
    root_carry.erase(std::unique(root_carry.begin(), root_carry.end()), root_carry.end());
    // Attributes a set of inputs must hand on.
    auto needed = [&](uint32_t set) {
        std::vector<uint32_t> v;
        for (uint32_t a = 0; a < ex.attrs.size(); a++)
            if ((set >> ex.attrs[a].input & 1) && is_out[a]) v.push_back(a);
        for (const Edge& e : edges) {
            const bool ia = set >> e.a & 1, ib = set >> e.b & 1;
            if (ia && !ib) v.push_back(e.attr_a);
            if (ib && !ia) v.push_back(e.attr_b);
        }
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        return v;
    };
    // The edge between two disjoint sets (their union is connected by one edge).
    auto edge_between = [&](uint32_t x, uint32_t y, uint32_t& ax, uint32_t& ay) {
        for (const Edge& e : edges) {
            if ((x >> e.a & 1) && (y >> e.b & 1)) {
                ax = e.attr_a;
                ay = e.attr_b;
                return true;
            }
            if ((x >> e.b & 1) && (y >> e.a & 1)) {
                ax = e.attr_b;
                ay = e.attr_a;
                return true;
            }
        }
        return false;
    };
    std::vector<uint32_t> pipe_set;  // per pipeline: its input set
    // Emits node `id`'s pipeline (hashed plans first); build_key: attr of the
    // set used as its key (-1: the output pipeline). Returns its index.
    std::function<int64_t(int32_t, int64_t)> emit = [&](int32_t id, int64_t build_key) -> int64_t {
        std::vector<int32_t> hashed;  // bottom-up
        int32_t n = id;
        while (tree[size_t(n)].probes > 0) {
            hashed.push_back(tree[size_t(n)].left);
            n = tree[size_t(n)].right;
        }
        std::reverse(hashed.begin(), hashed.end());
        const uint32_t base = __builtin_ctz(tree[size_t(n)].set);
        PipelinePlan pp;
        pp.input = base;
        uint32_t have = 1u << base;
        std::vector<uint32_t> probe_sets;
        std::vector<std::vector<uint32_t>> probe_carry;
        // Where attr a is available: -1 the scanned input, else (probe, slot).
        auto locate = [&](uint32_t a, int32_t& probe, uint32_t& slot) {
            if (ex.attrs[a].input == base) {
                probe = -1;
                return true;
            }
            for (size_t k = 0; k < probe_sets.size(); k++)
                if (probe_sets[k] >> ex.attrs[a].input & 1) {
                    const auto& c = probe_carry[k];
                    const auto it = std::find(c.begin(), c.end(), a);
                    if (it == c.end()) return false;
                    probe = int32_t(k);
                    slot = uint32_t(it - c.begin());
                    return true;
                }
            return false;
        };
        for (int32_t h : hashed) {
            const uint32_t hs = tree[size_t(h)].set;
            uint32_t ah = 0, ar = 0;
            if (!edge_between(hs, have, ah, ar)) return -1;
            const int64_t child = emit(h, int64_t(ah));
            if (child < 0) return -1;
            PipelinePlan::Probe pr;
            pr.child = uint32_t(child);
            pr.probe_attr = ar;
            int32_t kp;
            uint32_t ks = 0;
            if (!locate(ar, kp, ks)) return -1;
            pr.key_probe = kp;
            pr.key_slot = ks;
            pp.probes.push_back(pr);
            probe_sets.push_back(hs);
            std::vector<uint32_t> carry;
            for (const SlotPlan& sl : ex.pipelines[size_t(child)].slots) carry.push_back(sl.attr);
            probe_carry.push_back(carry);
            have |= hs;
        }
        pp.build_key = build_key;
        if (build_key >= 0) {
            int32_t kp;
            uint32_t ks = 0;
            if (!locate(uint32_t(build_key), kp, ks)) return -1;
            pp.build_key_probe = kp;
            pp.build_key_slot = ks;
        }
        const std::vector<uint32_t> carry = build_key >= 0 ? needed(have) : root_carry;
        for (uint32_t a : carry) {
            int32_t kp;
            uint32_t ks = 0;
            if (!locate(a, kp, ks)) return -1;
            if (kp < 0)
                pp.slots.push_back(SlotPlan{0, a, 0, 0});
            else
                pp.slots.push_back(SlotPlan{1, a, uint32_t(kp), ks});
        }
        if (pp.probes.size() > 16 || pp.slots.size() > 32) return -1;
        ex.pipelines.push_back(std::move(pp));
        pipe_set.push_back(have);
        return int64_t(ex.pipelines.size() - 1);
    };
    ex.pipelines.clear();
    const int64_t root = emit(0, -1);
    if (root < 0 || size_t(root) + 1 != ex.pipelines.size()) {
        err = "internal: a plan of the reference's space has no pipelines for it";
        return false;
    }
    ex.driver = ex.pipelines.back().input;
    ex.out_slot.clear();
    const PipelinePlan& rp = ex.pipelines.back();
    for (uint32_t a : out_src)
        for (uint32_t j = 0; j < rp.slots.size(); j++)
            if (rp.slots[j].attr == a) {
                ex.out_slot.push_back(j);
                break;
            }
    if (ex.out_slot.size() != out_src.size()) {
        err = "internal: result column without a source";
        return false;
    }
    ex.reference_space = true;
    return true;
}

} // namespace

int plan_graph(const bj_plan& plan, PlanGraph& g, std::string& err) {
    g = PlanGraph{};
    ExecPlan ex;
    if (plan.num_nodes == 0 || !plan.nodes || (plan.num_inputs && !plan.inputs)) {
        err = "empty plan or missing inputs";
        return BJ_ERR_INVALID;
    }
    Importer im{plan, ex, {}, {}, {}, BJ_OK};
    std::vector<uint32_t> root_attrs;
    if (!im.rec(plan.root, root_attrs, 0)) {
        err = im.err;
        return im.status;
    }
    for (const PlanInput& in : ex.inputs) g.inputs.push_back({in.table, in.rows});
    for (const Edge& e : im.edges)
        g.edges.push_back({e.a, e.b, ex.attrs[e.attr_a].column, ex.attrs[e.attr_b].column, ex.attrs[e.attr_a].type});
    return BJ_OK;
}

int join_order(const bj_plan& plan, const std::vector<double>* set_card, int forced_driver, uint32_t& driver,
               double& cost, std::string& err) {
    ExecPlan ex;
    if (plan.num_nodes == 0 || !plan.nodes || (plan.num_inputs && !plan.inputs)) {
        err = "empty plan or missing inputs";
        return BJ_ERR_INVALID;
    }
    Importer im{plan, ex, {}, {}, {}, BJ_OK};
    std::vector<uint32_t> root_attrs;
    if (!im.rec(plan.root, root_attrs, 0)) {
        err = im.err;
        return im.status;
    }
    const uint32_t ni = uint32_t(ex.inputs.size());
    if (set_card && set_card->size() < (size_t(1) << std::min<uint32_t>(ni, 31))) {
        err = "set cardinalities: fewer than 2^inputs entries";
        return BJ_ERR_INVALID;
    }
    std::vector<double> card(ni);
    for (uint32_t i = 0; i < ni; i++) card[i] = double(ex.inputs[i].rows);
    driver = choose_driver(card, im.edges, cost, set_card, forced_driver);
    return BJ_OK;
}

PlanSpace plan_space_default() {
    static const PlanSpace space = [] {
        const char* e = std::getenv("B200JOIN_PLAN_SPACE");
        if (!e) return PlanSpace::Auto;
        const std::string v(e);
        return v == "rooted" ? PlanSpace::Rooted : v == "reference" ? PlanSpace::Reference : PlanSpace::Auto;
    }();
    return space;
}

int make_exec_plan(const bj_plan& plan, ExecPlan& ex, std::string& err, bool reference_cost,
                   const std::vector<double>* set_card, PlanSpace space) {
    ex = ExecPlan{};
    if (plan.num_nodes == 0 || !plan.nodes) {
        err = "empty plan";
        return BJ_ERR_INVALID;
    }
    if (plan.num_inputs && !plan.inputs) {
        err = "missing input tables";
        return BJ_ERR_INVALID;
    }
    Importer im{plan, ex, {}, {}, {}, BJ_OK};
    std::vector<uint32_t> root_attrs;
    if (!im.rec(plan.root, root_attrs, 0)) {
        err = im.err;
        return im.status;
    }
    // Equivalence classes.
    for (auto& a : ex.attrs) a.eq = im.uf.find(a.eq);
    const uint32_t ni = uint32_t(ex.inputs.size());
    for (uint32_t i = 0; i < ni; i++)
        if (ex.inputs[i].rows == 0) ex.empty = true;
    ex.out_types.clear();
    for (uint32_t a : root_attrs) ex.out_types.push_back(ex.attrs[a].type);
    if (ex.empty) return BJ_OK;

    // Root the join tree at the driver of the cheapest plan (cardinality of
    // an input: its row count).
    std::vector<double> card(ni);
    for (uint32_t i = 0; i < ni; i++) card[i] = double(ex.inputs[i].rows);
    if (set_card && set_card->size() < (size_t(1) << std::min<uint32_t>(ni, 31))) set_card = nullptr;
    const uint32_t driver = choose_driver(card, im.edges, ex.est_cost, set_card);
    ex.driver = driver;
    ex.rooted_driver = driver;
    ex.rooted_cost = ex.est_cost;
    if (reference_cost) ex.ref_cost = reference_dp_cost(card, im.edges, &ex.ref_plan, set_card);
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> adj(ni);  // (neighbour, edge)
    for (uint32_t e = 0; e < im.edges.size(); e++) {
        adj[im.edges[e].a].push_back({im.edges[e].b, e});
        adj[im.edges[e].b].push_back({im.edges[e].a, e});
    }
    std::vector<int64_t> parent(ni, -1), parent_edge(ni, -1), depth(ni, -1);
    std::vector<uint32_t> order;
    std::queue<uint32_t> q;
    q.push(driver);
    depth[driver] = 0;
    while (!q.empty()) {
        uint32_t x = q.front();
        q.pop();
        order.push_back(x);
        for (auto [y, e] : adj[x]) {
            if (depth[y] >= 0) continue;
            depth[y] = depth[x] + 1;
            parent[y] = x;
            parent_edge[y] = e;
            q.push(y);
        }
    }
    if (order.size() != ni) {
        err = "plan's joins do not connect all scans";
        return BJ_ERR_INVALID;
    }
    // Subtree membership: input -> root-ward chain.
    auto in_subtree = [&](uint32_t node, uint32_t top) {
        for (int64_t x = node; x >= 0; x = parent[x])
            if (uint32_t(x) == top) return true;
        return false;
    };
    // Output sources: for each result column, the member of its class whose
    // input is nearest the driver (all members are equal on result rows).
    std::vector<uint32_t> out_src;
    for (uint32_t a : root_attrs) {
        uint32_t eq = ex.attrs[a].eq, best = a;
        for (uint32_t g = 0; g < ex.attrs.size(); g++) {
            if (ex.attrs[g].eq != eq || ex.attrs[g].type != ex.attrs[a].type) continue;
            if (depth[ex.attrs[g].input] < depth[ex.attrs[best].input] ||
                (depth[ex.attrs[g].input] == depth[ex.attrs[best].input] && g < best))
                best = g;
        }
        out_src.push_back(best);
    }
    std::vector<uint32_t> distinct_src = out_src;
    std::sort(distinct_src.begin(), distinct_src.end());
    distinct_src.erase(std::unique(distinct_src.begin(), distinct_src.end()), distinct_src.end());

    // Pipelines in reverse BFS order: children before parents, driver last.
    std::vector<int64_t> pipe_of(ni, -1);
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
        uint32_t x = *it;
        PipelinePlan pp;
        pp.input = x;
        if (parent[x] >= 0) {
            const Edge& e = im.edges[parent_edge[x]];
            pp.build_key = e.a == x ? e.attr_a : e.attr_b;
        }
        for (auto [y, ei] : adj[x]) {
            if (parent[y] != int64_t(x) || parent_edge[y] != int64_t(ei)) continue;
            const Edge& e = im.edges[ei];
            pp.probes.push_back({uint32_t(pipe_of[y]), e.a == x ? e.attr_a : e.attr_b});
        }
        for (uint32_t s : distinct_src) {
            uint32_t si = ex.attrs[s].input;
            if (!in_subtree(si, x)) continue;
            if (si == x) {
                pp.slots.push_back(SlotPlan{0, s, 0, 0});
                continue;
            }
            bool found = false;
            for (uint32_t k = 0; k < pp.probes.size(); k++) {
                const PipelinePlan& child = ex.pipelines[pp.probes[k].child];
                if (!in_subtree(si, child.input)) continue;
                for (uint32_t j = 0; j < child.slots.size(); j++)
                    if (child.slots[j].attr == s) {
                        pp.slots.push_back(SlotPlan{1, s, k, j});
                        found = true;
                    }
                break;
            }
            if (!found) {
                err = "internal: payload source not found in children";
                return BJ_ERR_INTERNAL;
            }
        }
        if (pp.probes.size() > 16) {
            err = "a scan joins more than 16 inputs";
            return BJ_ERR_UNSUPPORTED;
        }
        if (pp.slots.size() > 32) {
            err = "more than 32 distinct result columns";
            return BJ_ERR_UNSUPPORTED;
        }
        pipe_of[x] = int64_t(ex.pipelines.size());
        ex.pipelines.push_back(std::move(pp));
    }
    const PipelinePlan& root = ex.pipelines.back();
    for (uint32_t s : out_src) {
        for (uint32_t j = 0; j < root.slots.size(); j++)
            if (root.slots[j].attr == s) {
                ex.out_slot.push_back(j);
                break;
            }
    }
    if (ex.out_slot.size() != out_src.size()) {
        err = "internal: result column without a source";
        return BJ_ERR_INTERNAL;
    }
    // The reference's plan space (probes and builds keyed on an earlier
    // probe's payload, at most two probes per pipeline) under the same
    // cardinalities: run its plan when it is cheaper (or when asked to).
    if (space != PlanSpace::Rooted && ni >= 2 && ni <= kMaxDpInputs) {
        std::vector<RefNode> tree;
        const double rc = reference_dp_cost(card, im.edges, nullptr, set_card, &tree);
        if (rc >= 0 && !tree.empty() &&
            (space == PlanSpace::Reference || (ex.est_cost >= 0 && rc < ex.est_cost * (1.0 - 1e-9)))) {
            ExecPlan alt = ex;
            std::string aerr;
            if (reference_pipelines(alt, im.edges, tree, root_attrs, aerr)) {
                alt.est_cost = rc;
                ex = std::move(alt);
            } else if (space == PlanSpace::Reference) {
                err = aerr;
                return BJ_ERR_INTERNAL;
            }
        }
    }
    sideways_restrictions(ex);
    return BJ_OK;
}

void sideways_restrictions(ExecPlan& ex) {
    const size_t np = ex.pipelines.size();
    // A build of an input that probes nothing, keyed on one of its INT32
    // columns, batched with the other such builds.
    auto plain_leaf = [&](const PipelinePlan& pp) {
        return pp.probes.empty() && pp.build_key >= 0 && pp.build_key_probe < 0 &&
               pp.slots.size() <= kLeafBatchMaxSlots && ex.attrs[size_t(pp.build_key)].type == BJ_INT32;
    };
    // below[p][q]: pipeline q feeds pipeline p through its probes (children
    // come before parents, so one pass in order completes every row).
    std::vector<std::vector<uint8_t>> below(np, std::vector<uint8_t>(np, 0));
    for (size_t p = 0; p < np; p++)
        for (const auto& pr : ex.pipelines[p].probes) {
            below[p][pr.child] = 1;
            for (size_t q = 0; q < np; q++) below[p][q] |= below[pr.child][q];
        }
    for (size_t m = 0; m + 1 < np; m++) {
        PipelinePlan& pm = ex.pipelines[m];
        pm.restrict_by = -1;
        const bool leaf = plain_leaf(pm);
        // A build fed by probes runs after every batched leaf and pays only
        // a filter test per tuple; a leaf restricted pays a second batch.
        if (!leaf && (pm.probes.empty() || pm.build_key < 0 || ex.attrs[size_t(pm.build_key)].type != BJ_INT32))
            continue;
        const uint64_t rows_m = ex.inputs[pm.input].rows;
        if (leaf && rows_m < kSidewaysMinRows) continue;
        const uint32_t eq = ex.attrs[size_t(pm.build_key)].eq;
        // The smallest qualifying provider (never itself restricted: any
        // input that could restrict it would qualify here and be smaller).
        uint64_t best_rows = 0;
        for (size_t l = 0; l + 1 < np; l++) {
            const PipelinePlan& pl = ex.pipelines[l];
            if (l == m || below[m][l] || !plain_leaf(pl) || ex.attrs[size_t(pl.build_key)].eq != eq) continue;
            const uint64_t rows_l = ex.inputs[pl.input].rows;
            if (rows_l > kSidewaysMaxFilterRows || rows_l * 4 > rows_m) continue;
            if (pm.restrict_by < 0 || rows_l < best_rows || (rows_l == best_rows && int32_t(l) < pm.restrict_by)) {
                pm.restrict_by = int32_t(l);
                best_rows = rows_l;
            }
        }
    }
}

} // namespace bj
