// Host-side chain model, propagator codes, analyzer and scheduler.
// Reference behaviour followed (Langevin_FTS paths):
//   Polymer           src/common/Polymer.cpp:14-187
//   Molecules         src/common/Molecules.cpp:14-50
//   propagator codes  src/common/PropagatorCode.cpp:19-290
//   analyzer          src/common/PropagatorAnalyzer.cpp:14-470
//   scheduler         src/common/Scheduler.cpp:11-254
//   box               src/common/ComputationBox.cpp:10-308
#include "lfts_host.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <iostream>
#include <sstream>
#include <stack>

namespace lfts {

// ================================================================ codes
namespace code {

std::string key_from_code(const std::string &c) {
    // strip the trailing segment count: keep up to the last letter
    size_t end = c.size();
    while (end > 0 && !std::isalpha((unsigned char)c[end - 1])) end--;
    return c.substr(0, end);
}

std::vector<std::tuple<std::string, int, int>> deps_from_key(const std::string &key) {
    // Scan the top nesting level only: "<sub key><n>[:<repeat>]" items,
    // separated by ',' inside '[...]' keys (PropagatorCode.cpp:132-214).
    std::vector<std::tuple<std::string, int, int>> deps;
    std::vector<char> open;
    enum { KEY, COUNT, REPEAT } st = KEY;
    size_t mark = 1;
    std::string sub;
    int nseg = 0;
    for (size_t i = 0; i < key.size(); i++) {
        const char ch = key[i];
        const bool digit = std::isdigit((unsigned char)ch) != 0;
        if (open.size() == 1) {
            if (st == KEY && digit) {
                if (key[mark] == ',') mark++;
                sub = key.substr(mark, i - mark);
                st = COUNT;
                mark = i;
            } else if (st == COUNT && ch == ':') {
                nseg = std::stoi(key.substr(mark, i - mark));
                st = REPEAT;
                mark = i + 1;
            } else if (st == COUNT && !digit) {
                nseg = std::stoi(key.substr(mark, i - mark));
                deps.emplace_back(sub, nseg, 1);
                st = KEY;
                mark = i;
            } else if (st == REPEAT && !digit) {
                deps.emplace_back(sub, nseg, std::stoi(key.substr(mark, i - mark)));
                st = KEY;
                mark = i;
            }
        }
        if (ch == '(' || ch == '[') {
            open.push_back(ch);
        } else if (ch == ')' || ch == ']') {
            if (open.empty() || (open.back() == '(') != (ch == ')')) LFTS_THROW("Failed to match parentheses or braces.");
            open.pop_back();
        }
    }
    return deps;
}

std::string monomer_type_from_key(const std::string &key) {
    size_t start = 0;
    for (size_t i = key.size(); i > 0; i--) {
        const char ch = key[i - 1];
        if (ch == ')' || ch == ']' || ch == '}') { start = i; break; }
    }
    return key.substr(start);
}

std::string q_input_from_key(const std::string &key) {
    if (key.empty() || key[0] != '{') LFTS_THROW("There is no related initial condition in key (" + key + ").");
    const size_t close = key.rfind('}');
    return key.substr(1, close - 1);
}

int height_from_key(const std::string &key) {
    int h = 0;
    while (h < (int)key.size() && (key[h] == '[' || key[h] == '(')) h++;
    return h;
}

}  // namespace code

bool ComparePropagatorKey::operator()(const std::string &a, const std::string &b) const {
    const int ha = code::height_from_key(a), hb = code::height_from_key(b);
    if (ha != hb) return ha < hb;
    return a > b;
}

// ================================================================ Polymer
namespace {
// Memoised code of the propagator entering block (in_node, out_node) from the
// in_node side: sorted child codes in parentheses (or {q_init} at a marked free
// end), then monomer type and segment count (PropagatorCode.cpp:54-115).
std::string edge_code(std::map<std::pair<int, int>, std::string> &memo, Polymer &pc,
                      const std::map<int, std::string> &q_init, int in_node, int out_node) {
    const auto hit = memo.find({in_node, out_node});
    if (hit != memo.end()) return hit->second;
    std::vector<std::string> children;
    for (int nb : pc.get_adjacent_nodes()[in_node]) {
        if (nb == out_node) continue;
        std::string c;
        const auto m = memo.find({nb, in_node});
        if (m != memo.end()) {
            c = m->second;
        } else {
            c = edge_code(memo, pc, q_init, nb, in_node);
            memo[{nb, in_node}] = c;
        }
        children.push_back(c);
    }
    std::string out;
    if (!children.empty()) {
        std::sort(children.begin(), children.end());
        out = "(";
        for (auto &c : children) out += c;
        out += ")";
    } else {
        const auto q = q_init.find(in_node);
        if (q != q_init.end()) out = "{" + q->second + "}";
    }
    const Block &b = pc.get_blocks()[pc.get_block_indexes()[{in_node, out_node}]];
    out += b.monomer_type + std::to_string(b.n_segment);
    memo[{in_node, out_node}] = out;
    return out;
}
}  // namespace

Polymer::Polymer(double ds, const std::map<std::string, double> &bond_lengths, double volume_fraction,
                 const std::vector<BlockInput> &inputs, const std::map<int, std::string> &q_init) {
    for (const auto &kv : bond_lengths) {
        if (!std::all_of(kv.first.begin(), kv.first.end(), [](unsigned char c) { return std::isalpha(c) || c == '_'; }))
            LFTS_THROW("\"" + kv.first + "\" is an invalid monomer_type name. Only alphabets and underscore(_) are allowed.");
        if (kv.second <= 0) LFTS_THROW("bond_lengths[\"" + kv.first + "\"] must be a positive number.");
    }
    for (size_t i = 0; i < inputs.size(); i++) {
        const auto &b = inputs[i];
        if (b.contour_length <= 0)
            LFTS_THROW("block_inputs[" + std::to_string(i) + "].contour_lengths (" + std::to_string(b.contour_length) +
                       ") must be a positive number.");
        if (std::abs(std::lround(b.contour_length / ds) - b.contour_length / ds) > 1.e-6)
            LFTS_THROW("block_inputs[" + std::to_string(i) + "].contour_lengths/ds (" + std::to_string(b.contour_length) +
                       "/" + std::to_string(ds) + ") is not an integer.");
        if (bond_lengths.count(b.monomer_type) == 0)
            LFTS_THROW("block_inputs[" + std::to_string(i) + "].monomer_type (\"" + b.monomer_type + "\") is not in bond_lengths.");
    }
    if (inputs.empty()) LFTS_THROW("A polymer needs at least one block.");
    q_init_ = q_init;
    volume_fraction_ = volume_fraction;
    for (const auto &b : inputs)
        blocks_.push_back({b.monomer_type, (int)std::lround(b.contour_length / ds), b.contour_length, b.v, b.u});
    alpha_ = 0.0;
    for (const auto &b : blocks_) alpha_ += b.contour_length;

    for (size_t i = 0; i < inputs.size(); i++) {
        const int v = inputs[i].v, u = inputs[i].u;
        adjacent_[v].push_back(u);
        adjacent_[u].push_back(v);
        if (v < 0) LFTS_THROW("v[" + std::to_string(i) + "] (" + std::to_string(v) + ") must be a non-negative integer.");
        if (u < 0) LFTS_THROW("u[" + std::to_string(i) + "] (" + std::to_string(u) + ") must be a non-negative integer.");
        if (v == u) LFTS_THROW("v[" + std::to_string(i) + "] and u[" + std::to_string(i) + "] must be different integers.");
    }
    for (size_t i = 0; i < inputs.size(); i++) {
        const int v = inputs[i].v, u = inputs[i].u;
        if (edge_index_.count({v, u}))
            LFTS_THROW("There are duplicated edges. Please check the edge between (" + std::to_string(v) + ", " +
                       std::to_string(u) + ").");
        edge_index_[{v, u}] = (int)i;
        edge_index_[{u, v}] = (int)i;
    }
    // depth-first walk from the first block's v: a revisited non-parent node
    // closes a cycle; nodes never reached are isolated
    std::map<int, bool> seen;
    for (const auto &b : inputs) { seen[b.v] = false; seen[b.u] = false; }
    std::stack<std::pair<int, int>> todo;
    todo.push({inputs[0].v, -1});
    while (!todo.empty()) {
        const int cur = todo.top().first, parent = todo.top().second;
        todo.pop();
        seen[cur] = true;
        const std::vector<int> nbs = adjacent_[cur];
        for (int nb : nbs) {
            if (seen[nb] && nb != parent)
                LFTS_THROW("A cycle is detected, which contains nodes " + std::to_string(nb) + " and " +
                           std::to_string(parent) + ". Only acyclic branched polymers are allowed.");
            if (!seen[nb]) todo.push({nb, cur});
        }
    }
    std::set<int> isolated;
    for (const auto &b : inputs) {
        if (!seen[b.v]) isolated.insert(b.v);
        if (!seen[b.u]) isolated.insert(b.u);
    }
    if (!isolated.empty()) {
        std::string msg = "There is no route from node " + std::to_string(inputs[0].v) + " to nodes: ";
        bool first = true;
        for (int n : isolated) { msg += (first ? "" : ", ") + std::to_string(n); first = false; }
        LFTS_THROW(msg + ".");
    }
    std::map<std::pair<int, int>, std::string> memo;
    for (const auto &b : blocks_) {
        edge_key_[{b.v, b.u}] = code::key_from_code(edge_code(memo, *this, q_init_, b.v, b.u));
        edge_key_[{b.u, b.v}] = code::key_from_code(edge_code(memo, *this, q_init_, b.u, b.v));
    }
}

Block &Polymer::get_block(int v, int u) { return blocks_[get_block_index_from_edge(v, u)]; }

int Polymer::get_n_segment_total() const {
    int n = 0;
    for (const auto &b : blocks_) n += b.n_segment;
    return n;
}

int Polymer::get_block_index_from_edge(int v, int u) {
    const auto it = edge_index_.find({v, u});
    if (it == edge_index_.end()) LFTS_THROW("There is no such edge (" + std::to_string(v) + ", " + std::to_string(u) + ").");
    return it->second;
}

std::string Polymer::get_propagator_key(int v, int u) {
    const auto it = edge_key_.find({v, u});
    if (it == edge_key_.end())
        LFTS_THROW("There is no such block (v, u): (" + std::to_string(v) + ", " + std::to_string(u) + ").");
    return it->second;
}

// ================================================================ Molecules
Molecules::Molecules(std::string model, double ds, const std::map<std::string, double> &bond_lengths) {
    std::transform(model.begin(), model.end(), model.begin(), [](unsigned char c) { return std::tolower(c); });
    if (model != "continuous" && model != "discrete")
        LFTS_THROW(model + " is an invalid chain model. This must be 'Continuous' or 'Discrete'.");
    model_ = model;
    ds_ = ds;
    bonds_ = bond_lengths;
}

void Molecules::add_polymer(double vf, const std::vector<BlockInput> &blocks, const std::map<int, std::string> &q_init) {
    polymers_.emplace_back(ds_, bonds_, vf, blocks, q_init);
}

void Molecules::add_solvent(double vf, const std::string &monomer_type) { solvents_.emplace_back(vf, monomer_type); }

Polymer &Molecules::get_polymer(int p) {
    if (p < 0 || p >= (int)polymers_.size()) LFTS_THROW("Index (" + std::to_string(p) + ") is out of range.");
    return polymers_[p];
}

// ================================================================ analyzer
PropagatorAnalyzer::PropagatorAnalyzer(Molecules *molecules, bool aggregate) {
    if (molecules->get_n_polymer_types() == 0) LFTS_THROW("There is no chain. Add polymers first.");
    aggregate_ = aggregate;
    model_ = molecules->get_model_name();
    for (int p = 0; p < molecules->get_n_polymer_types(); p++) add_polymer(molecules->get_polymer(p), p);
}

static bool is_junction(Polymer &pc, int node) { return pc.get_adjacent_nodes()[node].size() != 1; }

void PropagatorAnalyzer::add_polymer(Polymer &pc, int polymer_id) {
    // left key >= right key for every block (PropagatorAnalyzer.cpp:41-168)
    std::map<std::string, RightMap> per_polymer;
    std::map<std::tuple<int, int>, std::string> vu_right;
    const std::vector<Block> blocks = pc.get_blocks();
    for (const auto &b : blocks) {
        int v = b.v, u = b.u;
        std::string kl = pc.get_propagator_key(v, u), kr = pc.get_propagator_key(u, v);
        if (kl < kr) {
            kl.swap(kr);
            std::swap(v, u);
        }
        ComputationBlock &cb = per_polymer[kl][kr];
        cb.monomer_type = b.monomer_type;
        cb.n_segment_right = b.n_segment;
        cb.n_segment_left = b.n_segment;
        cb.v_u.emplace_back(v, u);
        cb.n_repeated = (int)cb.v_u.size();
        vu_right[std::make_tuple(v, u)] = kr;
    }
    int total = 0;
    for (const auto &b : blocks) {
        if (model_ == "continuous") {
            total += b.n_segment;
        } else {
            total += b.n_segment - 1;
            if (is_junction(pc, b.v)) total++;
            if (is_junction(pc, b.u)) total++;
        }
    }
    total_segments_.push_back(total);

    if (aggregate_) {
        std::map<std::string, std::vector<std::string>> aggregated;
        // entries created while walking are visited when they sort later,
        // exactly like iterating a std::map that grows
        for (auto it = per_polymer.begin(); it != per_polymer.end(); ++it) {
            const std::string left = it->first;
            RightMap set_I = aggregate_common(it->second, model_ == "continuous" ? 0 : 1);
            per_polymer[left] = set_I;
            for (const auto &r : set_I)
                if (r.first[0] == '[' && r.second.n_segment_right == r.second.n_segment_left) aggregated[left].push_back(r.first);
            substitute_right_keys(pc, vu_right, per_polymer, aggregated, left);
        }
    }

    for (const auto &l : per_polymer) {
        for (const auto &r : l.second) {
            const std::string &kv = l.first, &ku = r.first;
            ComputationBlock &cb = blocks_[std::make_tuple(polymer_id, kv, ku)];
            cb.monomer_type = code::monomer_type_from_key(kv);
            cb.n_segment_right = r.second.n_segment_right;
            cb.n_segment_left = r.second.n_segment_left;
            cb.v_u = r.second.v_u;
            cb.n_repeated = r.second.n_repeated;
            const bool junction_left = code::height_from_key(kv) > 0;
            const bool junction_right = code::height_from_key(ku) > 0;
            update_propagator(kv, r.second.n_segment_left, junction_right);
            update_propagator(ku, r.second.n_segment_right, junction_left);
        }
    }
}

// Superpose right propagators of one left key that share n_segment_right
// (PropagatorAnalyzer.cpp:211-324).  The floor on the remaining segments is
// kept across groups once a same-monomer group lowered it, as the reference does.
PropagatorAnalyzer::RightMap PropagatorAnalyzer::aggregate_common(RightMap set_I, int minimum) {
    std::set<int> lengths;
    for (const auto &r : set_I) lengths.insert(r.second.n_segment_right);
    for (const int n_cur : lengths) {
        std::map<std::string, ComputationBlock, ComparePropagatorKey> group;
        for (const auto &r : set_I)
            if (r.second.n_segment_right == n_cur) group[r.first] = r.second;
        if (group.size() == 1 || n_cur < 2 * minimum) continue;
        const std::string mtype = code::monomer_type_from_key(group.begin()->second.monomer_type);
        bool same = true;
        for (auto it = group.rbegin(); it != group.rend(); ++it)
            if (it->second.monomer_type != mtype) same = false;
        if (same) minimum = 0;
        for (const auto &r : group) set_I[r.first].n_segment_right = minimum;
        std::vector<std::tuple<int, int>> vu;
        std::string key = "[";
        bool first = true;
        for (auto it = group.rbegin(); it != group.rend(); ++it) {
            const std::string &dep = it->first;
            if (!first) key += ",";
            first = false;
            key += dep + std::to_string(set_I[dep].n_segment_right);
            if (set_I[dep].n_repeated > 1) key += ":" + std::to_string(set_I[dep].n_repeated);
            vu.insert(vu.end(), set_I[dep].v_u.begin(), set_I[dep].v_u.end());
        }
        key += "]" + mtype;
        ComputationBlock &nb = set_I[key];
        nb.monomer_type = mtype;
        nb.n_segment_right = n_cur - minimum;
        nb.n_segment_left = n_cur - minimum;
        nb.v_u = vu;
        nb.n_repeated = 1;
    }
    return set_I;
}

// Re-key the blocks hanging below an aggregated block (PropagatorAnalyzer.cpp:330-407).
void PropagatorAnalyzer::substitute_right_keys(Polymer &pc, std::map<std::tuple<int, int>, std::string> &vu_right,
                                               std::map<std::string, RightMap> &per_polymer,
                                               std::map<std::string, std::vector<std::string>> &aggregated,
                                               const std::string &left) {
    for (size_t a = 0; a < aggregated[left].size(); a++) {
        const std::string agg = aggregated[left][a];
        ComputationBlock &blk = per_polymer[left][agg];
        for (size_t e = 0; e < blk.v_u.size(); e++) {
            const int v = std::get<0>(blk.v_u[e]), u = std::get<1>(blk.v_u[e]);
            std::vector<int> nbs = pc.get_adjacent_nodes()[v];
            nbs.erase(std::remove(nbs.begin(), nbs.end(), u), nbs.end());
            for (int j : nbs) {
                const std::string dep_j = pc.get_propagator_key(j, v);
                std::string nk = "(" + agg + std::to_string(blk.n_segment_right);
                std::vector<std::string> others;
                for (int k : nbs)
                    if (k != j) others.push_back(pc.get_propagator_key(k, v) + std::to_string(pc.get_block(k, v).n_segment));
                std::sort(others.begin(), others.end());
                for (auto &o : others) nk += o;
                nk += ")" + pc.get_block(j, v).monomer_type;
                RightMap &rm = per_polymer[dep_j];
                rm.erase(vu_right[std::make_tuple(j, v)]);
                auto found = rm.find(nk);
                if (found == rm.end()) {
                    ComputationBlock &nb = rm[nk];
                    nb.monomer_type = pc.get_block(j, v).monomer_type;
                    nb.n_segment_right = pc.get_block(j, v).n_segment;
                    nb.n_segment_left = pc.get_block(j, v).n_segment;
                    nb.v_u.emplace_back(j, v);
                    nb.n_repeated = (agg[0] == '[') ? 1 : blk.n_repeated;
                    aggregated[dep_j].push_back(nk);
                } else {
                    found->second.v_u.emplace_back(j, v);
                    if (std::get<1>(found->second.v_u[0]) == v) found->second.n_repeated += blk.n_repeated;
                }
            }
        }
    }
}

void PropagatorAnalyzer::update_propagator(const std::string &key, int n, bool junction_end) {
    auto it = props_.find(key);
    if (it == props_.end()) {
        ComputationEdge &e = props_[key];
        e.deps = code::deps_from_key(key);
        e.monomer_type = code::monomer_type_from_key(key);
        e.max_n_segment = n;
        e.height = code::height_from_key(key);
        it = props_.find(key);
    } else if (it->second.max_n_segment < n) {
        it->second.max_n_segment = n;
    }
    if (junction_end) it->second.junction_ends.insert(n);
}

ComputationEdge &PropagatorAnalyzer::get_computation_propagator(const std::string &key) {
    auto it = props_.find(key);
    if (it == props_.end()) LFTS_THROW("There is no such key (" + key + ").");
    return it->second;
}

ComputationBlock &PropagatorAnalyzer::get_computation_block(const BlockKey &key) {
    auto it = blocks_.find(key);
    if (it == blocks_.end())
        LFTS_THROW("There is no such key (" + std::to_string(std::get<0>(key)) + ", " + std::get<1>(key) + ", " +
                   std::get<2>(key) + ").");
    return it->second;
}

static std::string clip500(const std::string &s, const char *tail) {
    return s.size() <= 500 ? s : s.substr(0, 495) + tail;
}

void PropagatorAnalyzer::display_blocks() const {
    std::cout << "--------------- Blocks ---------------" << std::endl;
    std::cout << "Polymer id, left key:\n\taggregated, (left, right) is_junction, (left, right) n_segment, right key, n_repeat, {v, u} list"
              << std::endl;
    std::tuple<int, std::string> last(-1, "");
    for (const auto &it : blocks_) {
        const std::string &kl = std::get<1>(it.first), &kr = std::get<2>(it.first);
        if (last != std::make_tuple(std::get<0>(it.first), kl)) {
            std::cout << std::endl << std::to_string(std::get<0>(it.first)) + ", " << clip500(kl, " ... <omitted>, ") << ":"
                      << std::endl;
            last = std::make_tuple(std::get<0>(it.first), kl);
        }
        std::cout << "\t " << (kr.find('[') == std::string::npos ? "X, " : "O, ");
        std::cout << "(" << (code::height_from_key(kl) > 0 ? "O, " : "X, ")
                  << (code::height_from_key(kr) > 0 ? "O), " : "X), ");
        std::cout << "(" + std::to_string(it.second.n_segment_left) + ", " + std::to_string(it.second.n_segment_right) + "), ";
        std::cout << clip500(kr, " ... <omitted>") << ", " + std::to_string(it.second.n_repeated);
        for (const auto &vu : it.second.v_u)
            std::cout << ", {" + std::to_string(std::get<0>(vu)) + "," + std::to_string(std::get<1>(vu)) + "}";
        std::cout << std::endl;
    }
}

void PropagatorAnalyzer::display_propagators() const {
    int total = 0, reduced = 0;
    std::cout << "--------------- Propagators ---------------" << std::endl;
    std::cout << "Key:\n\theight, aggregated, max_n_segment, # dependencies, junction_ends" << std::endl;
    for (int t : total_segments_) total += 2 * t;
    for (const auto &it : props_) {
        if (model_ == "continuous") {
            reduced += it.second.max_n_segment;
        } else {
            reduced += it.second.max_n_segment - 1 + (int)it.second.junction_ends.size();
            if (!it.second.deps.empty()) reduced++;
        }
        std::cout << clip500(it.first, " ... <omitted> ") << ":\n\t " << it.second.height << ", "
                  << (it.first.find('[') == std::string::npos ? "X, " : "O, ") << it.second.max_n_segment << ", "
                  << it.second.deps.size() << ", {";
        bool first = true;
        for (int j : it.second.junction_ends) { std::cout << (first ? "" : ", ") << j; first = false; }
        std::cout << "}, " << std::endl;
    }
    if (model_ == "continuous")
        std::cout << "Total number of modified diffusion equation steps (time complexity) to compute propagators: " << total << std::endl;
    else
        std::cout << "(Total number of integral equation steps (time complexity to compute propagators: " << total << std::endl;
    std::cout << "Total number of steps after optimizing computation : " << reduced << std::endl;
    double pct = 100 * (1.0 - ((double)reduced) / ((double)total));
    pct = std::round(pct * 100) / 100;
    std::cout << "Computational cost reduction (higher is better) : " << pct << " %" << std::endl;
}

// ================================================================ scheduler
// List scheduling of propagators by height onto n_streams lanes, then cut into
// time slots at every start/finish (Scheduler.cpp:11-190).
Scheduler::Scheduler(PropagatorMap &props, int n_streams) {
    if (n_streams < 1) LFTS_THROW("n_streams must be positive");
    std::vector<int> lane_free(n_streams, 0);
    std::vector<std::vector<std::string>> lane_jobs(n_streams);
    std::map<std::string, int> ready;

    // heights in increasing order, keys of one height in map order
    std::vector<std::vector<std::string>> levels;
    {
        std::vector<std::string> rest;
        for (const auto &p : props) rest.push_back(p.first);
        int h = 0;
        while (!rest.empty()) {
            std::vector<std::string> lvl;
            for (const auto &k : rest)
                if (code::height_from_key(k) == h) lvl.push_back(k);
            if (!lvl.empty()) {
                for (const auto &k : lvl) rest.erase(std::remove(rest.begin(), rest.end(), k), rest.end());
                levels.push_back(lvl);
            }
            h++;
        }
    }
    for (const auto &lvl : levels) {
        std::vector<std::tuple<std::string, int>> queue;
        for (const auto &key : lvl) {
            int t_ready = 0;
            for (const auto &d : props[key].deps) {
                const int n_dep = std::max(std::get<1>(d), 1);
                const int t = std::get<1>(lane_start_finish_[std::get<0>(d)]) + n_dep;
                if (t_ready == 0 || t_ready < t) t_ready = t;
            }
            ready[key] = t_ready;
            queue.emplace_back(key, t_ready);
        }
        std::sort(queue.begin(), queue.end(), [](auto const &a, auto const &b) { return std::get<1>(a) < std::get<1>(b); });
        for (const auto &q : queue) {
            int lane = 0;
            for (int s = 1; s < n_streams; s++)
                if (lane_free[s] < lane_free[lane]) lane = s;
            const std::string &key = std::get<0>(q);
            const int len = std::max(props[key].max_n_segment, 1);
            const int start = std::max(lane_free[lane], ready[key]);
            lane_start_finish_[key] = std::make_tuple(lane, start, start + len);
            lane_free[lane] = start + len;
            lane_jobs[lane].push_back(key);
        }
    }
    for (const auto &it : lane_start_finish_) by_start_.emplace_back(it.first, std::get<1>(it.second));
    std::sort(by_start_.begin(), by_start_.end(), [](auto const &a, auto const &b) { return std::get<1>(a) < std::get<1>(b); });
    std::set<int> stamps;
    for (const auto &b : by_start_) {
        const int start = std::get<1>(b);
        stamps.insert(start);
        stamps.insert(start + std::max(props[std::get<0>(b)].max_n_segment, 1));
    }
    stamps_.assign(stamps.begin(), stamps.end());
    std::vector<size_t> pos(n_streams, 0);
    for (size_t i = 0; i + 1 < stamps_.size(); i++) {
        std::vector<ScheduleJob> slot;
        for (int s = 0; s < n_streams; s++) {
            if (pos[s] < lane_jobs[s].size() && stamps_[i + 1] > std::get<2>(lane_start_finish_[lane_jobs[s][pos[s]]])) pos[s]++;
            if (pos[s] < lane_jobs[s].size()) {
                const std::string &key = lane_jobs[s][pos[s]];
                const auto &sf = lane_start_finish_[key];
                if (stamps_[i] >= std::get<1>(sf) && stamps_[i + 1] <= std::get<2>(sf)) {
                    int from = 0, to = 0;
                    if (props[key].max_n_segment != 0) {
                        from = stamps_[i] - std::get<1>(sf);
                        to = stamps_[i + 1] - std::get<1>(sf);
                    }
                    slot.emplace_back(key, from, to);
                }
            }
        }
        schedule_.push_back(slot);
    }
}

void Scheduler::display(PropagatorMap &props) const {
    for (const auto &b : by_start_) {
        const int start = std::get<1>(b);
        std::cout << std::get<0>(b) << ":\n\tmax_n_segment: " << props[std::get<0>(b)].max_n_segment << ", start_time: " << start
                  << ", finish_time: " << start + props[std::get<0>(b)].max_n_segment << std::endl;
    }
    for (size_t i = 0; i < schedule_.size(); i++) {
        std::cout << "time: " << stamps_[i] + 1 << "-" << stamps_[i + 1] << std::endl;
        for (const auto &j : schedule_[i])
            std::cout << "\t" << std::get<0>(j) << ": " << std::get<1>(j) << ", " << std::get<2>(j) << std::endl;
    }
}

// ================================================================ box
ComputationBox::ComputationBox(const std::vector<int> &nx, const std::vector<double> &lx, const std::vector<std::string> &bc) {
    if (nx.size() != lx.size())
        LFTS_THROW("The sizes of nx (" + std::to_string(nx.size()) + ") and lx (" + std::to_string(lx.size()) + ") must match.");
    if (nx.size() < 1 || nx.size() > 3) LFTS_THROW("We expect 1D, 2D or 3D, but we get " + std::to_string(nx.size()));
    for (int n : nx)
        if (n <= 0) LFTS_THROW("nx must be positive numbers");
    for (double l : lx)
        if (l <= 0.0) LFTS_THROW("lx must be positive numbers");
    if (!bc.empty() && bc.size() != 2 * nx.size())
        LFTS_THROW("We expect 0 or " + std::to_string(2 * nx.size()) + " boundary conditions, but we get " +
                   std::to_string(bc.size()) + ". For each dimension, two boundary conditions (top and bottom) are required.");
    std::vector<std::string> lower;
    for (auto b : bc) {
        std::transform(b.begin(), b.end(), b.begin(), [](unsigned char c) { return std::tolower(c); });
        lower.push_back(b);
    }
    for (size_t i = 0; i < lower.size(); i += 2)
        if ((lower[i] == "periodic") != (lower[i + 1] == "periodic"))
            LFTS_THROW(lower[i] + " and " + lower[i + 1] + " are an invalid boundary condition combination. " +
                       "If one side imposes a periodic boundary condition, the other side must also be a periodic boundary condition.");
    for (const auto &b : lower) {
        if (b == "periodic") bc_.push_back(0);
        else if (b == "reflecting") bc_.push_back(1);
        else if (b == "absorbing") bc_.push_back(2);
        else LFTS_THROW(b + " is an invalid boundary condition. Choose among ['periodic', 'reflecting', 'absorbing']");
    }
    if (bc_.empty()) bc_.assign(2 * nx.size(), 0);
    nx_ = nx;
    lx_ = lx;
    n_grid_ = 1;
    for (int n : nx) n_grid_ *= n;
    for (size_t d = 0; d < nx.size(); d++) dx_.push_back(lx[d] / nx[d]);
    dv_ = 1.0;
    for (double d : dx_) dv_ *= d;
    volume_ = 1.0;
    for (double l : lx) volume_ *= l;
}

bool ComputationBox::is_periodic() const {
    for (int b : bc_)
        if (b != 0) return false;
    return true;
}

int ComputationBox::get_nx(int i) const {
    if (i < 0 || i >= get_dim()) LFTS_THROW("'" + std::to_string(i) + "' is out of range.");
    return nx_[i];
}
double ComputationBox::get_lx(int i) const {
    if (i < 0 || i >= get_dim()) LFTS_THROW("'" + std::to_string(i) + "' is out of range.");
    return lx_[i];
}
double ComputationBox::get_dx(int i) const {
    if (i < 0 || i >= get_dim()) LFTS_THROW("'" + std::to_string(i) + "' is out of range.");
    return dx_[i];
}
double ComputationBox::get_dv(int i) const {
    if (i < 0 || i >= n_grid_) LFTS_THROW("'" + std::to_string(i) + "' is out of range.");
    return dv_;
}

// The box volume after a resize is the sum of the cell weights, as in
// ComputationBox.cpp:229-262.
void ComputationBox::set_lx(const std::vector<double> &lx) {
    if (lx.size() != nx_.size())
        LFTS_THROW("The sizes of new lx (" + std::to_string(lx.size()) + ") and dim (" + std::to_string(nx_.size()) + ") must match.");
    for (double l : lx)
        if (l <= 0.0) LFTS_THROW("new lx must be positive numbers");
    lx_ = lx;
    for (size_t d = 0; d < nx_.size(); d++) dx_[d] = lx_[d] / nx_[d];
    dv_ = 1.0;
    for (double d : dx_) dv_ *= d;
    double v = 0.0;
    for (int i = 0; i < n_grid_; i++) v += dv_;
    volume_ = v;
}

double ComputationBox::integral(const double *g) const {
    double s = 0.0;
    for (int i = 0; i < n_grid_; i++) s += dv_ * g[i];
    return s;
}
double ComputationBox::inner_product(const double *g, const double *h) const {
    double s = 0.0;
    for (int i = 0; i < n_grid_; i++) s += dv_ * g[i] * h[i];
    return s;
}

}  // namespace lfts
