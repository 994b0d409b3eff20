// Host-side chain model, propagator codes, dedup/aggregation analysis and
// stream schedule of the langevinfts API (integer/string work, C++).
//
// Mirrors the reference's public types (src/common/Polymer.h, Molecules.h,
// PropagatorCode.h, PropagatorAnalyzer.h, Scheduler.h, ComputationBox.h) with
// the same names, argument meaning and error behaviour.  The key strings, the
// key order (ComparePropagatorKey) and the schedule must come out identical to
// the reference's, so the order-defining operations (std::map iteration order,
// std::sort of the ready list, first-minimum lane choice) are the same ones.
#pragma once

#include <array>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace lfts {

// Same message shape as the reference's Exception (src/common/Exception.h:7-16).
struct Error : std::runtime_error {
    Error(const std::string &msg, const char *file, int line, const char *func)
        : std::runtime_error("File: \"" + std::string(file) + "\", line: " + std::to_string(line) + ", function <" +
                             std::string(func) + ">\n\t" + msg) {}
};
#define LFTS_THROW(msg) throw ::lfts::Error((msg), __FILE__, __LINE__, __func__)

struct BlockInput {
    std::string monomer_type;
    double contour_length;
    int v;
    int u;
};

struct Block {
    std::string monomer_type;
    int n_segment;
    double contour_length;
    int v;
    int u;
};

class Polymer {
   public:
    Polymer(double ds, const std::map<std::string, double> &bond_lengths, double volume_fraction,
            const std::vector<BlockInput> &block_inputs, const std::map<int, std::string> &chain_end_to_q_init = {});
    double get_alpha() const { return alpha_; }
    double get_volume_fraction() const { return volume_fraction_; }
    int get_n_blocks() const { return (int)blocks_.size(); }
    std::vector<Block> &get_blocks() { return blocks_; }
    Block &get_block(int v, int u);
    int get_n_segment_total() const;
    int get_n_segment(int idx) const { return blocks_.at(idx).n_segment; }
    int get_block_index_from_edge(int v, int u);
    std::map<int, std::vector<int>> &get_adjacent_nodes() { return adjacent_; }
    std::map<std::pair<int, int>, int> &get_block_indexes() { return edge_index_; }
    std::string get_propagator_key(int v, int u);
    const std::map<int, std::string> &get_chain_end_to_q_init() const { return q_init_; }

   private:
    double alpha_ = 0, volume_fraction_ = 0;
    std::vector<Block> blocks_;
    std::map<int, std::vector<int>> adjacent_;
    std::map<std::pair<int, int>, int> edge_index_;
    std::map<std::pair<int, int>, std::string> edge_key_;
    std::map<int, std::string> q_init_;
};

class Molecules {
   public:
    Molecules(std::string model_name, double ds, const std::map<std::string, double> &bond_lengths);
    const std::string &get_model_name() const { return model_; }
    double get_ds() const { return ds_; }
    const std::map<std::string, double> &get_bond_lengths() const { return bonds_; }
    void add_polymer(double volume_fraction, const std::vector<BlockInput> &blocks,
                     const std::map<int, std::string> &chain_end_to_q_init = {});
    void add_solvent(double volume_fraction, const std::string &monomer_type);
    int get_n_polymer_types() const { return (int)polymers_.size(); }
    Polymer &get_polymer(int p);
    int get_n_solvent_types() const { return (int)solvents_.size(); }
    std::tuple<double, std::string> get_solvent(int s) const { return solvents_.at(s); }

   private:
    std::string model_;
    double ds_;
    std::map<std::string, double> bonds_;
    std::vector<Polymer> polymers_;
    std::vector<std::tuple<double, std::string>> solvents_;
};

// Propagator key grammar (src/common/PropagatorCode.cpp).
namespace code {
std::string key_from_code(const std::string &code);
// (sub key, sub n_segment, sub n_repeated)
std::vector<std::tuple<std::string, int, int>> deps_from_key(const std::string &key);
std::string monomer_type_from_key(const std::string &key);
std::string q_input_from_key(const std::string &key);
int height_from_key(const std::string &key);
}  // namespace code

// Heights ascending, then keys in descending string order.
struct ComparePropagatorKey {
    bool operator()(const std::string &a, const std::string &b) const;
};

struct ComputationEdge {
    int max_n_segment = 0;
    std::string monomer_type;
    std::vector<std::tuple<std::string, int, int>> deps;
    int height = 0;
    std::set<int> junction_ends;
};

struct ComputationBlock {
    std::string monomer_type;
    int n_segment_left = 0;
    int n_segment_right = 0;
    int n_repeated = 0;
    std::vector<std::tuple<int, int>> v_u;
};

using PropagatorMap = std::map<std::string, ComputationEdge, ComparePropagatorKey>;
using BlockKey = std::tuple<int, std::string, std::string>;

class PropagatorAnalyzer {
   public:
    PropagatorAnalyzer(Molecules *molecules, bool aggregate);
    bool is_aggregated() const { return aggregate_; }
    const std::string &get_model_name() const { return model_; }
    int get_n_computation_propagator_codes() const { return (int)props_.size(); }
    PropagatorMap &get_computation_propagators() { return props_; }
    ComputationEdge &get_computation_propagator(const std::string &key);
    std::map<BlockKey, ComputationBlock> &get_computation_blocks() { return blocks_; }
    ComputationBlock &get_computation_block(const BlockKey &key);
    void display_propagators() const;
    void display_blocks() const;

    using RightMap = std::map<std::string, ComputationBlock>;
    static RightMap aggregate_common(RightMap set_I, int minimum_n_segment);

   private:
    void add_polymer(Polymer &pc, int polymer_id);
    void substitute_right_keys(Polymer &pc, std::map<std::tuple<int, int>, std::string> &vu_right,
                               std::map<std::string, RightMap> &per_polymer,
                               std::map<std::string, std::vector<std::string>> &aggregated, const std::string &left);
    void update_propagator(const std::string &key, int n_segment, bool is_junction_end);

    std::string model_;
    bool aggregate_;
    std::map<BlockKey, ComputationBlock> blocks_;
    PropagatorMap props_;
    std::vector<int> total_segments_;
};

// One job of a time slot: (key, n_segment_from, n_segment_to).
using ScheduleJob = std::tuple<std::string, int, int>;

class Scheduler {
   public:
    Scheduler(PropagatorMap &props, int n_streams);
    const std::vector<std::vector<ScheduleJob>> &get_schedule() const { return schedule_; }
    void display(PropagatorMap &props) const;

   private:
    std::map<std::string, std::tuple<int, int, int>, ComparePropagatorKey> lane_start_finish_;
    std::vector<std::tuple<std::string, int>> by_start_;
    std::vector<int> stamps_;
    std::vector<std::vector<ScheduleJob>> schedule_;
};

// Periodic box; integral weights are uniform (no mask).
class ComputationBox {
   public:
    ComputationBox(const std::vector<int> &nx, const std::vector<double> &lx, const std::vector<std::string> &bc);
    int get_dim() const { return (int)nx_.size(); }
    std::vector<int> get_nx() const { return nx_; }
    int get_nx(int i) const;
    std::vector<double> get_lx() const { return lx_; }
    double get_lx(int i) const;
    std::vector<double> get_dx() const { return dx_; }
    double get_dx(int i) const;
    double get_dv(int i) const;
    int get_n_grid() const { return n_grid_; }
    double get_volume() const { return volume_; }
    void set_lx(const std::vector<double> &lx);
    double integral(const double *g) const;
    double inner_product(const double *g, const double *h) const;
    // boundary condition of each side, lower side of axis d at 2d: 0 periodic,
    // 1 reflecting, 2 absorbing (src/common/ComputationBox.cpp:88-150)
    const std::vector<int> &get_boundary_conditions() const { return bc_; }
    bool is_periodic() const;

   private:
    std::vector<int> bc_;
    std::vector<int> nx_;
    std::vector<double> lx_, dx_;
    int n_grid_ = 0;
    double dv_ = 0, volume_ = 0;
};

}  // namespace lfts
