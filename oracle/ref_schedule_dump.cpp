/*
 * Oracle infrastructure (test-only).
 *
 * Drives the reference's own host classes (Molecules, PropagatorAnalyzer,
 * Scheduler: src/common/Molecules.cpp:42-50, PropagatorAnalyzer.cpp:29-168,
 * Scheduler.cpp:11-190) on a molecule description read from stdin and prints
 * the resulting propagator table, computation blocks and stream schedule as
 * JSON, so the project's host code can be checked against them byte for byte.
 *
 * stdin format (one item per line):
 *   model <continuous|discrete>
 *   ds <value>
 *   bond <monomer> <segment length>
 *   aggregate <0|1>
 *   streams <n>
 *   polymer <volume fraction>
 *   block <monomer> <contour length> <v> <u>     (belongs to the last polymer)
 *   qinit <node> <name>                           (belongs to the last polymer)
 */
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "Molecules.h"
#include "PropagatorAnalyzer.h"
#include "Scheduler.h"

static std::string js(const std::string &s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o + "\"";
}

int main() {
    std::string model = "continuous";
    double ds = 0.01;
    std::map<std::string, double> bonds;
    bool aggregate = true;
    int streams = 4;
    struct P {
        double vf;
        std::vector<BlockInput> blocks;
        std::map<int, std::string> qinit;
    };
    std::vector<P> polymers;
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream is(line);
        std::string tag;
        if (!(is >> tag)) continue;
        if (tag == "model") is >> model;
        else if (tag == "ds") is >> ds;
        else if (tag == "bond") { std::string m; double b; is >> m >> b; bonds[m] = b; }
        else if (tag == "aggregate") { int a; is >> a; aggregate = a != 0; }
        else if (tag == "streams") is >> streams;
        else if (tag == "polymer") { P p; is >> p.vf; polymers.push_back(p); }
        else if (tag == "block") {
            BlockInput b; is >> b.monomer_type >> b.contour_length >> b.v >> b.u;
            polymers.back().blocks.push_back(b);
        } else if (tag == "qinit") { int n; std::string g; is >> n >> g; polymers.back().qinit[n] = g; }
    }
    try {
        Molecules mol(model, ds, bonds);
        for (auto &p : polymers) mol.add_polymer(p.vf, p.blocks, p.qinit);
        PropagatorAnalyzer pa(&mol, aggregate);
        Scheduler sc(pa.get_computation_propagators(), streams);

        std::cout << "{\"propagators\": [";
        bool first = true;
        for (auto &item : pa.get_computation_propagators()) {
            if (!first) std::cout << ", ";
            first = false;
            const auto &e = item.second;
            std::cout << "{\"key\": " << js(item.first) << ", \"max_n_segment\": " << e.max_n_segment
                      << ", \"monomer_type\": " << js(e.monomer_type) << ", \"height\": " << e.height
                      << ", \"deps\": [";
            for (size_t i = 0; i < e.deps.size(); i++) {
                if (i) std::cout << ", ";
                std::cout << "[" << js(std::get<0>(e.deps[i])) << ", " << std::get<1>(e.deps[i]) << ", "
                          << std::get<2>(e.deps[i]) << "]";
            }
            std::cout << "], \"junction_ends\": [";
            bool f2 = true;
            for (int j : e.junction_ends) { if (!f2) std::cout << ", "; f2 = false; std::cout << j; }
            std::cout << "]}";
        }
        std::cout << "], \"blocks\": [";
        first = true;
        for (auto &item : pa.get_computation_blocks()) {
            if (!first) std::cout << ", ";
            first = false;
            const auto &b = item.second;
            std::cout << "{\"polymer\": " << std::get<0>(item.first) << ", \"key_left\": " << js(std::get<1>(item.first))
                      << ", \"key_right\": " << js(std::get<2>(item.first)) << ", \"monomer_type\": " << js(b.monomer_type)
                      << ", \"n_segment_left\": " << b.n_segment_left << ", \"n_segment_right\": " << b.n_segment_right
                      << ", \"n_repeated\": " << b.n_repeated << ", \"v_u\": [";
            for (size_t i = 0; i < b.v_u.size(); i++) {
                if (i) std::cout << ", ";
                std::cout << "[" << std::get<0>(b.v_u[i]) << ", " << std::get<1>(b.v_u[i]) << "]";
            }
            std::cout << "]}";
        }
        std::cout << "], \"schedule\": [";
        first = true;
        for (auto &slot : sc.get_schedule()) {
            if (!first) std::cout << ", ";
            first = false;
            std::cout << "[";
            for (size_t i = 0; i < slot.size(); i++) {
                if (i) std::cout << ", ";
                std::cout << "[" << js(std::get<0>(slot[i])) << ", " << std::get<1>(slot[i]) << ", "
                          << std::get<2>(slot[i]) << "]";
            }
            std::cout << "]";
        }
        std::cout << "]}" << std::endl;
    } catch (std::exception &exc) {
        std::cout << "{\"error\": " << js(exc.what()) << "}" << std::endl;
        return 1;
    }
    return 0;
}
