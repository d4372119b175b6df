// Lumped-parameter (0D) netlist boundary circuits: the reference's
// NetlistCircuit (flowsolver/src/NetlistCircuit.cxx) for circuits of
// resistors, capacitors, inductors and diodes coupled to one 3D outlet
// surface.  Host code: each circuit is a dense linear system of a few dozen
// unknowns solved once per time step.
#pragma once

#include <vector>

#include "../../include/crimson_b200.h"

namespace crimson {

struct NetlistNode {
    bool fixed = false;    // prescribed pressure (input type 'f')
    double fixed_p = 0.0;  // its value
    double p = 0.0;        // current pressure
    double hist = 0.0;     // pressure of the previous step (capacitor ends)
    bool has_hist = false;
};

struct NetlistComp {
    int kind = 0;  // CRIMSON_NETLIST_RESISTOR ...
    int start = 0, end = 0;  // 1-based node indices
    double value = 0.0;      // R, C, L, or the open diode's resistance
    int flow_kind = -1;      // -1 none, CRIMSON_NETLIST_FLOW_FIXED, CRIMSON_NETLIST_FLOW_3D
    double flow_fixed = 0.0;
    double flow = 0.0;       // current flow (start -> end)
    double hist_flow = 0.0;  // flow of the previous step (inductors)
    bool open = true;        // diodes: permits flow
    // volume-tracking components (value = elastance for a pressure chamber)
    double volume = 0.0, hist_volume = 0.0, unstressed = 0.0;
};

}  // namespace crimson

struct crimson_netlist {
    int np = 0, nc = 0;
    std::vector<crimson::NetlistNode> node;  // node i at [i - 1]
    std::vector<crimson::NetlistComp> comp;  // component j at [j - 1]
    int iface_node = 1;
    int iface_comp = -1;  // 0-based
    double sign = 1.0;    // +1: the interface component's start node is the interface node
    // unknown layout of the linear system (NetlistCircuit.cxx:1057-1302):
    // [pressures (np) | history pressures (nhp) | flows (nc) | history flows (nhf)
    //  | tracked volumes (nv) | history volumes (nv)]
    std::vector<int> hist_nodes;   // ascending node indices with a history pressure
    std::vector<int> hist_comps;   // ascending 0-based inductor indices
    std::vector<int> vol_comps;    // ascending 0-based volume-tracking components
    std::vector<int> vol_ord;      // component -> position in vol_comps (-1: none)
    int nchamber = 0;              // pressure chambers (two rows each)
    std::vector<int> kirch_nodes;  // ascending node indices with more than one incident component
    std::vector<int> pp_nodes;     // ascending prescribed-pressure nodes
    std::vector<int> pf_comps;     // ascending 0-based prescribed-flow components
    std::vector<int> hist_node_ord, hist_comp_ord;
    std::vector<std::vector<int>> nb_start, nb_end;  // neighbouring components at each end
    int n = 0;                                       // system size
    std::vector<double> A, Ainv, b, x;
    std::vector<int> connect_nodes;  // ascending nodes shared with another circuit of a closed loop
    double last_q = 0.0;    // interface flow of the last update (the flow the reference reads from the 3D side)
    double last_p3d = 0.0;  // 3D surface pressure of the last Dirichlet-design update
    bool flow_permitted = true;  // false: closed diodes block the interface (Dirichlet design)
};

// A closed loop (ClosedLoopDownstreamSubsection): its members and the dense
// system they share.
struct crimson_netlist_loop {
    std::vector<crimson_netlist*> member;  // upstream circuits in input order, then the loop-closing circuit
    int nup = 0;
    std::vector<int> conn_down, conn_up, conn_node;  // connections in file order
    std::vector<int> down_nodes;                     // ascending distinct downstream shared nodes
    std::vector<int> row0, col0;                     // first row / column of each member's block
    int n = 0;
    std::vector<double> A, Ainv, b, x;
};

namespace crimson {
// initialiseAtStartOfTimestep: whether closed diodes block every path from
// the 3D interface (then the circuit takes the Dirichlet design and the
// surface becomes a Dirichlet boundary of the flow problem).
int netlist_begin_step(crimson_netlist* nl);
}  // namespace crimson
