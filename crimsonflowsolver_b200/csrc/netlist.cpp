// Netlist boundary circuits (host code): NetlistCircuit
// (flowsolver/src/NetlistCircuit.cxx) with CircuitData / CircuitComponent
// for resistors, capacitors, inductors and diodes, fixed nodal pressures,
// fixed component flows and one component carrying the 3D interface flow
// (the Neumann coupling the flow solver's ElmpvsQ netlist branch uses,
// elmgmr.f90:1430-1452).
//
// Each time step the circuit is one dense linear system in the reference's
// unknown order [nodal pressures | history pressures | component flows |
// history flows]; its inverse gives the implicit coefficients dp/dQ and H of
// the interface pressure p = dp/dQ * Q + H.  When closed diodes block every
// path from the interface the circuit switches to the reference's Dirichlet
// design (CircuitData.cxx:482-540): the interface node takes the 3D
// surface pressure as a prescribed pressure and the interface component's
// flow is no longer prescribed.
#include "netlist.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <new>
#include <string>

namespace crimson {
void set_last_error(const std::string& s);
}

using crimson::NetlistComp;
using crimson::NetlistNode;

namespace {

int fail(const char* msg, int code = CRIMSON_ERR_ARG) {
    crimson::set_last_error(msg);
    return code;
}

// Unknown offsets of the blocks of the system.
inline int col_hist_p(const crimson_netlist* nl) { return nl->np; }
inline int col_flow(const crimson_netlist* nl) { return nl->np + (int)nl->hist_nodes.size(); }
inline int col_hist_q(const crimson_netlist* nl) { return col_flow(nl) + nl->nc; }
inline int col_vol(const crimson_netlist* nl) { return col_hist_q(nl) + (int)nl->hist_comps.size(); }
inline int col_hist_v(const crimson_netlist* nl) { return col_vol(nl) + (int)nl->vol_comps.size(); }

// Pressure of a node as the reference reads it: a fixed-pressure node
// returns its prescribed value (CircuitPressureNode.cxx:55-66).
inline double node_pressure(const NetlistNode& d) { return d.fixed ? d.fixed_p : d.p; }

// Prescribed-pressure nodes and prescribed-flow components of the current
// design, ascending: in the Dirichlet design the interface node joins the
// pressures and the interface component leaves the flows.
std::vector<int> design_pp(const crimson_netlist* nl) {
    std::vector<int> pp(nl->pp_nodes);
    if (!nl->flow_permitted) {
        pp.push_back(nl->iface_node);
        std::sort(pp.begin(), pp.end());
    }
    return pp;
}

std::vector<int> design_pf(const crimson_netlist* nl) {
    std::vector<int> pf;
    for (int j : nl->pf_comps)
        if (nl->flow_permitted || j != nl->iface_comp) pf.push_back(j);
    return pf;
}

// generateLinearSystemWithoutFactorisation (NetlistCircuit.cxx:1057-1302):
// one row per component (two for a pressure chamber), one Kirchhoff row per
// node with more than one incident component, then one identity row per
// prescribed value (fixed pressures, history pressures, prescribed flows,
// history flows, history volumes).
// The rows go to M (leading dimension ld, zeroed by the caller) from row r0
// on, the circuit's unknowns at columns c0..c0 + n - 1; a circuit that shares
// nodes with another (a closed loop) writes n - (its shared nodes) rows.
void build_rows(const crimson_netlist* nl, double alfi_delt, double* M, size_t ld, int r0, int c0) {
    auto a = [&](int r, int c) -> double& { return M[(size_t)(r0 + r) * ld + (size_t)(c0 + c)]; };
    const int cf = col_flow(nl), chp = col_hist_p(nl), chq = col_hist_q(nl);
    const int cv = col_vol(nl), chv = col_hist_v(nl);
    int row = 0;
    for (int j = 0; j < nl->nc; ++j, ++row) {
        const NetlistComp& c = nl->comp[j];
        switch (c.kind) {
            case CRIMSON_NETLIST_VOLUME_TRACKING:
            case CRIMSON_NETLIST_PRESSURE_CHAMBER: {
                // dV/dt = q: V - V_hist - alfi_delt q = 0
                const int v = nl->vol_ord[j];
                a(row, cf + j) = -alfi_delt;
                a(row, cv + v) = 1.0;
                a(row, chv + v) = -1.0;
                if (c.kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) {
                    // p_start / E - V = -V_unstressed
                    ++row;
                    a(row, c.start - 1) = 1.0 / c.value;
                    a(row, cv + v) = -1.0;
                }
                break;
            }
            case CRIMSON_NETLIST_RESISTOR:
                a(row, c.start - 1) = 1.0;
                a(row, c.end - 1) = -1.0;
                a(row, cf + j) = -c.value;
                break;
            case CRIMSON_NETLIST_DIODE:
                if (c.open) {  // a resistor of the diode's value
                    a(row, c.start - 1) = 1.0;
                    a(row, c.end - 1) = -1.0;
                    a(row, cf + j) = -c.value;
                } else {  // zero flow
                    a(row, cf + j) = 1.0;
                }
                break;
            case CRIMSON_NETLIST_CAPACITOR:
                a(row, c.start - 1) = 1.0;
                a(row, c.end - 1) = -1.0;
                a(row, cf + j) = -alfi_delt / c.value;
                a(row, chp + nl->hist_node_ord[c.start - 1]) = -1.0;
                a(row, chp + nl->hist_node_ord[c.end - 1]) = 1.0;
                break;
            default:  // inductor
                a(row, c.start - 1) = 1.0;
                a(row, c.end - 1) = -1.0;
                a(row, cf + j) = -c.value / alfi_delt;
                a(row, chq + nl->hist_comp_ord[j]) = c.value / alfi_delt;
                break;
        }
    }
    // Kirchhoff: sum of flows ending at the node minus flows starting there
    for (size_t m = 0; m < nl->kirch_nodes.size(); ++m, ++row) {
        const int nd = nl->kirch_nodes[m];
        for (int j = 0; j < nl->nc; ++j) {
            if (nl->comp[j].end == nd) a(row, cf + j) = 1.0;
            if (nl->comp[j].start == nd) a(row, cf + j) = -1.0;
        }
    }
    for (int nd : design_pp(nl)) a(row++, nd - 1) = 1.0;
    for (size_t l = 0; l < nl->hist_nodes.size(); ++l) a(row++, chp + (int)l) = 1.0;
    for (int j : design_pf(nl)) a(row++, cf + j) = 1.0;
    for (size_t l = 0; l < nl->hist_comps.size(); ++l) a(row++, chq + (int)l) = 1.0;
    for (size_t l = 0; l < nl->vol_comps.size(); ++l) a(row++, chv + (int)l) = 1.0;
}

void build_system(crimson_netlist* nl, double alfi_delt) {
    std::fill(nl->A.begin(), nl->A.end(), 0.0);
    build_rows(nl, alfi_delt, nl->A.data(), (size_t)nl->n, 0, 0);
}

// First row of the prescribed values (after the component and Kirchhoff rows).
inline int first_prescribed_row(const crimson_netlist* nl) {
    return nl->nc + nl->nchamber + (int)nl->kirch_nodes.size();
}

// Row of the system that carries the 3D interface flow.
int iface_row(const crimson_netlist* nl) {
    int r = first_prescribed_row(nl) + (int)nl->pp_nodes.size() + (int)nl->hist_nodes.size();
    for (int j : nl->pf_comps) {
        if (j == nl->iface_comp) return r;
        ++r;
    }
    return -1;
}

// assembleRHS (NetlistCircuit.cxx:1370-1580) in the same row order.
void rhs_rows(const crimson_netlist* nl, double* b, int r0) {
    b += r0;
    int row = first_prescribed_row(nl);
    // a fixed pressure, or the 3D surface pressure at the interface node
    // (Pressure_3DInterface, NetlistCircuit.cxx:1386-1410)
    for (int nd : design_pp(nl)) b[row++] = nl->node[nd - 1].fixed ? nl->node[nd - 1].fixed_p : nl->last_p3d;
    for (int nd : nl->hist_nodes) b[row++] = nl->node[nd - 1].hist;
    for (int j : design_pf(nl)) {
        const NetlistComp& c = nl->comp[j];
        b[row++] = c.flow_kind == CRIMSON_NETLIST_FLOW_3D ? nl->last_q * nl->sign : c.flow_fixed;
    }
    for (int j : nl->hist_comps) b[row++] = nl->comp[j].hist_flow;
    for (int j : nl->vol_comps) b[row++] = nl->comp[j].hist_volume;
    // a chamber's second row: compliance * pressure = volume - unstressed volume
    int r = 0;
    for (int j = 0; j < nl->nc; ++j, ++r)
        if (nl->comp[j].kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) b[++r] = -nl->comp[j].unstressed;
}

void assemble_rhs(crimson_netlist* nl) {
    std::fill(nl->b.begin(), nl->b.end(), 0.0);
    rhs_rows(nl, nl->b.data(), 0);
}

// solveLinearSystem (NetlistCircuit.cxx:1723-1733): the inverse of the
// system matrix (Gauss-Jordan with partial pivoting), then x = A^-1 b.
int gj_solve(int n, const std::vector<double>& A, std::vector<double>& inv, const std::vector<double>& b,
             std::vector<double>& x) {
    std::vector<double> m(A);
    std::fill(inv.begin(), inv.end(), 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    double amax = 0.0;
    for (double v : m) amax = std::max(amax, std::fabs(v));
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(m[(size_t)i * n + k]) > std::fabs(m[(size_t)p * n + k])) p = i;
        const double piv = m[(size_t)p * n + k];
        if (!(std::fabs(piv) > 1e-14 * amax)) return fail("netlist: singular circuit system", CRIMSON_ERR_SINGULAR);
        if (p != k)
            for (int c = 0; c < n; ++c) {
                std::swap(m[(size_t)p * n + c], m[(size_t)k * n + c]);
                std::swap(inv[(size_t)p * n + c], inv[(size_t)k * n + c]);
            }
        const double r = 1.0 / piv;
        for (int c = 0; c < n; ++c) {
            m[(size_t)k * n + c] *= r;
            inv[(size_t)k * n + c] *= r;
        }
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            const double f = m[(size_t)i * n + k];
            if (f == 0.0) continue;
            for (int c = 0; c < n; ++c) {
                m[(size_t)i * n + c] -= f * m[(size_t)k * n + c];
                inv[(size_t)i * n + c] -= f * inv[(size_t)k * n + c];
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int c = 0; c < n; ++c) s += inv[(size_t)i * n + c] * b[c];
        x[i] = s;
    }
    for (double v : x)
        if (!std::isfinite(v)) return fail("netlist: non-finite circuit solution", CRIMSON_ERR_NONFINITE);
    return CRIMSON_OK;
}

int solve(crimson_netlist* nl) { return gj_solve(nl->n, nl->A, nl->Ainv, nl->b, nl->x); }

// giveNodesTheirPressuresFromSolutionVector / giveComponentsTheirFlows... /
// giveComponentsTheirVolumes... (NetlistCircuit.cxx:1596-1660): the
// circuit's segment xs of a solution; a chamber passes E (V - V_unstressed)
// to its start node (CircuitComponent.cxx:188-209).
void take_solution(crimson_netlist* nl, const double* xs) {
    for (int i = 0; i < nl->np; ++i) nl->node[i].p = xs[i];
    const int cf = col_flow(nl);
    for (int j = 0; j < nl->nc; ++j) nl->comp[j].flow = xs[(size_t)cf + j];
    const int cv = col_vol(nl);
    for (int j : nl->vol_comps) {
        NetlistComp& c = nl->comp[j];
        c.volume = xs[(size_t)cv + nl->vol_ord[j]];
        if (c.kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) nl->node[(size_t)c.start - 1].p = (c.volume - c.unstressed) * c.value;
    }
}

// detectWhetherClosedDiodesStopAllFlowAt3DInterface (CircuitData.cxx:
// 388-470): walk the flow-permitting components from the interface
// component; flow can cross the interface if one of them has an end with no
// other component attached (a sink) that is not the interface node.
bool detect_flow_permitted(const crimson_netlist* nl) {
    if (nl->iface_comp < 0) return true;  // a loop-closing circuit has no 3D interface
    std::vector<int> stack{nl->iface_comp};
    std::vector<char> seen((size_t)nl->nc, 0);
    while (!stack.empty()) {
        const int j = stack.back();
        stack.pop_back();
        if (seen[j]) continue;
        seen[j] = 1;
        const NetlistComp& c = nl->comp[j];
        if (!c.open) continue;
        const bool start_sink = nl->nb_start[j].empty() && c.start != nl->iface_node;
        const bool end_sink = nl->nb_end[j].empty() && c.end != nl->iface_node;
        if (start_sink || end_sink) return true;
        for (int k : nl->nb_end[j]) stack.push_back(k);
        for (int k : nl->nb_start[j]) stack.push_back(k);
    }
    return false;
}

}  // namespace

namespace crimson {

int netlist_begin_step(crimson_netlist* nl) {
    nl->flow_permitted = detect_flow_permitted(nl);
    return CRIMSON_OK;
}

}  // namespace crimson

extern "C" {

int crimson_netlist_create(crimson_netlist** out, int ncomp, const int* kind, const int* start_node,
                           const int* end_node, const double* value, const double* initial_volume,
                           const double* unstressed_volume, int nnodes, const double* initial_pressure, int npres,
                           const int* pres_node, const double* pres_value, int nflow, const int* flow_comp,
                           const int* flow_kind, const double* flow_value, int interface_node) {
    if (interface_node != 1) return fail("netlist: the 3D interface node must be node 1");
    return crimson_netlist_create_member(out, ncomp, kind, start_node, end_node, value, initial_volume,
                                         unstressed_volume, nnodes, initial_pressure, npres, pres_node, pres_value,
                                         nflow, flow_comp, flow_kind, flow_value, interface_node, 0, nullptr);
}

int crimson_netlist_create_member(crimson_netlist** out, int ncomp, const int* kind, const int* start_node,
                                  const int* end_node, const double* value, const double* initial_volume,
                                  const double* unstressed_volume, int nnodes, const double* initial_pressure,
                                  int npres, const int* pres_node, const double* pres_value, int nflow,
                                  const int* flow_comp, const int* flow_kind, const double* flow_value,
                                  int interface_node, int nshared, const int* shared_nodes) {
    if (!out) return CRIMSON_ERR_ARG;
    *out = nullptr;
    if (ncomp < 1 || nnodes < 1 || !kind || !start_node || !end_node || !value || !initial_pressure)
        return fail("netlist: need at least one component and one node");
    if (npres < 0 || nflow < 0 || (npres > 0 && (!pres_node || !pres_value)) ||
        (nflow > 0 && (!flow_comp || !flow_kind || !flow_value)))
        return fail("netlist: bad prescribed pressure / flow lists");
    if (nshared < 0 || (nshared > 0 && !shared_nodes)) return fail("netlist: bad shared-node list");
    crimson_netlist* nl = new (std::nothrow) crimson_netlist;
    if (!nl) return CRIMSON_ERR_OOM;
    auto bad = [&](const char* msg) {
        delete nl;
        return fail(msg);
    };
    nl->np = nnodes;
    nl->nc = ncomp;
    nl->node.resize((size_t)nnodes);
    nl->comp.resize((size_t)ncomp);
    std::vector<int> uses((size_t)nnodes, 0);
    for (int j = 0; j < ncomp; ++j) {
        NetlistComp& c = nl->comp[j];
        c.kind = kind[j];
        c.start = start_node[j];
        c.end = end_node[j];
        c.value = value[j];
        if (c.kind < CRIMSON_NETLIST_RESISTOR || c.kind > CRIMSON_NETLIST_PRESSURE_CHAMBER)
            return bad("netlist: unknown component kind");
        if (c.start < 1 || c.start > nnodes || c.end < 1 || c.end > nnodes || c.start == c.end)
            return bad("netlist: component nodes out of range or equal");
        if (!std::isfinite(c.value) ||
            ((c.kind == CRIMSON_NETLIST_CAPACITOR || c.kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) && c.value == 0.0))
            return bad("netlist: bad component value");
        if (c.kind >= CRIMSON_NETLIST_VOLUME_TRACKING) {
            if (!initial_volume || !std::isfinite(initial_volume[j]))
                return bad("netlist: a volume-tracking component needs its initial volume");
            c.volume = initial_volume[j];
            c.unstressed = unstressed_volume ? unstressed_volume[j] : 0.0;
            if (!std::isfinite(c.unstressed)) return bad("netlist: non-finite unstressed volume");
        }
        uses[c.start - 1] += 1;
        uses[c.end - 1] += 1;
    }
    for (int i = 0; i < nnodes; ++i) {
        if (uses[i] == 0) return bad("netlist: every node 1..nnodes must belong to a component");
        if (!std::isfinite(initial_pressure[i])) return bad("netlist: non-finite initial pressure");
        nl->node[i].p = initial_pressure[i];
    }
    for (int k = 0; k < npres; ++k) {
        const int nd = pres_node[k];
        if (nd < 1 || nd > nnodes || nl->node[nd - 1].fixed) return bad("netlist: bad prescribed-pressure node");
        nl->node[nd - 1].fixed = true;
        nl->node[nd - 1].fixed_p = pres_value[k];
        nl->pp_nodes.push_back(nd);
    }
    int n3d = 0;
    for (int k = 0; k < nflow; ++k) {
        const int j = flow_comp[k];
        if (j < 1 || j > ncomp || nl->comp[j - 1].flow_kind >= 0) return bad("netlist: bad prescribed-flow component");
        if (flow_kind[k] != CRIMSON_NETLIST_FLOW_FIXED && flow_kind[k] != CRIMSON_NETLIST_FLOW_3D)
            return bad("netlist: unknown flow prescription");
        nl->comp[j - 1].flow_kind = flow_kind[k];
        nl->comp[j - 1].flow_fixed = flow_value[k];
        nl->pf_comps.push_back(j - 1);
        if (flow_kind[k] == CRIMSON_NETLIST_FLOW_3D) {
            ++n3d;
            nl->iface_comp = j - 1;
        }
    }
    std::sort(nl->pp_nodes.begin(), nl->pp_nodes.end());
    std::sort(nl->pf_comps.begin(), nl->pf_comps.end());
    // initialiseNodeAndComponentAtInterface (CircuitData.cxx:130-262); the
    // coupling coefficients are read from unknown 0, the pressure of node 1
    // (NetlistCircuit.cxx:1770-1790), so the interface node is node 1.  A
    // loop-closing circuit (interface_node 0) has none.
    if (interface_node == 0) {
        if (n3d != 0) return bad("netlist: a circuit without a 3D interface cannot carry the 3D flow");
        nl->iface_node = 0;
        nl->iface_comp = -1;
    } else {
        if (n3d != 1) return bad("netlist: exactly one component must carry the 3D interface flow");
        if (interface_node != 1) return bad("netlist: the 3D interface node must be node 1");
        nl->iface_node = interface_node;
        const NetlistComp& ic = nl->comp[nl->iface_comp];
        if (ic.start != interface_node && ic.end != interface_node)
            return bad("netlist: the 3D-flow component does not touch the interface node");
        if (uses[interface_node - 1] != 1)
            return bad("netlist: the interface node must belong to exactly one component");
        if (nl->node[interface_node - 1].fixed)
            return bad("netlist: the interface node cannot have a prescribed pressure");
        nl->sign = ic.start == interface_node ? 1.0 : -1.0;
    }
    // nodes shared with another circuit of a closed loop: their Kirchhoff
    // equation is the loop's (createListOfNodesWithMultipleIncidentCurrents,
    // NetlistCircuit.cxx:880-920)
    for (int k = 0; k < nshared; ++k) {
        const int nd = shared_nodes[k];
        if (nd < 1 || nd > nnodes || nd == interface_node) return bad("netlist: bad shared node");
        nl->connect_nodes.push_back(nd);
    }
    std::sort(nl->connect_nodes.begin(), nl->connect_nodes.end());
    if (std::adjacent_find(nl->connect_nodes.begin(), nl->connect_nodes.end()) != nl->connect_nodes.end())
        return bad("netlist: a shared node is listed twice");
    // history pressures at capacitor ends, history flows of inductors
    // (NetlistCircuit.cxx:930-979), Kirchhoff nodes (876-917)
    for (const NetlistComp& c : nl->comp)
        if (c.kind == CRIMSON_NETLIST_CAPACITOR) {
            nl->node[c.start - 1].has_hist = true;
            nl->node[c.end - 1].has_hist = true;
        }
    nl->hist_node_ord.assign((size_t)nnodes, -1);
    for (int i = 0; i < nnodes; ++i)
        if (nl->node[i].has_hist) {
            nl->hist_node_ord[i] = (int)nl->hist_nodes.size();
            nl->hist_nodes.push_back(i + 1);
        }
    nl->hist_comp_ord.assign((size_t)ncomp, -1);
    for (int j = 0; j < ncomp; ++j)
        if (nl->comp[j].kind == CRIMSON_NETLIST_INDUCTOR) {
            nl->hist_comp_ord[j] = (int)nl->hist_comps.size();
            nl->hist_comps.push_back(j);
        }
    // volume-tracking components: a tracked and a history volume each
    // (NetlistCircuit.cxx:981-1041)
    nl->vol_ord.assign((size_t)ncomp, -1);
    for (int j = 0; j < ncomp; ++j)
        if (nl->comp[j].kind >= CRIMSON_NETLIST_VOLUME_TRACKING) {
            nl->vol_ord[j] = (int)nl->vol_comps.size();
            nl->vol_comps.push_back(j);
            if (nl->comp[j].kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) ++nl->nchamber;
        }
    for (int i = 0; i < nnodes; ++i)
        if (uses[i] > 1 && !std::binary_search(nl->connect_nodes.begin(), nl->connect_nodes.end(), i + 1))
            nl->kirch_nodes.push_back(i + 1);
    const int nv = (int)nl->vol_comps.size();
    if (nl->nchamber + (int)(nl->kirch_nodes.size() + nl->pp_nodes.size() + nl->pf_comps.size()) !=
        nnodes + nv - (int)nl->connect_nodes.size())
        return bad(nl->connect_nodes.empty() ? "netlist: malformed circuit (the system is not square)"
                                             : "netlist: malformed circuit (its rows and its shared nodes do not "
                                               "make up its unknowns)");
    nl->n = nnodes + (int)nl->hist_nodes.size() + ncomp + (int)nl->hist_comps.size() + 2 * nv;
    nl->A.assign((size_t)nl->n * nl->n, 0.0);
    nl->Ainv.assign((size_t)nl->n * nl->n, 0.0);
    nl->b.assign((size_t)nl->n, 0.0);
    nl->x.assign((size_t)nl->n, 0.0);
    // neighbours at each end (CircuitData.cxx:84-128)
    nl->nb_start.resize((size_t)ncomp);
    nl->nb_end.resize((size_t)ncomp);
    for (int j = 0; j < ncomp; ++j)
        for (int k = 0; k < ncomp; ++k) {
            if (k == j) continue;
            const NetlistComp &c = nl->comp[j], &o = nl->comp[k];
            if (o.start == c.start || o.end == c.start) nl->nb_start[j].push_back(k);
            if (o.start == c.end || o.end == c.end) nl->nb_end[j].push_back(k);
        }
    // NetlistBoundaryCondition::initialiseModel (NetlistBoundaryCondition.cxx:
    // 10-35): diodes start closed; the histories start from the initial state
    // (setInternalHistoryPressureFlowsAndVolumes, NetlistCircuit.cxx:654-688)
    for (NetlistComp& c : nl->comp)
        if (c.kind == CRIMSON_NETLIST_DIODE) c.open = false;
    for (NetlistNode& d : nl->node)
        if (d.has_hist) d.hist = node_pressure(d);
    for (int j : nl->hist_comps) nl->comp[j].hist_flow = nl->comp[j].flow;
    for (int j : nl->vol_comps) nl->comp[j].hist_volume = nl->comp[j].volume;
    nl->flow_permitted = detect_flow_permitted(nl);
    *out = nl;
    return CRIMSON_OK;
}

void crimson_netlist_free(crimson_netlist* nl) { delete nl; }

int crimson_netlist_flow_permitted(crimson_netlist* nl, int* permitted) {
    if (!nl || !permitted) return CRIMSON_ERR_ARG;
    nl->flow_permitted = detect_flow_permitted(nl);
    *permitted = nl->flow_permitted ? 1 : 0;
    return CRIMSON_OK;
}

// computeImplicitCoefficients (NetlistCircuit.cxx:1764-1800)
int crimson_netlist_implicit_coefficients(crimson_netlist* nl, double alfi_delt, double* dp_dq, double* hop) {
    if (!nl || !dp_dq || !hop || !(alfi_delt > 0.0)) return CRIMSON_ERR_ARG;
    if (!nl->flow_permitted)
        return fail("netlist: no flow across the 3D interface (Dirichlet design: no implicit coefficients)",
                    CRIMSON_ERR_STATE);
    if (nl->iface_comp < 0 || !nl->connect_nodes.empty())
        return fail("netlist: no 3D interface, or a member of a closed loop (use the loop)", CRIMSON_ERR_STATE);
    build_system(nl, alfi_delt);
    assemble_rhs(nl);
    const int st = solve(nl);
    if (st != CRIMSON_OK) return st;
    const int col = iface_row(nl);
    const double g = nl->Ainv[(size_t)col];  // row 0
    *dp_dq = nl->sign * g;
    *hop = nl->x[0] - g * nl->b[(size_t)col];
    return CRIMSON_OK;
}

// updateLPN (NetlistCircuit.cxx:1582-1594): solve with the step's
// interface flow (Neumann design) or the 3D surface pressure (Dirichlet
// design) and take the nodal pressures, component flows and volumes.
static int netlist_solve_update(crimson_netlist* nl, double delt) {
    if (!nl->connect_nodes.empty())
        return fail("netlist: a member of a closed loop is solved through its loop", CRIMSON_ERR_STATE);
    build_system(nl, delt);
    assemble_rhs(nl);
    const int st = solve(nl);
    if (st != CRIMSON_OK) return st;
    take_solution(nl, nl->x.data());
    return CRIMSON_OK;
}

int crimson_netlist_update(crimson_netlist* nl, double delt, double interface_flow) {
    if (!nl || !(delt > 0.0) || !std::isfinite(interface_flow)) return CRIMSON_ERR_ARG;
    if (!nl->flow_permitted)
        return fail("netlist: the circuit is in the Dirichlet design; update it with the 3D surface pressure",
                    CRIMSON_ERR_STATE);
    nl->last_q = interface_flow;
    return netlist_solve_update(nl, delt);
}

int crimson_netlist_update_pressure(crimson_netlist* nl, double delt, double interface_pressure) {
    if (!nl || !(delt > 0.0) || !std::isfinite(interface_pressure)) return CRIMSON_ERR_ARG;
    if (nl->flow_permitted)
        return fail("netlist: the circuit is in the Neumann design; update it with the 3D interface flow",
                    CRIMSON_ERR_STATE);
    nl->last_p3d = interface_pressure;
    return netlist_solve_update(nl, delt);
}

// finalizeLPNAtEndOfTimestep (NetlistCircuit.cxx:732-737): the current
// pressures and flows become the histories, then the diodes switch
// (CircuitData.cxx:357-377; rule CircuitComponent.cxx:4-17).
int crimson_netlist_finalize_step(crimson_netlist* nl) {
    if (!nl) return CRIMSON_ERR_ARG;
    for (NetlistNode& d : nl->node)
        if (d.has_hist) d.hist = node_pressure(d);
    for (int j : nl->hist_comps) nl->comp[j].hist_flow = nl->comp[j].flow;
    for (int j : nl->vol_comps) nl->comp[j].hist_volume = nl->comp[j].volume;
    const double tol = 1e-8;
    for (NetlistComp& c : nl->comp) {
        if (c.kind != CRIMSON_NETLIST_DIODE) continue;
        const bool gradient = node_pressure(nl->node[c.start - 1]) - node_pressure(nl->node[c.end - 1]) >= 0.0 - tol;
        const bool forward = c.flow >= tol;
        c.open = gradient || forward;
    }
    // detectWhetherClosedDiodesStopAllFlowAt3DInterface for the next step
    // (initialiseAtStartOfTimestep, NetlistCircuit.cxx:723-728)
    nl->flow_permitted = detect_flow_permitted(nl);
    return CRIMSON_OK;
}

// The parameters a control system adjusts between steps
// (ControlSystemsManager.cxx:125-330): a component's parameter value, a
// pressure chamber's unstressed volume, a node's pressure (the prescribed
// value of a fixed-pressure node) or a component's fixed prescribed flow.
static double* netlist_parameter(crimson_netlist* nl, int what, int index) {
    switch (what) {
        case CRIMSON_NETLIST_PARAM_COMPONENT:
            return index >= 1 && index <= nl->nc ? &nl->comp[(size_t)index - 1].value : nullptr;
        case CRIMSON_NETLIST_PARAM_UNSTRESSED_VOLUME:
            return index >= 1 && index <= nl->nc && nl->comp[(size_t)index - 1].kind == CRIMSON_NETLIST_PRESSURE_CHAMBER
                       ? &nl->comp[(size_t)index - 1].unstressed
                       : nullptr;
        case CRIMSON_NETLIST_PARAM_PRESSURE: {
            if (index < 1 || index > nl->np) return nullptr;
            NetlistNode& d = nl->node[(size_t)index - 1];
            return d.fixed ? &d.fixed_p : &d.p;
        }
        case CRIMSON_NETLIST_PARAM_FLOW:
            return index >= 1 && index <= nl->nc && nl->comp[(size_t)index - 1].flow_kind == CRIMSON_NETLIST_FLOW_FIXED
                       ? &nl->comp[(size_t)index - 1].flow_fixed
                       : nullptr;
        default:
            return nullptr;
    }
}

int crimson_netlist_get_parameter(crimson_netlist* nl, int what, int index, double* value) {
    if (!nl || !value) return CRIMSON_ERR_ARG;
    const double* v = netlist_parameter(nl, what, index);
    if (!v) return fail("netlist: no such parameter (kind, index) in this circuit");
    *value = *v;
    return CRIMSON_OK;
}

int crimson_netlist_set_parameter(crimson_netlist* nl, int what, int index, double value) {
    if (!nl || !std::isfinite(value)) return CRIMSON_ERR_ARG;
    double* v = netlist_parameter(nl, what, index);
    if (!v) return fail("netlist: no such parameter (kind, index) in this circuit");
    if (what == CRIMSON_NETLIST_PARAM_COMPONENT && value == 0.0) {
        const int k = nl->comp[(size_t)index - 1].kind;
        if (k == CRIMSON_NETLIST_CAPACITOR || k == CRIMSON_NETLIST_PRESSURE_CHAMBER)
            return fail("netlist: a capacitance or elastance cannot be 0");
    }
    *v = value;
    return CRIMSON_OK;
}

int crimson_netlist_get(const crimson_netlist* nl, double* pressures, double* flows, int* open, double* volumes) {
    if (!nl) return CRIMSON_ERR_ARG;
    for (int i = 0; pressures && i < nl->np; ++i) pressures[i] = node_pressure(nl->node[i]);
    for (int j = 0; flows && j < nl->nc; ++j) flows[j] = nl->comp[j].flow;
    for (int j = 0; open && j < nl->nc; ++j) open[j] = nl->comp[j].open ? 1 : 0;
    for (int j = 0; volumes && j < nl->nc; ++j) volumes[j] = nl->comp[j].volume;
    return CRIMSON_OK;
}

int crimson_netlist_state_size(const crimson_netlist* nl, int* n) {
    if (!nl || !n) return CRIMSON_ERR_ARG;
    *n = 2 * nl->np + 5 * nl->nc + 2;
    return CRIMSON_OK;
}

// Checkpoint layout: [p (np), hist (np), flow (nc), hist_flow (nc), open (nc),
// volume (nc), hist_volume (nc), last_q, last_p3d]
int crimson_netlist_state(crimson_netlist* nl, double* buf, int set) {
    if (!nl || !buf) return CRIMSON_ERR_ARG;
    const int np = nl->np, nc = nl->nc;
    if (set) {
        for (int i = 0; i < np; ++i) {
            nl->node[i].p = buf[i];
            nl->node[i].hist = buf[np + i];
        }
        for (int j = 0; j < nc; ++j) {
            nl->comp[j].flow = buf[2 * np + j];
            nl->comp[j].hist_flow = buf[2 * np + nc + j];
            nl->comp[j].open = buf[2 * np + 2 * nc + j] != 0.0;
            nl->comp[j].volume = buf[2 * np + 3 * nc + j];
            nl->comp[j].hist_volume = buf[2 * np + 4 * nc + j];
        }
        nl->last_q = buf[2 * np + 5 * nc];
        nl->last_p3d = buf[2 * np + 5 * nc + 1];
        nl->flow_permitted = detect_flow_permitted(nl);
    } else {
        for (int i = 0; i < np; ++i) {
            buf[i] = nl->node[i].p;
            buf[np + i] = nl->node[i].hist;
        }
        for (int j = 0; j < nc; ++j) {
            buf[2 * np + j] = nl->comp[j].flow;
            buf[2 * np + nc + j] = nl->comp[j].hist_flow;
            buf[2 * np + 2 * nc + j] = nl->comp[j].open ? 1.0 : 0.0;
            buf[2 * np + 3 * nc + j] = nl->comp[j].volume;
            buf[2 * np + 4 * nc + j] = nl->comp[j].hist_volume;
        }
        buf[2 * np + 5 * nc] = nl->last_q;
        buf[2 * np + 5 * nc + 1] = nl->last_p3d;
    }
    return CRIMSON_OK;
}

// ---------------------------------------------------------------------------
// Closed loops: ClosedLoopDownstreamSubsection (ClosedLoopDownstreamSubsection
// .cxx:101-500, 609-940).  The upstream circuits' row blocks (each without the
// Kirchhoff rows of its shared nodes) and the loop-closing circuit's block are
// tiled along the diagonal in that order, then one Kirchhoff row per shared
// node of the loop-closing circuit (ascending: the flows of the connected
// upstream circuits at their mapped nodes, in input order, then its own) and
// one pressure-equality row per connection (file order: +1 at the upstream
// node, -1 at the downstream node).  One dense solve gives every member's
// unknowns; the implicit coefficients of upstream circuit k are read from
// the inverse at (its node 1, its 3D-flow row).
// ---------------------------------------------------------------------------

namespace {

void loop_build(crimson_netlist_loop* L, double alfi_delt) {
    std::fill(L->A.begin(), L->A.end(), 0.0);
    std::fill(L->b.begin(), L->b.end(), 0.0);
    const size_t ld = (size_t)L->n;
    const int nm = (int)L->member.size();
    for (int m = 0; m < nm; ++m) {
        build_rows(L->member[m], alfi_delt, L->A.data(), ld, L->row0[m], L->col0[m]);
        rhs_rows(L->member[m], L->b.data(), L->row0[m]);
    }
    int row = L->row0[nm - 1] + L->member[nm - 1]->n - (int)L->member[nm - 1]->connect_nodes.size();
    auto kirchhoff_part = [&](int m, int node) {
        const crimson_netlist* nl = L->member[m];
        const int cf = L->col0[m] + nl->np + (int)nl->hist_nodes.size();
        for (int j = 0; j < nl->nc; ++j) {
            if (nl->comp[j].end == node) L->A[(size_t)row * ld + cf + j] = 1.0;
            if (nl->comp[j].start == node) L->A[(size_t)row * ld + cf + j] = -1.0;
        }
    };
    // appendKirchoffLawsAtInterfacesBetweenCircuits (609-715)
    for (int d : L->down_nodes) {
        for (int k = 0; k < L->nup; ++k)
            for (size_t c = 0; c < L->conn_down.size(); ++c)
                if (L->conn_down[c] == d && L->conn_up[c] == k) {
                    kirchhoff_part(k, L->conn_node[c]);
                    break;
                }
        kirchhoff_part(nm - 1, d);
        ++row;
    }
    // enforcePressureEqualityBetweenDuplicatedNodes (770-840)
    for (size_t c = 0; c < L->conn_down.size(); ++c, ++row) {
        L->A[(size_t)row * ld + L->col0[L->conn_up[c]] + L->conn_node[c] - 1] = 1.0;
        L->A[(size_t)row * ld + L->col0[nm - 1] + L->conn_down[c] - 1] = -1.0;
    }
}

int loop_solve(crimson_netlist_loop* L, double alfi_delt) {
    loop_build(L, alfi_delt);
    return gj_solve(L->n, L->A, L->Ainv, L->b, L->x);
}

}  // namespace

int crimson_netlist_loop_create(crimson_netlist_loop** out, int nupstream, crimson_netlist* const* upstream,
                                crimson_netlist* downstream, int nconn, const int* conn_down_node,
                                const int* conn_upstream, const int* conn_upstream_node) {
    if (!out) return CRIMSON_ERR_ARG;
    *out = nullptr;
    if (nupstream < 1 || !upstream || !downstream || nconn < 1 || !conn_down_node || !conn_upstream ||
        !conn_upstream_node)
        return fail("netlist loop: need upstream circuits, a loop-closing circuit and connections");
    if (downstream->iface_comp >= 0) return fail("netlist loop: the loop-closing circuit has a 3D interface");
    std::vector<std::vector<int>> up_nodes((size_t)nupstream);
    std::vector<int> down_nodes;
    for (int c = 0; c < nconn; ++c) {
        const int k = conn_upstream[c], u = conn_upstream_node[c], d = conn_down_node[c];
        if (k < 0 || k >= nupstream || !upstream[k]) return fail("netlist loop: bad upstream circuit index");
        if (upstream[k]->iface_comp < 0) return fail("netlist loop: an upstream circuit has no 3D interface");
        if (u < 1 || u > upstream[k]->np || d < 1 || d > downstream->np)
            return fail("netlist loop: connection node out of range");
        up_nodes[k].push_back(u);
        down_nodes.push_back(d);
        for (int e = 0; e < c; ++e)
            if (conn_upstream[e] == k && (conn_upstream_node[e] == u || conn_down_node[e] == d))
                return fail("netlist loop: a connection is listed twice");
    }
    for (int k = 0; k < nupstream; ++k) {
        if (up_nodes[k].empty()) return fail("netlist loop: an upstream circuit without a connection");
        std::sort(up_nodes[k].begin(), up_nodes[k].end());
        if (up_nodes[k] != upstream[k]->connect_nodes)
            return fail("netlist loop: an upstream circuit's shared nodes are not its connections");
        for (int e = 0; e < k; ++e)
            if (upstream[e] == upstream[k]) return fail("netlist loop: a circuit is listed twice");
    }
    std::sort(down_nodes.begin(), down_nodes.end());
    down_nodes.erase(std::unique(down_nodes.begin(), down_nodes.end()), down_nodes.end());
    if (down_nodes != downstream->connect_nodes)
        return fail("netlist loop: the loop-closing circuit's shared nodes are not its connections");
    crimson_netlist_loop* L = new (std::nothrow) crimson_netlist_loop;
    if (!L) return CRIMSON_ERR_OOM;
    L->nup = nupstream;
    L->member.assign(upstream, upstream + nupstream);
    L->member.push_back(downstream);
    L->conn_down.assign(conn_down_node, conn_down_node + nconn);
    L->conn_up.assign(conn_upstream, conn_upstream + nconn);
    L->conn_node.assign(conn_upstream_node, conn_upstream_node + nconn);
    L->down_nodes = down_nodes;
    int r = 0, c = 0;
    for (crimson_netlist* nl : L->member) {
        L->row0.push_back(r);
        L->col0.push_back(c);
        r += nl->n - (int)nl->connect_nodes.size();
        c += nl->n;
    }
    L->n = c;
    if (r + (int)down_nodes.size() + nconn != c) {
        delete L;
        return fail("netlist loop: malformed loop (the system is not square)");
    }
    L->A.assign((size_t)c * c, 0.0);
    L->Ainv.assign((size_t)c * c, 0.0);
    L->b.assign((size_t)c, 0.0);
    L->x.assign((size_t)c, 0.0);
    *out = L;
    return CRIMSON_OK;
}

void crimson_netlist_loop_free(crimson_netlist_loop* loop) { delete loop; }

// getImplicitCoefficients (ClosedLoopDownstreamSubsection.cxx:852-888)
int crimson_netlist_loop_implicit_coefficients(crimson_netlist_loop* L, double alfi_delt, double* dp_dq,
                                               double* hop) {
    if (!L || !dp_dq || !hop || !(alfi_delt > 0.0)) return CRIMSON_ERR_ARG;
    const int st = loop_solve(L, alfi_delt);
    if (st != CRIMSON_OK) return st;
    for (int k = 0; k < L->nup; ++k) {
        const crimson_netlist* nl = L->member[k];
        if (!nl->flow_permitted) {  // Dirichlet design: the surface is not coupled
            dp_dq[k] = hop[k] = std::numeric_limits<double>::quiet_NaN();
            continue;
        }
        const size_t row = (size_t)L->col0[k], col = (size_t)(L->row0[k] + iface_row(nl));
        const double g = L->Ainv[row * L->n + col];
        dp_dq[k] = nl->sign * g;
        hop[k] = L->x[row] - g * L->b[col];
    }
    return CRIMSON_OK;
}

// updateLPN of the loop's circuits (NetlistBoundaryCircuitWhenDownstream
// CircuitsExist.cxx:27-52): one solve with Delt and, per upstream circuit,
// its interface flow (Neumann design) or its 3D surface pressure (Dirichlet
// design); every member takes its segment of the solution.
int crimson_netlist_loop_update(crimson_netlist_loop* L, double delt, const double* interface_flow,
                                const double* interface_pressure) {
    if (!L || !(delt > 0.0) || !interface_flow || !interface_pressure) return CRIMSON_ERR_ARG;
    for (int k = 0; k < L->nup; ++k) {
        crimson_netlist* nl = L->member[k];
        const double v = nl->flow_permitted ? interface_flow[k] : interface_pressure[k];
        if (!std::isfinite(v)) return CRIMSON_ERR_ARG;
        if (nl->flow_permitted) nl->last_q = v;
        else nl->last_p3d = v;
    }
    const int st = loop_solve(L, delt);
    if (st != CRIMSON_OK) return st;
    for (size_t m = 0; m < L->member.size(); ++m) take_solution(L->member[m], L->x.data() + L->col0[m]);
    return CRIMSON_OK;
}

int crimson_netlist_loop_finalize_step(crimson_netlist_loop* L) {
    if (!L) return CRIMSON_ERR_ARG;
    for (crimson_netlist* nl : L->member) crimson_netlist_finalize_step(nl);
    return CRIMSON_OK;
}

}  // extern "C"
