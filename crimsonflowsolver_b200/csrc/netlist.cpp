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
void build_system(crimson_netlist* nl, double alfi_delt) {
    const int n = nl->n;
    std::fill(nl->A.begin(), nl->A.end(), 0.0);
    auto a = [&](int r, int c) -> double& { return nl->A[(size_t)r * n + c]; };
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
void assemble_rhs(crimson_netlist* nl) {
    std::fill(nl->b.begin(), nl->b.end(), 0.0);
    int row = first_prescribed_row(nl);
    // a fixed pressure, or the 3D surface pressure at the interface node
    // (Pressure_3DInterface, NetlistCircuit.cxx:1386-1410)
    for (int nd : design_pp(nl)) nl->b[row++] = nl->node[nd - 1].fixed ? nl->node[nd - 1].fixed_p : nl->last_p3d;
    for (int nd : nl->hist_nodes) nl->b[row++] = nl->node[nd - 1].hist;
    for (int j : design_pf(nl)) {
        const NetlistComp& c = nl->comp[j];
        nl->b[row++] = c.flow_kind == CRIMSON_NETLIST_FLOW_3D ? nl->last_q * nl->sign : c.flow_fixed;
    }
    for (int j : nl->hist_comps) nl->b[row++] = nl->comp[j].hist_flow;
    for (int j : nl->vol_comps) nl->b[row++] = nl->comp[j].hist_volume;
    // a chamber's second row: compliance * pressure = volume - unstressed volume
    int r = 0;
    for (int j = 0; j < nl->nc; ++j, ++r)
        if (nl->comp[j].kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) nl->b[++r] = -nl->comp[j].unstressed;
}

// solveLinearSystem (NetlistCircuit.cxx:1723-1733): the inverse of the
// system matrix (Gauss-Jordan with partial pivoting), then x = A^-1 b.
int solve(crimson_netlist* nl) {
    const int n = nl->n;
    std::vector<double> m(nl->A);
    std::vector<double>& inv = nl->Ainv;
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
        for (int c = 0; c < n; ++c) s += inv[(size_t)i * n + c] * nl->b[c];
        nl->x[i] = s;
    }
    for (double v : nl->x)
        if (!std::isfinite(v)) return fail("netlist: non-finite circuit solution", CRIMSON_ERR_NONFINITE);
    return CRIMSON_OK;
}

// detectWhetherClosedDiodesStopAllFlowAt3DInterface (CircuitData.cxx:
// 388-470): walk the flow-permitting components from the interface
// component; flow can cross the interface if one of them has an end with no
// other component attached (a sink) that is not the interface node.
bool detect_flow_permitted(const crimson_netlist* nl) {
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
    if (!out) return CRIMSON_ERR_ARG;
    *out = nullptr;
    if (ncomp < 1 || nnodes < 1 || !kind || !start_node || !end_node || !value || !initial_pressure)
        return fail("netlist: need at least one component and one node");
    if (npres < 0 || nflow < 1 || (npres > 0 && (!pres_node || !pres_value)) || !flow_comp || !flow_kind ||
        !flow_value)
        return fail("netlist: bad prescribed pressure / flow lists");
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
    // (NetlistCircuit.cxx:1770-1790), so the interface node is node 1.
    if (n3d != 1) return bad("netlist: exactly one component must carry the 3D interface flow");
    if (interface_node != 1) return bad("netlist: the 3D interface node must be node 1");
    nl->iface_node = interface_node;
    const NetlistComp& ic = nl->comp[nl->iface_comp];
    if (ic.start != interface_node && ic.end != interface_node)
        return bad("netlist: the 3D-flow component does not touch the interface node");
    if (uses[interface_node - 1] != 1) return bad("netlist: the interface node must belong to exactly one component");
    if (nl->node[interface_node - 1].fixed) return bad("netlist: the interface node cannot have a prescribed pressure");
    nl->sign = ic.start == interface_node ? 1.0 : -1.0;
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
        if (uses[i] > 1) nl->kirch_nodes.push_back(i + 1);
    const int nv = (int)nl->vol_comps.size();
    if (nl->nchamber + (int)(nl->kirch_nodes.size() + nl->pp_nodes.size() + nl->pf_comps.size()) != nnodes + nv)
        return bad("netlist: malformed circuit (the system is not square)");
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
    build_system(nl, delt);
    assemble_rhs(nl);
    const int st = solve(nl);
    if (st != CRIMSON_OK) return st;
    for (int i = 0; i < nl->np; ++i) nl->node[i].p = nl->x[i];
    const int cf = col_flow(nl);
    for (int j = 0; j < nl->nc; ++j) nl->comp[j].flow = nl->x[(size_t)cf + j];
    // volumes; a chamber passes E (V - V_unstressed) to its start node
    // (giveComponentsTheirVolumesFromSolutionVector, NetlistCircuit.cxx:
    // 1636-1660; CircuitComponent.cxx:188-209)
    const int cv = col_vol(nl);
    for (int j : nl->vol_comps) {
        NetlistComp& c = nl->comp[j];
        c.volume = nl->x[(size_t)cv + nl->vol_ord[j]];
        if (c.kind == CRIMSON_NETLIST_PRESSURE_CHAMBER) nl->node[(size_t)c.start - 1].p = (c.volume - c.unstressed) * c.value;
    }
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

}  // extern "C"
