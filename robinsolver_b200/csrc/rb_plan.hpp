// rb_plan.hpp -- host-side tree geometry of the HPS factor/solve (no CUDA calls).
//
// Restates the reference's tree construction so that every node of a level has the same shape:
//   node_divide  robin_tree_module.f90:1369-1412  (cut the longest side, first on ties; child1 is
//                the lower half; child1%iface = 2*edge, child2%iface = 2*edge-1; isbndry inherited)
//   get_h        fd_module.f90:1060-1084          (grid = max(ceiling(w/h_tgt), 3), h = w/grid)
//   merge ptbox  robin_tree_module.f90:404-407    (child1's grid doubled along the cut)
//   get_pt_face  fd_module.f90:1033-1049          (faces x1 x2 y1 y2 hold b, b, a, a points in 2D;
//                                                  x1 x2 y1 y2 z1 z2 hold bc, bc, ac, ac, ab, ab in 3D)
// A merged node's face is its children's faces concatenated, child1's part first (the block
// placement of compute_RTR, robin_tree_module.f90:538-615), in 2D and 3D alike.
// Nodes of level l are numbered 0..2^l-1 left to right, so node i's children are 2i and 2i+1 and
// the leaf order is the DFS order of get_solution (robin_output_module.f90:305-322).
#pragma once
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace rb {

struct PlanLevel {
    int nnodes = 0;
    int a = 0, b = 0, c = 1;     // grid (ptbox) of every node of the level (c = 1 in 2D)
    int nb = 0;                  // boundary points: 2(a+b) in 2D, 2(bc+ac+ab) in 3D
    int pf[6] = {0, 0, 0, 0, 0, 0};    // points per face x1 x2 y1 y2 (z1 z2)
    int off[6] = {0, 0, 0, 0, 0, 0};   // face offsets in the node's boundary ordering
    std::vector<double> lo, hi;  // nnodes*3 box corners
    std::vector<unsigned char> isb;  // nnodes*2d: face lies on the domain boundary
    // merge of this level's nodes (children on level+1); unused on the leaf level
    int edge = -1;               // cut axis, 0 = x, 1 = y
    int iface1 = 0, iface2 = 0;  // 1-based interface face of child1 / child2
    int m = 0;                   // interface points
    int nbc = 0;                 // child boundary points
    int n1 = 0, n2 = 0;          // child non-interface points
    int o1 = 0, o2 = 0;          // offsets of the interface faces in the children
    std::vector<int> pmap1, pmap2;  // parent boundary index of each child non-interface point
};

struct Plan {
    int d = 2, L = 0;
    double domain_lo[3] = {0, 0, 0}, domain_hi[3] = {0, 0, 0};
    double h_tgt = 0.0, kb = 0.0;
    std::vector<PlanLevel> lv;   // 0..L
    std::vector<double> leaf_h;  // d per leaf (each leaf's own h from get_h)
    double h_last[3] = {0, 0, 0};// robin_tree%opts%h after the factorization: the last leaf's
    int nf() const { return 2 * d; }
    int nleaves() const { return lv.back().nnodes; }
    int leaf_a() const { return lv.back().a; }
    int leaf_b() const { return lv.back().b; }
    int leaf_c() const { return lv.back().c; }
    int leaf_nb() const { return lv.back().nb; }
    int leaf_interior() const { return leaf_a() * leaf_b() * leaf_c(); }
    int leaf_n() const { return leaf_nb() + leaf_interior(); }
};

// Builds the plan; returns an empty string on success or the reference's error message.
inline std::string build_plan(int d, int L, const double* domain6, double h_tgt, double kb, Plan& P) {
    if (d != 2 && d != 3) return "Error in ROBIN_TREE_FACTOR: Dimension must be 2 or 3.";
    for (int j = 0; j < 3; ++j)
        if (domain6[2 * j + 1] - domain6[2 * j] < 0) return "Error in ROBIN_TREE_FACTOR: Invalid operator domain format.";
    if (L < 1 || L > 24) return "tree level count L must be in 1..24";
    if (!(h_tgt > 0.0)) return "solve_opts%h_tgt must be positive";
    P = Plan();
    P.d = d; P.L = L; P.h_tgt = h_tgt; P.kb = kb;
    for (int j = 0; j < 3; ++j) { P.domain_lo[j] = domain6[2 * j]; P.domain_hi[j] = domain6[2 * j + 1]; }
    P.lv.resize(L + 1);
    PlanLevel& r = P.lv[0];
    r.nnodes = 1;
    r.lo.assign(P.domain_lo, P.domain_lo + 3);
    r.hi.assign(P.domain_hi, P.domain_hi + 3);
    const int nf = 2 * d;
    r.isb.assign(nf, 1);
    // top-down bisection (node_divide)
    for (int l = 0; l < L; ++l) {
        PlanLevel& p = P.lv[l];
        PlanLevel& c = P.lv[l + 1];
        c.nnodes = 2 * p.nnodes;
        c.lo.resize(3 * c.nnodes); c.hi.resize(3 * c.nnodes);
        c.isb.assign((size_t)nf * c.nnodes, 0);
        for (int i = 0; i < p.nnodes; ++i) {
            double w[3] = {0, 0, 0};
            for (int j = 0; j < d; ++j) w[j] = p.hi[3 * i + j] - p.lo[3 * i + j];
            int edge = 0;
            for (int j = 1; j < 3; ++j) if (w[j] > w[edge]) edge = j;   // maxloc: first maximum
            if (i == 0) p.edge = edge;
            else if (p.edge != edge) return "Error: Interface sizes of node children do not match (cut axis differs within a level)";
            const int c1 = 2 * i, c2 = 2 * i + 1;
            for (int j = 0; j < 3; ++j) {
                c.lo[3 * c1 + j] = p.lo[3 * i + j]; c.hi[3 * c1 + j] = p.hi[3 * i + j];
                c.lo[3 * c2 + j] = p.lo[3 * i + j]; c.hi[3 * c2 + j] = p.hi[3 * i + j];
            }
            c.hi[3 * c1 + edge] = p.lo[3 * i + edge] + w[edge] * 0.5;
            c.lo[3 * c2 + edge] = c.hi[3 * c1 + edge];
            const int if1 = 2 * (edge + 1), if2 = 2 * (edge + 1) - 1;
            for (int f = 0; f < nf; ++f)
                if (p.isb[nf * i + f]) {
                    if (f + 1 != if1) c.isb[nf * c1 + f] = 1;
                    if (f + 1 != if2) c.isb[nf * c2 + f] = 1;
                }
        }
        p.iface1 = 2 * (p.edge + 1);
        p.iface2 = 2 * (p.edge + 1) - 1;
    }
    // leaf grids (get_h), must be uniform
    PlanLevel& lf = P.lv[L];
    P.leaf_h.resize((size_t)d * lf.nnodes);
    for (int i = 0; i < lf.nnodes; ++i) {
        int grid[3] = {1, 1, 1};
        for (int j = 0; j < d; ++j) {
            const double w = lf.hi[3 * i + j] - lf.lo[3 * i + j];
            const double q = std::ceil(w / h_tgt);
            if (!(q < 1e7)) return "leaf grid too large";
            grid[j] = std::max((int)q, 3);
            P.leaf_h[(size_t)d * i + j] = w / grid[j];
        }
        if (i == 0) { lf.a = grid[0]; lf.b = grid[1]; lf.c = grid[2]; }
        else if (grid[0] != lf.a || grid[1] != lf.b || grid[2] != lf.c)
            return "Error: Interface sizes of node children do not match (leaf grids differ)";
    }
    for (int j = 0; j < 3; ++j) P.h_last[j] = j < d ? P.leaf_h[(size_t)d * (lf.nnodes - 1) + j] : 0.0;
    // bottom-up grids of the merged nodes
    for (int l = L - 1; l >= 0; --l) {
        PlanLevel& p = P.lv[l];
        const PlanLevel& c = P.lv[l + 1];
        int ax = -1;
        for (int i = 0; i < p.nnodes; ++i) {
            double diff[3] = {0, 0, 0};
            for (int j = 0; j < d; ++j) {
                const double wp = p.hi[3 * i + j] - p.lo[3 * i + j];
                const double wc = c.hi[3 * (2 * i) + j] - c.lo[3 * (2 * i) + j];
                diff[j] = std::fabs(wp - wc);
            }
            int a_ = 0;                          // maxloc: the first largest difference
            for (int j = 1; j < d; ++j)
                if (diff[j] > diff[a_]) a_ = j;
            if (ax < 0) ax = a_;
            else if (ax != a_) return "Error: Interface sizes of node children do not match (merge axis differs within a level)";
        }
        p.a = c.a; p.b = c.b; p.c = c.c;
        if (ax == 0) p.a *= 2; else if (ax == 1) p.b *= 2; else p.c *= 2;
    }
    for (int l = 0; l <= L; ++l) {
        PlanLevel& p = P.lv[l];
        if (d == 2) {
            p.pf[0] = p.b; p.pf[1] = p.b; p.pf[2] = p.a; p.pf[3] = p.a;
        } else {
            p.pf[0] = p.pf[1] = p.b * p.c;
            p.pf[2] = p.pf[3] = p.a * p.c;
            p.pf[4] = p.pf[5] = p.a * p.b;
        }
        p.off[0] = 0;
        for (int f = 1; f < nf; ++f) p.off[f] = p.off[f - 1] + p.pf[f - 1];
        p.nb = p.off[nf - 1] + p.pf[nf - 1];
    }
    for (int l = 0; l < L; ++l) {
        PlanLevel& p = P.lv[l];
        const PlanLevel& c = P.lv[l + 1];
        const int i1 = p.iface1, i2 = p.iface2;
        p.m = c.pf[i1 - 1];
        if (p.m != c.pf[i2 - 1]) return "Error: Interface sizes of node children do not match";
        p.nbc = c.nb;
        p.o1 = c.off[i1 - 1];
        p.o2 = c.off[i2 - 1];
        p.n1 = c.nb - p.m;
        p.n2 = c.nb - p.m;
        p.pmap1.resize(p.n1); p.pmap2.resize(p.n2);
        for (int k = 0; k < 2; ++k) {
            const int o = k == 0 ? p.o1 : p.o2;
            std::vector<int>& pm = k == 0 ? p.pmap1 : p.pmap2;
            for (int t = 0; t < (int)pm.size(); ++t) {
                const int phys = t < o ? t : t + p.m;
                int f = 0;
                while (f < nf - 1 && phys >= c.off[f + 1]) ++f;
                const int loc = phys - c.off[f];
                int base = p.off[f];
                const bool along_cut = (f + 1 == i1) || (f + 1 == i2);
                if (k == 1 && !along_cut) base += c.pf[f];
                pm[t] = base + loc;
            }
        }
    }
    return "";
}

}  // namespace rb
