// Canonical-order Nedelec-2 pair blocks as fixed sparse linear forms (the table-driven assembly).
//
// The reference orients every edge and face of a tet by the global ids of its vertices
// (curlcurl.py:180-412 sorts the local vertex letters by global node id before it evaluates an entry).
// Renumbering a tet's vertices by rank (rank 0 = smallest global id) therefore makes every local entity
// canonically oriented: in that numbering each pair block (pair_block with the identity orientation) is
//
//     block[q] = r_x[kx] * r_y[ky] * s * sum_k c[csx][csy][q][k] * inv_k          (q = 2 kx + ky)
//
// with inv the 16 complex P and 36 complex Q invariants in canonical vertex order, r the entity length
// factors (edge: its length for both DOF kinds; face with sorted vertices (a, b, c): |ac| for the first
// kind, |ab| for the second), s the D or F element scale, and c real constants (volume coefficients
// times the formulas' integer weights).  The constants are read off pair_block itself on the host, one
// invariant at a time, so the linear forms are the reference's formulas by construction.
#pragma once
#include "ned2_math.cuh"

namespace emfem {

// canonical per-tet record (doubles)
constexpr int CAN_P = 0;           // 16 complex P, canonical vertex order
constexpr int CAN_Q = 32;          // 36 complex Q, canonical pairs
constexpr int CAN_R = 104;         // r[canonical entity 0..9][kind 0..1]
constexpr int CAN_SD = 124;
constexpr int CAN_SF = 125;
constexpr int CAN_RANK = 126;      // original rank code (maps a tet's local slots to canonical ones)
constexpr int CAN_STRIDE = 128;    // 1024 B per tet, 16-byte aligned complex entries

// recipe capacity: terms per output of each block kind (curl-curl D reads Q, mass F reads P)
constexpr int RCP_ND_EE = 1, RCP_ND_EF = 3, RCP_ND_FF = 9, RCP_NF = 4, RCP_ND_MAX = 9;

// Canonical slot of a tet's local entity slot s (0..5 edges, 6..9 faces) for the rank code of its vertices.
EMFEM_HD int canon_edge_of(int ra, int rb) {
    int lo = ra < rb ? ra : rb, hi = ra < rb ? rb : ra;
    // canonical edges are the local edge list over rank-numbered vertices: (0,1)(0,2)(0,3)(1,2)(3,1)(2,3);
    // equal ranks (a tet with a repeated vertex, flagged degenerate by the invariants) map to edge 0, so
    // every result indexes inside the tables
    if (lo == hi) return 0;
    return lo == 0 ? hi - 1 : (lo == 1 ? (hi == 2 ? 3 : 4) : 5);
}
EMFEM_HD int canon_slot(int s, int code) {
    const Orient o = unpack_rank(code);
    if (s < 6) return canon_edge_of(o.rank(tet_edge_p(s)), o.rank(tet_edge_q(s)));
    // faces (0,1,2)(0,2,3)(0,3,1)(1,2,3) miss local vertex 3, 1, 2, 0; a canonical face is named the same way
    const int f = s - 6;
    const int miss = f == 0 ? 3 : f == 1 ? 1 : f == 2 ? 2 : 0;
    const int rm = o.rank(miss);
    return 6 + (rm == 3 ? 0 : rm == 1 ? 1 : rm == 2 ? 2 : 3);
}

// The canonical record of one tet from its invariants in the original layout (INV_*): values are only
// permuted (and sign-flipped for reversed vertex pairs), never recomputed.
EMFEM_HD void canon_record(const double* loc, double* out) {
    const InvView I{loc, 1};
    const int code = (int)loc[INV_RANK];
    const Orient o = unpack_rank(code);
    int pi[4] = {0, 1, 2, 3};                    // pi[r] = local vertex of rank r (stays a valid index
    for (int v = 0; v < 4; v++) pi[o.rank(v)] = v;  // even for the repeated ranks of a degenerate tet)
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            cd v = I.P(pi[a], pi[b]);
            out[CAN_P + 2 * (4 * a + b)] = v.x;
            out[CAN_P + 2 * (4 * a + b) + 1] = v.y;
        }
    for (int p = 0; p < 6; p++)
        for (int q = 0; q < 6; q++) {
            cd v = I.Q(pi[tet_edge_p(p) < tet_edge_q(p) ? tet_edge_p(p) : tet_edge_q(p)],
                       pi[tet_edge_p(p) < tet_edge_q(p) ? tet_edge_q(p) : tet_edge_p(p)],
                       pi[tet_edge_p(q) < tet_edge_q(q) ? tet_edge_p(q) : tet_edge_q(q)],
                       pi[tet_edge_p(q) < tet_edge_q(q) ? tet_edge_q(q) : tet_edge_p(q)]);
            // canonical pair index of (lo, hi) over rank numbers, the layout InvView::Q reads
            int pa = tet_edge_p(p) < tet_edge_q(p) ? tet_edge_p(p) : tet_edge_q(p);
            int pb = tet_edge_p(p) < tet_edge_q(p) ? tet_edge_q(p) : tet_edge_p(p);
            int qa = tet_edge_p(q) < tet_edge_q(q) ? tet_edge_p(q) : tet_edge_q(q);
            int qb = tet_edge_p(q) < tet_edge_q(q) ? tet_edge_q(q) : tet_edge_p(q);
            int f = CAN_Q + 2 * (6 * pair_index(pa, pb) + pair_index(qa, qb));
            out[f] = v.x;
            out[f + 1] = v.y;
        }
    // entity length factors
    for (int ce = 0; ce < 6; ce++) {
        int a = pi[tet_edge_p(ce)], b = pi[tet_edge_q(ce)];
        int e = 0;
        for (int k = 0; k < 6; k++)
            if ((tet_edge_p(k) == a && tet_edge_q(k) == b) || (tet_edge_p(k) == b && tet_edge_q(k) == a)) e = k;
        out[CAN_R + 2 * ce] = I.L(e);
        out[CAN_R + 2 * ce + 1] = I.L(e);
    }
    for (int cf = 0; cf < 4; cf++) {
        // canonical face vertices, ascending rank
        int v0 = tet_face_v(cf, 0), v1 = tet_face_v(cf, 1), v2 = tet_face_v(cf, 2), t;
        if (v1 < v0) { t = v0; v0 = v1; v1 = t; }
        if (v2 < v1) { t = v1; v1 = v2; v2 = t; }
        if (v1 < v0) { t = v0; v0 = v1; v1 = t; }
        out[CAN_R + 2 * (6 + cf)] = I.Ds(pi[v0], pi[v2]);
        out[CAN_R + 2 * (6 + cf) + 1] = I.Ds(pi[v0], pi[v1]);
    }
    out[CAN_SD] = loc[INV_SD];
    out[CAN_SF] = loc[INV_SF];
    out[CAN_RANK] = loc[INV_RANK];
    out[CAN_STRIDE - 1] = 0.0;
}

// Recipe tables for the 100 canonical (row, column) entity pairs b = 10 csx + csy:
// D terms: coefD[(b * 4 + q) * RCP_ND_MAX + k], idxD[...] (Q index 0..35); F terms: coefF[(b * 4 + q) *
// RCP_NF + k], idxF[...] (P index 0..15).  Unused terms have coefficient 0 and index 0.
struct Recipes {
    double coefD[100 * 4 * RCP_ND_MAX];
    double coefF[100 * 4 * RCP_NF];
    unsigned char idxD[100 * 4 * RCP_ND_MAX];
    unsigned char idxF[100 * 4 * RCP_NF];
};

// Reads the recipes off pair_block (identity orientation, unit lengths and scales, one unit invariant at a
// time).  Returns false if a block needs more terms than the capacity or mixes P into D / Q into F.
inline bool build_recipes(Recipes& R) {
    double vt[625];
    fill_volume_table(vt);
    const VTab T{vt};
    int ident = 0;
    for (int v = 0; v < 4; v++) ident |= v << (2 * v);
    const Orient o = unpack_rank(ident);
    double rec[INV_STRIDE];
    for (int i = 0; i < 100 * 4 * RCP_ND_MAX; i++) { R.coefD[i] = 0.0; R.idxD[i] = 0; }
    for (int i = 0; i < 100 * 4 * RCP_NF; i++) { R.coefF[i] = 0.0; R.idxF[i] = 0; }
    for (int b = 0; b < 100; b++) {
        const int sx = b / 10, sy = b % 10;
        const bool xe = sx < 6, ye = sy < 6;
        const int nd = (xe && ye) ? RCP_ND_EE : (xe != ye) ? RCP_ND_EF : RCP_ND_FF;
        int cntD[4] = {0, 0, 0, 0}, cntF[4] = {0, 0, 0, 0};
        for (int k = 0; k < 52; k++) {
            for (int i = 0; i < INV_STRIDE; i++) rec[i] = 0.0;
            for (int i = 0; i < 6; i++) { rec[INV_DS + i] = 1.0; rec[INV_L + i] = 1.0; }
            rec[INV_SD] = 1.0;
            rec[INV_SF] = 1.0;
            rec[INV_RANK] = (double)ident;
            rec[k < 16 ? INV_P + 2 * k : INV_Q + 2 * (k - 16)] = 1.0;
            const InvView I{rec, 1};
            cd d[4], f[4];
            pair_block(I, o, T, sx, sy, d, f);
            for (int q = 0; q < 4; q++) {
                if (d[q].y != 0.0 || f[q].y != 0.0) return false;
                if (d[q].x != 0.0) {
                    if (k < 16 || cntD[q] >= nd) return false;
                    const int at = (b * 4 + q) * RCP_ND_MAX + cntD[q]++;
                    R.coefD[at] = d[q].x;
                    R.idxD[at] = (unsigned char)(k - 16);
                }
                if (f[q].x != 0.0) {
                    if (k >= 16 || cntF[q] >= RCP_NF) return false;
                    const int at = (b * 4 + q) * RCP_NF + cntF[q]++;
                    R.coefF[at] = f[q].x;
                    R.idxF[at] = (unsigned char)k;
                }
            }
        }
    }
    return true;
}

// Recipe terms per block kind, and the packed tables the device reads: block b's D terms start at
// offD[b] (output q at offD[b] + q * nd, nd = 1 / 3 / 9 for edge-edge / edge-face / face-face), its F
// terms at 16 b + 4 q.
EMFEM_HD int recipe_nd(int csx, int csy) {
    const bool xe = csx < 6, ye = csy < 6;
    return (xe && ye) ? RCP_ND_EE : (xe != ye) ? RCP_ND_EF : RCP_ND_FF;
}
constexpr int RCP_TOTAL_D = 36 * 4 * RCP_ND_EE + 48 * 4 * RCP_ND_EF + 16 * 4 * RCP_ND_FF;   // 1296
constexpr int RCP_TOTAL_F = 100 * 4 * RCP_NF;                                                 // 1600
struct PackedRecipes {
    double coefD[RCP_TOTAL_D];
    double coefF[RCP_TOTAL_F];
    int offD[100];
    unsigned char idxD[RCP_TOTAL_D];
    unsigned char idxF[RCP_TOTAL_F];
};

inline bool pack_recipes(PackedRecipes& P) {
    static Recipes R;                      // 40 KB: off the stack
    if (!build_recipes(R)) return false;
    int o = 0;
    for (int b = 0; b < 100; b++) {
        const int nd = recipe_nd(b / 10, b % 10);
        P.offD[b] = o;
        for (int q = 0; q < 4; q++)
            for (int k = 0; k < nd; k++) {
                P.coefD[o + q * nd + k] = R.coefD[(b * 4 + q) * RCP_ND_MAX + k];
                P.idxD[o + q * nd + k] = R.idxD[(b * 4 + q) * RCP_ND_MAX + k];
            }
        o += 4 * nd;
    }
    if (o != RCP_TOTAL_D) return false;
    for (int i = 0; i < RCP_TOTAL_F; i++) { P.coefF[i] = R.coefF[i]; P.idxF[i] = R.idxF[i]; }
    return true;
}

}  // namespace emfem
