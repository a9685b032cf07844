// Nedelec-2 element math shared by the tet kernels (host-and-device inline functions).
//
// The reference builds each 20x20 curl-curl (D) and mass (F) element matrix entry by entry
// (src/emerge/_emerge/physics/microwave/assembly/curlcurl.py:180-412).  Every entry is a short
// linear combination of two families of per-tet invariants:
//   P[a][b] = G_a . (er G_b)                     (16 complex; mass terms)
//   Q[p][q] = (G_p0 x G_p1) . Ms (G_q0 x G_q1)   (6x6 complex over vertex pairs p<q; curl terms)
// with G_i the barycentric-gradient numerators (cofactors), Ms = ur^-1.  This file computes the
// invariants once per tet and evaluates one "pair block" = the 2x2 (first/second-kind) sub-block
// of D and of F coupling one local entity (edge or face) with another, using exactly the
// reference's coefficient formulas (edge-edge :213-264, edge-face :266-317, mirrored face-edge
// :321-328, face-face :330-407).  The DOF/entity layout follows elements/nedelec2.py:42-58.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define EMFEM_HD __host__ __device__ __forceinline__
#define EMFEM_HDC __host__ __device__ constexpr
#else
#define EMFEM_HD inline
#define EMFEM_HDC constexpr
#endif

namespace emfem {

struct cd { double x, y; };

EMFEM_HD cd mk(double x, double y) { cd r; r.x = x; r.y = y; return r; }
EMFEM_HD cd operator+(cd a, cd b) { return mk(a.x + b.x, a.y + b.y); }
EMFEM_HD cd operator-(cd a, cd b) { return mk(a.x - b.x, a.y - b.y); }
EMFEM_HD cd operator-(cd a) { return mk(-a.x, -a.y); }
EMFEM_HD cd operator*(double s, cd a) { return mk(s * a.x, s * a.y); }
EMFEM_HD cd operator*(cd a, double s) { return mk(s * a.x, s * a.y); }
EMFEM_HD cd operator*(cd a, cd b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
EMFEM_HD cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }
EMFEM_HD bool is_zero(cd a) { return a.x == 0.0 && a.y == 0.0; }

// Smith's complex division (R. L. Smith, CACM 5(8), 1962).
EMFEM_HD cd cdiv(cd a, cd b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

// local vertex pairs/triples of a tet (Mesh3D order, mesh3d.py:427,431), 0-based
EMFEM_HDC int tet_edge_p(int e) { return e == 0 ? 0 : e == 1 ? 0 : e == 2 ? 0 : e == 3 ? 1 : e == 4 ? 3 : 2; }
EMFEM_HDC int tet_edge_q(int e) { return e == 0 ? 1 : e == 1 ? 2 : e == 2 ? 3 : e == 3 ? 2 : e == 4 ? 1 : 3; }
EMFEM_HDC int tet_face_v(int f, int k) {
    return f == 0 ? (k == 0 ? 0 : k == 1 ? 1 : 2)
         : f == 1 ? (k == 0 ? 0 : k == 1 ? 2 : 3)
         : f == 2 ? (k == 0 ? 0 : k == 1 ? 3 : 1)
                  : (k == 0 ? 1 : k == 1 ? 2 : 3);
}
// canonical pair index for i<j: (0,1)0 (0,2)1 (0,3)2 (1,2)3 (1,3)4 (2,3)5
EMFEM_HD int pair_index(int i, int j) {
    int lo = i < j ? i : j, hi = i < j ? j : i;
    return lo == 0 ? hi - 1 : (lo == 1 ? hi + 1 : 5);
}

// Per-tet invariants.  The same struct is used in registers and, field by field, in the SoA
// device buffer (see TetInvSoA).
constexpr int INV_P = 0;          // 16 complex -> 32 doubles
constexpr int INV_Q = 32;         // 36 complex -> 72 doubles
constexpr int INV_DS = 104;       // 6 vertex-pair distances (canonical pair order)
constexpr int INV_L = 110;        // 6 edge lengths (tet_to_edge order)
constexpr int INV_SD = 116;       // 1/(6V)^3  (D scale: 6V from the coefficient table times KA)
constexpr int INV_SF = 117;       // 1/(6V)    (F scale)
constexpr int INV_RANK = 118;     // vertex ranks packed as a double-encoded int (2 bits each)
constexpr int INV_NDOUBLE = 119;
constexpr int INV_STRIDE = 120;   // per-tet record length in the array-of-structs buffer (960 B)

// Orientation of the tet's local entities from the rank (0..3) of each vertex's global id,
// packed 2 bits per vertex (no per-thread arrays, so nothing spills to local memory).
struct Orient {
    int code;
    EMFEM_HD int rank(int v) const { return (code >> (2 * v)) & 3; }
    EMFEM_HD void edge(int e, int& a, int& b) const {
        int p = tet_edge_p(e), q = tet_edge_q(e);
        bool keep = rank(p) < rank(q);
        a = keep ? p : q;
        b = keep ? q : p;
    }
    EMFEM_HD void face(int f, int& a, int& b, int& c) const {
        int v0 = tet_face_v(f, 0), v1 = tet_face_v(f, 1), v2 = tet_face_v(f, 2), t;
        if (rank(v1) < rank(v0)) { t = v0; v0 = v1; v1 = t; }
        if (rank(v2) < rank(v1)) { t = v1; v1 = v2; v2 = t; }
        if (rank(v1) < rank(v0)) { t = v0; v0 = v1; v1 = t; }
        a = v0; b = v1; c = v2;
    }
};

EMFEM_HD int pack_rank(const int64_t ids[4]) {
    int code = 0;
    for (int i = 0; i < 4; i++) {
        int r = 0;
        for (int j = 0; j < 4; j++) r += (ids[j] < ids[i]) ? 1 : 0;
        code |= r << (2 * i);
    }
    return code;
}
EMFEM_HD Orient unpack_rank(int code) {
    Orient o;
    o.code = code;
    return o;
}

// Volume coefficient of letters a..d (1..4 name vertices, 0 = absent) without arrays:
// prod k_i! over the letter multiplicities, divided by (n + 3)!.
EMFEM_HD double volume_coeff_closed(int a, int b, int c, int d) {
    int l[4] = {a, b, c, d};
    int n = (a > 0) + (b > 0) + (c > 0) + (d > 0);
    double num = 1.0;
    for (int v = 1; v <= 4; v++) {
        int k = (l[0] == v) + (l[1] == v) + (l[2] == v) + (l[3] == v);
        num *= k == 2 ? 2.0 : k == 3 ? 6.0 : k == 4 ? 24.0 : 1.0;
    }
    double den = n == 0 ? 6.0 : n == 1 ? 24.0 : n == 2 ? 120.0 : n == 3 ? 720.0 : 5040.0;
    return num / den;
}

// det of [[1,p_j,q_j],[1,p_k,q_k],[1,p_l,q_l]]
EMFEM_HD double det1(const double* p, const double* q, int j, int k, int l) {
    return (p[k] * q[l] - p[l] * q[k]) - (p[j] * q[l] - p[l] * q[j]) + (p[j] * q[k] - p[k] * q[j]);
}

// 3x3 complex inverse with the reference's diagonal fast path (mth/optimized.py:342-370).
EMFEM_HD void matinv3(const cd M[9], cd out[9]) {
    for (int i = 0; i < 9; i++) out[i] = mk(0, 0);
    if (is_zero(M[1]) && is_zero(M[2]) && is_zero(M[3]) && is_zero(M[5]) && is_zero(M[6]) && is_zero(M[7])) {
        out[0] = cdiv(mk(1, 0), M[0]); out[4] = cdiv(mk(1, 0), M[4]); out[8] = cdiv(mk(1, 0), M[8]);
        return;
    }
    cd det = M[0] * M[4] * M[8] - M[0] * M[5] * M[7] - M[1] * M[3] * M[8]
           + M[1] * M[5] * M[6] + M[2] * M[3] * M[7] - M[2] * M[4] * M[6];
    out[0] = M[4] * M[8] - M[5] * M[7];
    out[1] = -(M[1] * M[8]) + M[2] * M[7];
    out[2] = M[1] * M[5] - M[2] * M[4];
    out[3] = -(M[3] * M[8]) + M[5] * M[6];
    out[4] = M[0] * M[8] - M[2] * M[6];
    out[5] = -(M[0] * M[5]) + M[2] * M[3];
    out[6] = M[3] * M[7] - M[4] * M[6];
    out[7] = -(M[0] * M[7]) + M[1] * M[6];
    out[8] = M[0] * M[4] - M[1] * M[3];
    for (int i = 0; i < 9; i++) out[i] = cdiv(out[i], det);
}

// Compute the invariants of one tet into inv[INV_NDOUBLE].
//   xs,ys,zs: vertex coordinates in the tet's own order; ids: global node ids;
//   elen: edge lengths in tet_to_edge order; ur, er: row-major 3x3.
EMFEM_HD void tet_invariants(const double xs[4], const double ys[4], const double zs[4], const int64_t ids[4],
                             const double elen[6], const cd ur[9], const cd er[9], double* inv) {
    double G[4][3];
    for (int i = 0; i < 4; i++) {
        int j = i == 0 ? 1 : 0;
        int k = i <= 1 ? 2 : 1;
        int l = i <= 2 ? 3 : 2;
        double s = (i % 2 == 0) ? -1.0 : 1.0;
        G[i][0] = s * det1(ys, zs, j, k, l);
        G[i][1] = -s * det1(xs, zs, j, k, l);
        G[i][2] = s * det1(xs, ys, j, k, l);
    }
    double u0 = xs[1] - xs[0], u1 = ys[1] - ys[0], u2 = zs[1] - zs[0];
    double v0 = xs[2] - xs[0], v1 = ys[2] - ys[0], v2 = zs[2] - zs[0];
    double w0 = xs[3] - xs[0], w1 = ys[3] - ys[0], w2 = zs[3] - zs[0];
    double V6 = fabs(u0 * (v1 * w2 - v2 * w1) + u1 * (v2 * w0 - v0 * w2) + u2 * (v0 * w1 - v1 * w0));
    inv[INV_SD] = 1.0 / (V6 * V6 * V6);
    inv[INV_SF] = 1.0 / V6;
    for (int i = 0; i < 4; i++) for (int j = i + 1; j < 4; j++) {
        double dx = xs[i] - xs[j], dy = ys[i] - ys[j], dz = zs[i] - zs[j];
        inv[INV_DS + pair_index(i, j)] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    for (int e = 0; e < 6; e++) inv[INV_L + e] = elen[e];
    inv[INV_RANK] = (double)pack_rank(ids);

    // P = G^T er G
    cd eG[4][3];
    for (int b = 0; b < 4; b++)
        for (int i = 0; i < 3; i++) eG[b][i] = er[3 * i] * G[b][0] + er[3 * i + 1] * G[b][1] + er[3 * i + 2] * G[b][2];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            cd p = G[a][0] * eG[b][0] + G[a][1] * eG[b][1] + G[a][2] * eG[b][2];
            inv[INV_P + 2 * (4 * a + b)] = p.x;
            inv[INV_P + 2 * (4 * a + b) + 1] = p.y;
        }
    // Q over canonical pairs
    cd Ms[9];
    matinv3(ur, Ms);
    double X[6][3];
    for (int i = 0; i < 4; i++) for (int j = i + 1; j < 4; j++) {
        int p = pair_index(i, j);
        X[p][0] = G[i][1] * G[j][2] - G[i][2] * G[j][1];
        X[p][1] = G[i][2] * G[j][0] - G[i][0] * G[j][2];
        X[p][2] = G[i][0] * G[j][1] - G[i][1] * G[j][0];
    }
    for (int q = 0; q < 6; q++) {
        cd mx[3];
        for (int i = 0; i < 3; i++) mx[i] = Ms[3 * i] * X[q][0] + Ms[3 * i + 1] * X[q][1] + Ms[3 * i + 2] * X[q][2];
        for (int p = 0; p < 6; p++) {
            cd v = X[p][0] * mx[0] + X[p][1] * mx[1] + X[p][2] * mx[2];
            inv[INV_Q + 2 * (6 * p + q)] = v.x;
            inv[INV_Q + 2 * (6 * p + q) + 1] = v.y;
        }
    }
}

// Invariant accessor over a strided layout: field f of tet t lives at base[f * stride].
struct InvView {
    const double* base;
    long long stride;
    EMFEM_HD double g(int f) const { return base[(long long)f * stride]; }
    EMFEM_HD cd P(int a, int b) const { int f = INV_P + 2 * (4 * a + b); return mk(g(f), g(f + 1)); }
    // (Ga x Gb) . Ms (Gc x Gd) for oriented pairs
    EMFEM_HD cd Q(int a, int b, int c, int d) const {
        int p = pair_index(a, b), q = pair_index(c, d);
        double s = ((a < b) == (c < d)) ? 1.0 : -1.0;
        int f = INV_Q + 2 * (6 * p + q);
        return mk(s * g(f), s * g(f + 1));
    }
    EMFEM_HD double Ds(int a, int b) const { return g(INV_DS + pair_index(a, b)); }
    EMFEM_HD double L(int e) const { return g(INV_L + e); }
};

// The same accessors over one tet's record in the array-of-structs buffer (records of INV_STRIDE doubles,
// 16-byte aligned): on the device every complex invariant is one 16-byte load instead of two 8-byte
// ones, with the same values (so the same results) as InvView.
struct InvRec {
    const double* base;
    EMFEM_HD double g(int f) const { return base[f]; }
    EMFEM_HD cd c(int f) const {
#if defined(__CUDA_ARCH__)
        const double2 v = __ldg(reinterpret_cast<const double2*>(base + f));
        return mk(v.x, v.y);
#else
        return mk(base[f], base[f + 1]);
#endif
    }
    EMFEM_HD cd P(int a, int b) const { return c(INV_P + 2 * (4 * a + b)); }
    EMFEM_HD cd Q(int a, int b, int cc, int d) const {
        int p = pair_index(a, b), q = pair_index(cc, d);
        double s = ((a < b) == (cc < d)) ? 1.0 : -1.0;
        cd v = c(INV_Q + 2 * (6 * p + q));
        return mk(s * v.x, s * v.y);
    }
    EMFEM_HD double Ds(int a, int b) const { return g(INV_DS + pair_index(a, b)); }
    EMFEM_HD double L(int e) const { return g(INV_L + e); }
};
static_assert(INV_STRIDE % 2 == 0 && INV_P % 2 == 0 && INV_Q % 2 == 0, "complex invariants are 16-byte aligned");

// Volume coefficient table: vc[A*125 + B*25 + C*5 + D] = prod k_i! / (sum k_i + 3)!,
// letters 1..4 name vertices, 0 = absent (curlcurl.py:64-92).
EMFEM_HD void fill_volume_table(double* vc) {
    const double fact[10] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
    for (int a = 0; a < 5; a++) for (int b = 0; b < 5; b++)
    for (int c = 0; c < 5; c++) for (int d = 0; d < 5; d++) {
        int cnt[7] = {0, 0, 0, 0, 0, 0, 0};
        cnt[a]++; cnt[b]++; cnt[c]++; cnt[d]++;
        double num = 1; int n = 0;
        for (int i = 1; i < 7; i++) { num *= fact[cnt[i]]; n += cnt[i]; }
        vc[((a * 5 + b) * 5 + c) * 5 + d] = num / fact[n + 3];
    }
}

struct VTab {
    const double* vc;
    EMFEM_HD double v(int A, int B) const { return vc[(A * 5 + B) * 25]; }
    EMFEM_HD double v(int A, int B, int C, int D) const { return vc[((A * 5 + B) * 5 + C) * 5 + D]; }
};

// One pair block: row entity slot sx, column entity slot sy (0..5 edges, 6..9 faces).
// d[0..3] = D at (x1,y1),(x1,y2),(x2,y1),(x2,y2) (1 = first-kind DOF, 2 = second-kind), f[] same for F.
// Values include the final element scaling.
template <class IV>
EMFEM_HD void pair_block(const IV& I, const Orient& o, const VTab& T, int sx, int sy, cd d[4], cd f[4]) {
    const bool xe = sx < 6, ye = sy < 6;
    if (xe && ye) {
        int a, b, c, dd; o.edge(sx, a, b); o.edge(sy, c, dd);
        int A = a + 1, B = b + 1, C = c + 1, D = dd + 1;
        double L12 = I.L(sx) * I.L(sy);
        cd fac = (9.0 * L12) * I.Q(a, b, c, dd);
        d[0] = fac * T.v(A, C); d[1] = fac * T.v(A, D); d[2] = fac * T.v(B, C); d[3] = fac * T.v(B, D);
        cd pac = I.P(a, c), pad = I.P(a, dd), pbc = I.P(b, c), pbd = I.P(b, dd);
        f[0] = L12 * (T.v(A, B, C, D) * pac - T.v(A, B, C, C) * pad - T.v(A, A, C, D) * pbc + T.v(A, A, C, C) * pbd);
        f[1] = L12 * (T.v(A, B, D, D) * pac - T.v(A, B, C, D) * pad - T.v(A, A, D, D) * pbc + T.v(A, A, C, D) * pbd);
        f[2] = L12 * (T.v(B, B, C, D) * pac - T.v(B, B, C, C) * pad - T.v(A, B, C, D) * pbc + T.v(A, B, C, C) * pbd);
        f[3] = L12 * (T.v(B, B, D, D) * pac - T.v(B, B, C, D) * pad - T.v(A, B, D, D) * pbc + T.v(A, B, C, D) * pbd);
    } else if (xe != ye) {
        // edge-face block; a face row uses the transposed edge-face block (curlcurl.py:321-328)
        int es = xe ? sx : sy, fs = (xe ? sy : sx) - 6;
        int a, b, c, dd, ff; o.edge(es, a, b); o.face(fs, c, dd, ff);
        int A = a + 1, B = b + 1, C = c + 1, D = dd + 1, F = ff + 1;
        double L1 = I.L(es), Lab2 = I.Ds(c, dd), Lac2 = I.Ds(c, ff);
        cd qcf = I.Q(a, b, c, ff), qdf = I.Q(a, b, dd, ff), qcd = I.Q(a, b, c, dd);
        cd paf = I.P(a, ff), pac = I.P(a, c), pbf = I.P(b, ff), pbc = I.P(b, c), pad = I.P(a, dd), pbd = I.P(b, dd);
        double k0 = L1 * Lac2, k1 = L1 * Lab2;
        cd e00 = k0 * (-6.0 * T.v(A, D) * qcf - 3.0 * T.v(A, C) * qdf - 3.0 * T.v(A, F) * qcd);
        cd e01 = k1 * (6.0 * T.v(A, F) * qcd + 3.0 * T.v(A, D) * qcf - 3.0 * T.v(A, C) * qdf);
        cd e10 = k0 * (-6.0 * T.v(B, D) * qcf - 3.0 * T.v(B, C) * qdf - 3.0 * T.v(B, F) * qcd);
        cd e11 = k1 * (6.0 * T.v(B, F) * qcd + 3.0 * T.v(B, D) * qcf - 3.0 * T.v(B, C) * qdf);
        cd g00 = k0 * (T.v(A, B, C, D) * paf - T.v(A, B, D, F) * pac - T.v(A, A, C, D) * pbf + T.v(A, A, D, F) * pbc);
        cd g01 = k1 * (T.v(A, B, D, F) * pac - T.v(A, B, F, C) * pad - T.v(A, A, D, F) * pbc + T.v(A, A, C, F) * pbd);
        cd g10 = k0 * (T.v(B, B, C, D) * paf - T.v(B, B, D, F) * pac - T.v(A, B, C, D) * pbf + T.v(A, B, D, F) * pbc);
        cd g11 = k1 * (T.v(B, B, D, F) * pac - T.v(B, B, F, C) * pad - T.v(A, B, D, F) * pbc + T.v(A, B, F, C) * pbd);
        if (xe) {
            d[0] = e00; d[1] = e01; d[2] = e10; d[3] = e11;
            f[0] = g00; f[1] = g01; f[2] = g10; f[3] = g11;
        } else {
            d[0] = e00; d[1] = e10; d[2] = e01; d[3] = e11;
            f[0] = g00; f[1] = g10; f[2] = g01; f[3] = g11;
        }
    } else {
        int a, b, e, c, dd, ff; o.face(sx - 6, a, b, e); o.face(sy - 6, c, dd, ff);
        int A = a + 1, B = b + 1, E = e + 1, C = c + 1, D = dd + 1, F = ff + 1;
        double Lac1 = I.Ds(a, e), Lab1 = I.Ds(a, b), Lac2 = I.Ds(c, ff), Lab2 = I.Ds(c, dd);
        cd ae_cf = I.Q(a, e, c, ff), ae_df = I.Q(a, e, dd, ff), ae_cd = I.Q(a, e, c, dd);
        cd be_cf = I.Q(b, e, c, ff), be_df = I.Q(b, e, dd, ff), be_cd = I.Q(b, e, c, dd);
        cd ab_cf = I.Q(a, b, c, ff), ab_df = I.Q(a, b, dd, ff), ab_cd = I.Q(a, b, c, dd);
        cd pef = I.P(e, ff), pec = I.P(e, c), ped = I.P(e, dd);
        cd paf = I.P(a, ff), pac = I.P(a, c), pad = I.P(a, dd);
        cd pbf = I.P(b, ff), pbc = I.P(b, c), pbd = I.P(b, dd);
        double vAD = T.v(A, D), vAC = T.v(A, C), vAF = T.v(A, F), vBF = T.v(B, F), vBC = T.v(B, C), vBD = T.v(B, D);
        double vDE = T.v(E, D), vEF = T.v(E, F), vCE = T.v(E, C);
        cd q1 = 2.0 * vAD * be_cf + vAC * be_df + vAF * be_cd;
        cd q2 = -2.0 * vAF * be_cd - vAD * be_cf + vAC * be_df;
        d[0] = (Lac1 * Lac2) * (4.0 * vBD * ae_cf + 2.0 * vBC * ae_df + 2.0 * vBF * ae_cd + q1 + 2.0 * vDE * ab_cf + vCE * ab_df + vEF * ab_cd);
        d[1] = (Lac1 * Lab2) * (-4.0 * vBF * ae_cd - 2.0 * vBD * ae_cf + 2.0 * vBC * ae_df + q2 - 2.0 * vEF * ab_cd - vDE * ab_cf + vCE * ab_df);
        d[2] = (Lab1 * Lac2) * (-4.0 * vDE * ab_cf - 2.0 * vCE * ab_df - 2.0 * vEF * ab_cd - 2.0 * vBD * ae_cf - vBC * ae_df - vBF * ae_cd + q1);
        d[3] = (Lab1 * Lab2) * (4.0 * vEF * ab_cd + 2.0 * vDE * ab_cf - 2.0 * vCE * ab_df + 2.0 * vBF * ae_cd + vBD * ae_cf - vBC * ae_df + q2);
        double vABCD = T.v(A, B, C, D), vABDF = T.v(A, B, D, F), vBCDF = T.v(B, C, D, F), vBEDF = T.v(B, E, D, F);
        double vABFC = T.v(A, B, F, C), vBEFC = T.v(B, E, F, C), vEACD = T.v(E, A, C, D), vEADF = T.v(E, A, D, F);
        double vACEF = T.v(A, C, E, F);
        f[0] = (Lac1 * Lac2) * (vABCD * pef - vABDF * pec - vBCDF * paf + vBEDF * pac);
        f[1] = (Lac1 * Lab2) * (vABDF * pec - vABFC * ped - vBEDF * pac + vBEFC * pad);
        f[2] = (Lab1 * Lac2) * (vBCDF * paf - vBEDF * pac - vEACD * pbf + vEADF * pbc);
        f[3] = (Lab1 * Lab2) * (vBEDF * pac - vBEFC * pad - vEADF * pbc + vACEF * pbd);
    }
    double sD = I.g(INV_SD), sF = I.g(INV_SF);
    for (int i = 0; i < 4; i++) { d[i] = sD * d[i]; f[i] = sF * f[i]; }
}

// Local DOF row/column index of the first (k=0) or second (k=1) kind DOF of entity slot s.
EMFEM_HD int local_dof(int s, int k) { return s < 6 ? s + 10 * k : s + 10 * k; }

}  // namespace emfem
