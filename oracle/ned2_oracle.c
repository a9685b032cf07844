/*
 * CPU oracle for the Nedelec-2 hot path.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check
 * and the CPU-baseline leg of bench.py call it as the checker; the product path never does.
 *
 * A plain-C restatement of EMerge's numba kernels, formula for formula, so that its outputs can
 * be compared with the CUDA path on machines where the reference checkout is absent.  It is
 * pinned against golden vectors produced by the reference itself (tests/golden/make_golden.py).
 *
 *   ned2_tet_stiff_mass  src/emerge/_emerge/physics/microwave/assembly/curlcurl.py:180-412
 *   tet_coefficients_bcd curlcurl.py:99-138      volume_coeff / cache  curlcurl.py:64-92
 *   _matrix_builder      curlcurl.py:419-466     local_mapping  src/emerge/_emerge/mth/optimized.py:293-327
 *   matinv               optimized.py:342-370    compute_distances optimized.py:330-338
 *   ned2_tri_stiff_force .../assembly/robinbc.py:126-292    ned2_tri_stiff robinbc.py:314-427
 *   area_coeff / cache   robinbc.py:36-55
 *
 * Complex arrays are interleaved (re, im) doubles, i.e. numpy complex128.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef double complex cplx;

static const int64_t FACT[10] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
static double VOLC[5][5][5][5];
static double AREAC[5][5][5][5];
static int tables_ready = 0;

/* Integral of a product of barycentric coordinates; letter 0 means "absent".
 * volume: prod k_i! / (sum k_i + 3)!   area: 2 prod k_i! / (sum k_i + 2)! */
static void init_tables(void) {
    if (tables_ready) return;
    for (int a = 0; a < 5; a++) for (int b = 0; b < 5; b++)
    for (int c = 0; c < 5; c++) for (int d = 0; d < 5; d++) {
        int cnt[7] = {0, 0, 0, 0, 0, 0, 0};
        cnt[a]++; cnt[b]++; cnt[c]++; cnt[d]++;
        int64_t num = 1; int n = 0;
        for (int i = 1; i < 7; i++) { num *= FACT[cnt[i]]; n += cnt[i]; }
        VOLC[a][b][c][d] = (double)num / (double)FACT[n + 3];
        AREAC[a][b][c][d] = 2.0 * (double)num / (double)FACT[n + 2];
    }
    tables_ready = 1;
}

static inline void cross_r(const double *u, const double *v, double *w) {
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
}
static inline void matvec(const cplx M[3][3], const double *v, cplx *w) {
    for (int i = 0; i < 3; i++) w[i] = M[i][0] * v[0] + M[i][1] * v[1] + M[i][2] * v[2];
}
static inline cplx dot_rc(const double *u, const cplx *w) {
    return u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
}
/* (u1 x u2) . M (v1 x v2) */
static inline cplx cross_pair(const double *u1, const double *u2, const cplx M[3][3],
                              const double *v1, const double *v2) {
    double cu[3], cv[3]; cplx mv[3];
    cross_r(u1, u2, cu); cross_r(v1, v2, cv); matvec(M, cv, mv);
    return dot_rc(cu, mv);
}

/* 3x3 minor determinant with a column of ones: rows j,k,l of (p, q) */
static inline double det1(const double *p, const double *q, int j, int k, int l) {
    return (p[k] * q[l] - p[l] * q[k]) - (p[j] * q[l] - p[l] * q[j]) + (p[j] * q[k] - p[k] * q[j]);
}

void oracle_matinv(const cplx M[3][3], cplx out[3][3]) {
    memset(out, 0, 9 * sizeof(cplx));
    if (M[0][1] == 0 && M[0][2] == 0 && M[1][0] == 0 && M[1][2] == 0 && M[2][0] == 0 && M[2][1] == 0) {
        out[0][0] = 1.0 / M[0][0]; out[1][1] = 1.0 / M[1][1]; out[2][2] = 1.0 / M[2][2];
        return;
    }
    cplx det = M[0][0] * M[1][1] * M[2][2] - M[0][0] * M[1][2] * M[2][1] - M[0][1] * M[1][0] * M[2][2]
             + M[0][1] * M[1][2] * M[2][0] + M[0][2] * M[1][0] * M[2][1] - M[0][2] * M[1][1] * M[2][0];
    out[0][0] = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    out[0][1] = -M[0][1] * M[2][2] + M[0][2] * M[2][1];
    out[0][2] = M[0][1] * M[1][2] - M[0][2] * M[1][1];
    out[1][0] = -M[1][0] * M[2][2] + M[1][2] * M[2][0];
    out[1][1] = M[0][0] * M[2][2] - M[0][2] * M[2][0];
    out[1][2] = -M[0][0] * M[1][2] + M[0][2] * M[1][0];
    out[2][0] = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    out[2][1] = -M[0][0] * M[2][1] + M[0][1] * M[2][0];
    out[2][2] = M[0][0] * M[1][1] - M[0][1] * M[1][0];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) out[i][j] /= det;
}

/* One tet: Dmat (curl-curl with Ms = ur^-1) and Fmat (mass with Mm = er), row-major 20x20. */
void oracle_tet_element(const double xs[4], const double ys[4], const double zs[4],
                        const double elen[6], const int64_t lem[2][6], const int64_t ltm[3][4],
                        const cplx Ms[3][3], const cplx Mm[3][3], cplx D[20][20], cplx F[20][20]) {
    init_tables();
    double G[4][3];
    static const int others[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    for (int i = 0; i < 4; i++) {
        int j = others[i][0], k = others[i][1], l = others[i][2];
        double s = (i % 2 == 0) ? -1.0 : 1.0;
        G[i][0] = s * det1(ys, zs, j, k, l);
        G[i][1] = -s * det1(xs, zs, j, k, l);
        G[i][2] = s * det1(xs, ys, j, k, l);
    }
    double u[3] = {xs[1] - xs[0], ys[1] - ys[0], zs[1] - zs[0]};
    double v[3] = {xs[2] - xs[0], ys[2] - ys[0], zs[2] - zs[0]};
    double w[3] = {xs[3] - xs[0], ys[3] - ys[0], zs[3] - zs[0]};
    double uv[3]; cross_r(v, w, uv);
    double V = fabs(u[0] * uv[0] + u[1] * uv[1] + u[2] * uv[2]) / 6.0;
    double Ds[4][4];
    for (int i = 0; i < 4; i++) for (int j = i; j < 4; j++) {
        Ds[i][j] = sqrt((xs[i] - xs[j]) * (xs[i] - xs[j]) + (ys[i] - ys[j]) * (ys[i] - ys[j]) +
                        (zs[i] - zs[j]) * (zs[i] - zs[j]));
        Ds[j][i] = Ds[i][j];
    }
    double V6 = 6.0 * V;
    double KA = 1.0 / pow(V6, 4), KB = 1.0 / (V6 * V6);
    double VC[5][5][5][5];
    for (int a = 0; a < 625; a++) (&VC[0][0][0][0])[a] = (&VOLC[0][0][0][0])[a] * V6;

    for (int ei = 0; ei < 6; ei++) {
        int a = (int)lem[0][ei], b = (int)lem[1][ei];
        int A = a + 1, B = b + 1;
        const double *GA = G[a], *GB = G[b];
        double L1 = elen[ei];
        for (int ej = 0; ej < 6; ej++) {
            int c = (int)lem[0][ej], d = (int)lem[1][ej];
            int C = c + 1, Dd = d + 1;
            const double *GC = G[c], *GD = G[d];
            double L2 = elen[ej], L12 = L1 * L2;
            cplx MC[3], MD[3];
            matvec(Mm, GC, MC); matvec(Mm, GD, MD);
            cplx pac = dot_rc(GA, MC), pad = dot_rc(GA, MD), pbc = dot_rc(GB, MC), pbd = dot_rc(GB, MD);
            cplx fac = L12 * 9.0 * cross_pair(GA, GB, Ms, GC, GD);
            D[ei][ej] = fac * VC[A][C][0][0];
            D[ei][ej + 10] = fac * VC[A][Dd][0][0];
            D[ei + 10][ej] = fac * VC[B][C][0][0];
            D[ei + 10][ej + 10] = fac * VC[B][Dd][0][0];
            F[ei][ej] = L12 * (VC[A][B][C][Dd] * pac - VC[A][B][C][C] * pad - VC[A][A][C][Dd] * pbc + VC[A][A][C][C] * pbd);
            F[ei][ej + 10] = L12 * (VC[A][B][Dd][Dd] * pac - VC[A][B][C][Dd] * pad - VC[A][A][Dd][Dd] * pbc + VC[A][A][C][Dd] * pbd);
            F[ei + 10][ej] = L12 * (VC[B][B][C][Dd] * pac - VC[B][B][C][C] * pad - VC[A][B][C][Dd] * pbc + VC[A][B][C][C] * pbd);
            F[ei + 10][ej + 10] = L12 * (VC[B][B][Dd][Dd] * pac - VC[B][B][C][Dd] * pad - VC[A][B][Dd][Dd] * pbc + VC[A][B][C][Dd] * pbd);
        }
        for (int ej = 0; ej < 4; ej++) {
            int c = (int)ltm[0][ej], d = (int)ltm[1][ej], f = (int)ltm[2][ej];
            int C = c + 1, Dd = d + 1, Ff = f + 1;
            const double *GC = G[c], *GD = G[d], *GF = G[f];
            double Lab2 = Ds[c][d], Lac2 = Ds[c][f];
            cplx q_cf = cross_pair(GA, GB, Ms, GC, GF);
            cplx q_df = cross_pair(GA, GB, Ms, GD, GF);
            cplx q_cd = cross_pair(GA, GB, Ms, GC, GD);
            cplx MF[3], MC[3], MD[3];
            matvec(Mm, GF, MF); matvec(Mm, GC, MC); matvec(Mm, GD, MD);
            cplx paf = dot_rc(GA, MF), pac = dot_rc(GA, MC), pbf = dot_rc(GB, MF), pbc = dot_rc(GB, MC);
            cplx pad = dot_rc(GA, MD), pbd = dot_rc(GB, MD);
            double vAD = VC[A][Dd][0][0], vAC = VC[A][C][0][0], vAF = VC[A][Ff][0][0];
            double vBF = VC[B][Ff][0][0], vBC = VC[B][C][0][0], vBD = VC[B][Dd][0][0];
            D[ei][ej + 6] = L1 * Lac2 * (-6.0 * vAD * q_cf - 3.0 * vAC * q_df - 3.0 * vAF * q_cd);
            D[ei][ej + 16] = L1 * Lab2 * (6.0 * vAF * q_cd + 3.0 * vAD * q_cf - 3.0 * vAC * q_df);
            D[ei + 10][ej + 6] = L1 * Lac2 * (-6.0 * vBD * q_cf - 3.0 * vBC * q_df - 3.0 * vBF * q_cd);
            D[ei + 10][ej + 16] = L1 * Lab2 * (6.0 * vBF * q_cd + 3.0 * vBD * q_cf - 3.0 * vBC * q_df);
            F[ei][ej + 6] = L1 * Lac2 * (VC[A][B][C][Dd] * paf - VC[A][B][Dd][Ff] * pac - VC[A][A][C][Dd] * pbf + VC[A][A][Dd][Ff] * pbc);
            F[ei][ej + 16] = L1 * Lab2 * (VC[A][B][Dd][Ff] * pac - VC[A][B][Ff][C] * pad - VC[A][A][Dd][Ff] * pbc + VC[A][A][C][Ff] * pbd);
            F[ei + 10][ej + 6] = L1 * Lac2 * (VC[B][B][C][Dd] * paf - VC[B][B][Dd][Ff] * pac - VC[A][B][C][Dd] * pbf + VC[A][B][Dd][Ff] * pbc);
            F[ei + 10][ej + 16] = L1 * Lab2 * (VC[B][B][Dd][Ff] * pac - VC[B][B][Ff][C] * pad - VC[A][B][Dd][Ff] * pbc + VC[A][B][Ff][C] * pbd);
        }
    }
    /* transposed copies of the edge/face blocks (curlcurl.py:321-328) */
    for (int i = 0; i < 4; i++) for (int j = 0; j < 6; j++) {
        D[i + 6][j] = D[j][i + 6];            F[i + 6][j] = F[j][i + 6];
        D[i + 16][j] = D[j][i + 16];          F[i + 16][j] = F[j][i + 16];
        D[i + 6][j + 10] = D[j + 10][i + 6];  F[i + 6][j + 10] = F[j + 10][i + 6];
        D[i + 16][j + 10] = D[j + 10][i + 16]; F[i + 16][j + 10] = F[j + 10][i + 16];
    }
    for (int ei = 0; ei < 4; ei++) {
        int a = (int)ltm[0][ei], b = (int)ltm[1][ei], e = (int)ltm[2][ei];
        int A = a + 1, B = b + 1, E = e + 1;
        const double *GA = G[a], *GB = G[b], *GE = G[e];
        double Lac1 = Ds[a][e], Lab1 = Ds[a][b];
        for (int ej = 0; ej < 4; ej++) {
            int c = (int)ltm[0][ej], d = (int)ltm[1][ej], f = (int)ltm[2][ej];
            int C = c + 1, Dd = d + 1, Ff = f + 1;
            const double *GC = G[c], *GD = G[d], *GF = G[f];
            double Lac2 = Ds[c][f], Lab2 = Ds[c][d];
            double vAD = VC[A][Dd][0][0], vAC = VC[A][C][0][0], vAF = VC[A][Ff][0][0];
            double vBF = VC[B][Ff][0][0], vBC = VC[B][C][0][0], vBD = VC[B][Dd][0][0];
            double vDE = VC[E][Dd][0][0], vEF = VC[E][Ff][0][0], vCE = VC[E][C][0][0];
            double vABCD = VC[A][B][C][Dd], vABDF = VC[A][B][Dd][Ff], vACEF = VC[A][C][E][Ff];
            double vABCF = VC[A][B][Ff][C], vBCDF = VC[B][C][Dd][Ff], vBEDF = VC[B][E][Dd][Ff];
            double vEACD = VC[E][A][C][Dd], vBEFC = VC[B][E][Ff][C], vEADF = VC[E][A][Dd][Ff];
            cplx ae_cf = cross_pair(GA, GE, Ms, GC, GF), ae_df = cross_pair(GA, GE, Ms, GD, GF), ae_cd = cross_pair(GA, GE, Ms, GC, GD);
            cplx be_cf = cross_pair(GB, GE, Ms, GC, GF), be_df = cross_pair(GB, GE, Ms, GD, GF), be_cd = cross_pair(GB, GE, Ms, GC, GD);
            cplx ab_cf = cross_pair(GA, GB, Ms, GC, GF), ab_df = cross_pair(GA, GB, Ms, GD, GF), ab_cd = cross_pair(GA, GB, Ms, GC, GD);
            cplx MF[3], MC[3], MD[3];
            matvec(Mm, GF, MF); matvec(Mm, GC, MC); matvec(Mm, GD, MD);
            cplx pef = dot_rc(GE, MF), pec = dot_rc(GE, MC), ped = dot_rc(GE, MD);
            cplx paf = dot_rc(GA, MF), pac = dot_rc(GA, MC), pad = dot_rc(GA, MD);
            cplx pbf = dot_rc(GB, MF), pbc = dot_rc(GB, MC), pbd = dot_rc(GB, MD);
            cplx q1 = 2.0 * vAD * be_cf + vAC * be_df + vAF * be_cd;
            cplx q2 = -2.0 * vAF * be_cd - vAD * be_cf + vAC * be_df;
            D[ei + 6][ej + 6] = Lac1 * Lac2 * (4.0 * vBD * ae_cf + 2.0 * vBC * ae_df + 2.0 * vBF * ae_cd + q1 + 2.0 * vDE * ab_cf + vCE * ab_df + vEF * ab_cd);
            D[ei + 6][ej + 16] = Lac1 * Lab2 * (-4.0 * vBF * ae_cd - 2.0 * vBD * ae_cf + 2.0 * vBC * ae_df + q2 - 2.0 * vEF * ab_cd - vDE * ab_cf + vCE * ab_df);
            D[ei + 16][ej + 6] = Lab1 * Lac2 * (-4.0 * vDE * ab_cf - 2.0 * vCE * ab_df - 2.0 * vEF * ab_cd - 2.0 * vBD * ae_cf - vBC * ae_df - vBF * ae_cd + q1);
            D[ei + 16][ej + 16] = Lab1 * Lab2 * (4.0 * vEF * ab_cd + 2.0 * vDE * ab_cf - 2.0 * vCE * ab_df + 2.0 * vBF * ae_cd + vBD * ae_cf - vBC * ae_df + q2);
            F[ei + 6][ej + 6] = Lac1 * Lac2 * (vABCD * pef - vABDF * pec - vBCDF * paf + vBEDF * pac);
            F[ei + 6][ej + 16] = Lac1 * Lab2 * (vABDF * pec - vABCF * ped - vBEDF * pac + vBEFC * pad);
            F[ei + 16][ej + 6] = Lab1 * Lac2 * (vBCDF * paf - vBEDF * pac - vEACD * pbf + vEADF * pbc);
            F[ei + 16][ej + 16] = Lab1 * Lab2 * (vBEDF * pac - vBEFC * pad - vEADF * pbc + vACEF * pbd);
        }
    }
    for (int i = 0; i < 20; i++) for (int j = 0; j < 20; j++) { D[i][j] *= KA; F[i][j] *= KB; }
}

/* Local slot (0..3) of each global id in `ids` among the tet's vertices `tv`. */
static void local_map(const int64_t tv[4], const int64_t *ids, int n, int64_t *out) {
    for (int j = 0; j < n; j++) {
        out[j] = 0;
        for (int k = 0; k < 4; k++) if (tv[k] == ids[j]) { out[j] = k; break; }
    }
}

/* _matrix_builder: per-tet element matrices plus row-major COO indices.
 * nodes (3, nn); tets (4, nt); tris (3, nf); edges (2, ne); tet_to_field (20, nt);
 * tet_to_edge (6, nt); ur, er (3, 3, nt) complex. */
void oracle_matrix_builder(int64_t nn, int64_t nt, int64_t nf, int64_t ne,
                           const double *nodes, const int64_t *tets, const int64_t *tris,
                           const int64_t *edges, const double *edge_lengths,
                           const int64_t *tet_to_field, const int64_t *tet_to_edge,
                           const cplx *ur, const cplx *er,
                           cplx *dataE, cplx *dataB, int64_t *rows, int64_t *cols) {
    init_tables();
    (void)nf;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; t++) {
        int64_t tv[4];
        double xs[4], ys[4], zs[4], el[6];
        for (int i = 0; i < 4; i++) {
            tv[i] = tets[i * nt + t];
            xs[i] = nodes[0 * nn + tv[i]]; ys[i] = nodes[1 * nn + tv[i]]; zs[i] = nodes[2 * nn + tv[i]];
        }
        int64_t lem[2][6], ltm[3][4];
        for (int e = 0; e < 6; e++) {
            int64_t eid = tet_to_field[e * nt + t];
            int64_t ids[2] = {edges[0 * ne + eid], edges[1 * ne + eid]};
            int64_t loc[2]; local_map(tv, ids, 2, loc);
            lem[0][e] = loc[0]; lem[1][e] = loc[1];
            el[e] = edge_lengths[tet_to_edge[e * nt + t]];
        }
        for (int f = 0; f < 4; f++) {
            int64_t fid = tet_to_field[(6 + f) * nt + t] - ne;
            int64_t ids[3] = {tris[0 * nf + fid], tris[1 * nf + fid], tris[2 * nf + fid]};
            int64_t loc[3]; local_map(tv, ids, 3, loc);
            ltm[0][f] = loc[0]; ltm[1][f] = loc[1]; ltm[2][f] = loc[2];
        }
        cplx U[3][3], Mm[3][3], Ms[3][3];
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
            U[i][j] = ur[(i * 3 + j) * nt + t];
            Mm[i][j] = er[(i * 3 + j) * nt + t];
        }
        oracle_matinv(U, Ms);
        cplx D[20][20], F[20][20];
        oracle_tet_element(xs, ys, zs, el, lem, ltm, Ms, Mm, D, F);
        int64_t p = t * 400;
        for (int i = 0; i < 20; i++) {
            int64_t ri = tet_to_field[i * nt + t];
            for (int j = 0; j < 20; j++) {
                rows[p + 20 * i + j] = ri;
                cols[p + 20 * i + j] = tet_to_field[j * nt + t];
                dataE[p + 20 * i + j] = D[i][j];
                dataB[p + 20 * i + j] = F[i][j];
            }
        }
    }
}

static inline double dot2(const double *u, const double *v) { return u[0] * v[0] + u[1] * v[1]; }

/* Robin triangle 8x8 (and, with Uinc != NULL, the 8-entry force vector).
 * gv (3, 3): rows x, y, z of the three vertices; Uinc (3, npts) complex; dpts (4, npts). */
void oracle_tri_robin(const double gv[9], cplx gamma, const cplx *Uinc, const double *dpts, int npts,
                      cplx Bm[64], cplx bv[8]) {
    init_tables();
    static const int lem[2][3] = {{0, 1, 0}, {1, 2, 2}};
    memset(Bm, 0, 64 * sizeof(cplx));
    if (bv) memset(bv, 0, 8 * sizeof(cplx));
    double o[3] = {gv[0], gv[3], gv[6]};
    double e1[3] = {gv[1] - o[0], gv[4] - o[1], gv[7] - o[2]};
    double e2[3] = {gv[2] - o[0], gv[5] - o[1], gv[8] - o[2]};
    double zh[3], xh[3], yh[3], n;
    cross_r(e1, e2, zh); n = sqrt(zh[0] * zh[0] + zh[1] * zh[1] + zh[2] * zh[2]);
    for (int i = 0; i < 3; i++) zh[i] /= n;
    n = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    for (int i = 0; i < 3; i++) xh[i] = e1[i] / n;
    cross_r(zh, xh, yh); n = sqrt(yh[0] * yh[0] + yh[1] * yh[1] + yh[2] * yh[2]);
    for (int i = 0; i < 3; i++) yh[i] /= n;
    double xs[3], ys[3];
    for (int v = 0; v < 3; v++) {
        double d0 = gv[v] - o[0], d1 = gv[3 + v] - o[1], d2 = gv[6 + v] - o[2];
        xs[v] = xh[0] * d0 + xh[1] * d1 + xh[2] * d2;
        ys[v] = yh[0] * d0 + yh[1] * d1 + yh[2] * d2;
    }
    double x1 = xs[0], x2 = xs[1], x3 = xs[2], y1 = ys[0], y2 = ys[1], y3 = ys[2];
    double As[3] = {x2 * y3 - y2 * x3, x3 * y1 - y3 * x1, x1 * y2 - y1 * x2};
    double Bs[3] = {y2 - y3, y3 - y1, y1 - y2};
    double Cs[3] = {x3 - x2, x1 - x3, x2 - x1};
    double Ds[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
        Ds[i][j] = sqrt((xs[i] - xs[j]) * (xs[i] - xs[j]) + (ys[i] - ys[j]) * (ys[i] - ys[j]));
    double GL[3][2] = {{Bs[0], Cs[0]}, {Bs[1], Cs[1]}, {Bs[2], Cs[2]}};
    double sgnarg = (x1 - x3) * (y2 - y1) - (x1 - x2) * (y3 - y1);
    double Area = 0.5 * fabs(sgnarg);
    double signA = (sgnarg > 0) ? -1.0 : ((sgnarg < 0) ? 1.0 : 0.0);
    const int tA = 1, tB = 2, tC = 3;
    const double *GtA = GL[0], *GtB = GL[1], *GtC = GL[2];
    double Lt1 = Ds[2][0], Lt2 = Ds[1][0];
    double AC[5][5][5][5];
    for (int a = 0; a < 625; a++) (&AC[0][0][0][0])[a] = (&AREAC[0][0][0][0])[a] * Area;

    for (int ei = 0; ei < 3; ei++) {
        int a = lem[0][ei], b = lem[1][ei];
        double Li = Ds[a][b];
        int A = a + 1, B = b + 1;
        const double *GA = GL[a], *GB = GL[b];
        for (int ej = 0; ej < 3; ej++) {
            int c = lem[0][ej], d = lem[1][ej];
            double Lj = Ds[c][d];
            int C = c + 1, D = d + 1;
            const double *GC = GL[c], *GD = GL[d];
            double DAC = dot2(GA, GC), DAD = dot2(GA, GD), DBC = dot2(GB, GC), DBD = dot2(GB, GD);
            double LL = Li * Lj;
            Bm[ei * 8 + ej] += LL * (AC[A][B][C][D] * DAC - AC[A][B][C][C] * DAD - AC[A][A][C][D] * DBC + AC[A][A][C][C] * DBD);
            Bm[ei * 8 + ej + 4] += LL * (AC[A][B][D][D] * DAC - AC[A][B][C][D] * DAD - AC[A][A][D][D] * DBC + AC[A][A][C][D] * DBD);
            Bm[(ei + 4) * 8 + ej] += LL * (AC[B][B][C][D] * DAC - AC[B][B][C][C] * DAD - AC[A][B][C][D] * DBC + AC[A][B][C][C] * DBD);
            Bm[(ei + 4) * 8 + ej + 4] += LL * (AC[B][B][D][D] * DAC - AC[B][B][C][D] * DAD - AC[A][B][D][D] * DBC + AC[A][B][C][D] * DBD);
        }
        double FA = dot2(GA, GtC), FB = dot2(GA, GtA), FC = dot2(GB, GtC), FD = dot2(GB, GtA);
        double FE = dot2(GA, GtB), FF = dot2(GB, GtB);
        Bm[ei * 8 + 3] += Li * Lt1 * (AC[A][B][tA][tB] * FA - AC[A][B][tB][tC] * FB - AC[A][A][tA][tB] * FC + AC[A][A][tB][tC] * FD);
        Bm[ei * 8 + 7] += Li * Lt2 * (AC[A][B][tB][tC] * FB - AC[A][B][tC][tA] * FE - AC[A][A][tB][tC] * FD + AC[A][A][tC][tA] * FF);
        Bm[3 * 8 + ei] += Lt1 * Li * (AC[tA][tB][A][B] * FA - AC[tA][tB][A][A] * FC - AC[tB][tC][A][B] * FB + AC[tB][tC][A][A] * FD);
        Bm[7 * 8 + ei] += Lt2 * Li * (AC[tB][tC][A][B] * FB - AC[tB][tC][A][A] * FD - AC[tC][tA][A][B] * FE + AC[tC][tA][A][A] * FF);
        Bm[(ei + 4) * 8 + 3] += Li * Lt1 * (AC[B][B][tA][tB] * FA - AC[B][B][tB][tC] * FB - AC[A][B][tA][tB] * FC + AC[A][B][tB][tC] * FD);
        Bm[(ei + 4) * 8 + 7] += Li * Lt2 * (AC[B][B][tB][tC] * FB - AC[B][B][tC][tA] * FE - AC[A][B][tB][tC] * FD + AC[A][B][tC][tA] * FF);
        Bm[3 * 8 + ei + 4] += Lt1 * Li * (AC[tA][tB][B][B] * FA - AC[tA][tB][A][B] * FC - AC[tB][tC][B][B] * FB + AC[tB][tC][A][B] * FD);
        Bm[7 * 8 + ei + 4] += Lt2 * Li * (AC[tB][tC][B][B] * FB - AC[tB][tC][A][B] * FD - AC[tC][tA][B][B] * FE + AC[tC][tA][A][B] * FF);
        if (bv) {
            double A1 = As[a], A2 = As[b], B1 = Bs[a], B2 = Bs[b], C1 = Cs[a], C2 = Cs[b];
            cplx s1 = 0, s2 = 0;
            double A4 = 4.0 * Area * Area, Ar2 = 1.0 / (2.0 * Area);
            for (int p = 0; p < npts; p++) {
                double x = x1 * dpts[npts + p] + x2 * dpts[2 * npts + p] + x3 * dpts[3 * npts + p];
                double y = y1 * dpts[npts + p] + y2 * dpts[2 * npts + p] + y3 * dpts[3 * npts + p];
                cplx ux = xh[0] * Uinc[p] + xh[1] * Uinc[npts + p] + xh[2] * Uinc[2 * npts + p];
                cplx uy = yh[0] * Uinc[p] + yh[1] * Uinc[npts + p] + yh[2] * Uinc[2 * npts + p];
                double Q = A2 + B2 * x + C2 * y, Z = A1 + B1 * x + C1 * y;
                double Q2 = Q / A4, Z2 = Z / A4;
                double ex1 = (B1 * Q2 - B2 * Z2) * Z * Ar2, ey1 = (C1 * Q2 - C2 * Z2) * Z * Ar2;
                double ex2 = (B1 * Q2 - B2 * Z2) * Q * Ar2, ey2 = (C1 * Q2 - C2 * Z2) * Q * Ar2;
                s1 += dpts[p] * (ex1 * ux + ey1 * uy);
                s2 += dpts[p] * (ex2 * ux + ey2 * uy);
            }
            bv[ei] += signA * Area * Li * s1;
            bv[ei + 4] += signA * Area * Li * s2;
        }
    }
    double H1 = dot2(GtA, GtC), H2 = dot2(GtA, GtA), H3 = dot2(GtA, GtB);
    Bm[3 * 8 + 3] += Lt1 * Lt1 * (AC[tA][tB][tA][tB] * dot2(GtC, GtC) - AC[tA][tB][tB][tC] * H1 - AC[tB][tC][tA][tB] * H1 + AC[tB][tC][tB][tC] * H2);
    Bm[3 * 8 + 7] += Lt1 * Lt2 * (AC[tA][tB][tB][tC] * H1 - AC[tA][tB][tC][tA] * dot2(GtB, GtC) - AC[tB][tC][tB][tC] * H2 + AC[tB][tC][tC][tA] * H3);
    Bm[7 * 8 + 3] += Lt2 * Lt1 * (AC[tB][tC][tA][tB] * H1 - AC[tB][tC][tB][tC] * H2 - AC[tC][tA][tA][tB] * dot2(GtB, GtC) + AC[tC][tA][tB][tC] * H3);
    Bm[7 * 8 + 7] += Lt2 * Lt2 * (AC[tB][tC][tB][tC] * H2 - AC[tB][tC][tC][tA] * H3 - AC[tC][tA][tB][tC] * H3 + AC[tC][tA][tC][tA] * dot2(GtB, GtB));
    if (bv) {
        cplx s1 = 0, s2 = 0;
        double FAr = 8.0 * Area * Area * Area;
        for (int p = 0; p < npts; p++) {
            double x = x1 * dpts[npts + p] + x2 * dpts[2 * npts + p] + x3 * dpts[3 * npts + p];
            double y = y1 * dpts[npts + p] + y2 * dpts[2 * npts + p] + y3 * dpts[3 * npts + p];
            cplx ux = xh[0] * Uinc[p] + xh[1] * Uinc[npts + p] + xh[2] * Uinc[2 * npts + p];
            cplx uy = yh[0] * Uinc[p] + yh[1] * Uinc[npts + p] + yh[2] * Uinc[2 * npts + p];
            double Q = As[1] + Bs[1] * x + Cs[1] * y, Z = As[0] + Bs[0] * x + Cs[0] * y;
            double W = (As[2] + Bs[2] * x + Cs[2] * y) / FAr, W2 = Q * W;
            double ef1x = Lt1 * (-Bs[0] * W2 + Bs[2] * Z * Q / FAr), ef1y = Lt1 * (-Cs[0] * W2 + Cs[2] * Z * Q / FAr);
            double ef2x = Lt2 * (Bs[0] * W2 - Bs[1] * Z * W), ef2y = Lt2 * (Cs[0] * W2 - Cs[1] * Z * W);
            s1 += dpts[p] * (ef1x * ux + ef1y * uy);
            s2 += dpts[p] * (ef2x * ux + ef2y * uy);
        }
        bv[3] += signA * Area * s1;
        bv[7] += signA * Area * s2;
    }
    cplx coeff = gamma / ((2.0 * Area) * (2.0 * Area));
    for (int i = 0; i < 64; i++) Bm[i] *= coeff;
}

/* compute_bc_entries(_excited) (robinbc.py:294-311, 429-443): accumulate the 64-blocks of the
 * listed triangles into the flat (n_tris*64,) Bmat and, when U is given, the force into Bvec.
 * U is (3, npts, ns) complex as the reference reshapes it; tri_to_field is (8, nf). */
void oracle_robin_entries(int64_t nn, int64_t nf, const double *nodes, const int64_t *tris,
                          const int64_t *tri_ids, int64_t ns, double gamma_re, double gamma_im,
                          const cplx *U, const double *dpts, int npts, const int64_t *tri_to_field,
                          cplx *Bmat, cplx *Bvec) {
    cplx gamma = gamma_re + I * gamma_im;
    cplx *Ul = 0;
    cplx Bm[64], bv[8], Uloc[3 * 64];
    if (npts > 64) return;
    for (int64_t i = 0; i < ns; i++) {
        int64_t it = tri_ids[i];
        double gv[9];
        for (int v = 0; v < 3; v++) {
            int64_t nid = tris[v * nf + it];
            gv[v] = nodes[nid]; gv[3 + v] = nodes[nn + nid]; gv[6 + v] = nodes[2 * nn + nid];
        }
        if (U) {
            for (int c = 0; c < 3; c++) for (int p = 0; p < npts; p++)
                Uloc[c * npts + p] = U[(c * npts + p) * ns + i];
            Ul = Uloc;
            oracle_tri_robin(gv, gamma, Ul, dpts, npts, Bm, bv);
            for (int k = 0; k < 8; k++) Bvec[tri_to_field[k * nf + it]] += bv[k];
        } else {
            oracle_tri_robin(gv, gamma, 0, dpts, npts, Bm, 0);
        }
        for (int k = 0; k < 64; k++) Bmat[it * 64 + k] += Bm[k];
    }
}

#ifdef _OPENMP
#include <omp.h>
#endif
/* Number of host threads the oracle's tet loop uses (the reference's prange width). */
int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}
