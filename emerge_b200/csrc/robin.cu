// Robin / wave-port boundary triangles (ASM/robinbc.py:126-443), one thread per selected triangle.
//
// Each triangle is mapped to its own 2-D frame (x along v1-v0, z along the normal), the closed-form
// 8x8 matrix gamma/(2A)^2 * sum(area-coefficient * gradient-dot) is accumulated exactly as the
// reference does (:187-266), and, for an excited port, the force vector is the 6-point Dunavant
// quadrature of the first/second-kind basis functions dotted with the in-plane incident field
// (:246-290).  Outputs are per-triangle blocks; the host-side mirror accumulates them in the
// reference's triangle order, and the sweep path scatters them onto CSR slots with a
// deterministic segmented sum.
#include "emfem_internal.cuh"
#include "ned2_math.cuh"

namespace emfem {

constexpr int MAX_NPTS = 16;

__device__ double area_coeff(int a, int b, int c, int d) {
    int cnt[7] = {0, 0, 0, 0, 0, 0, 0};
    cnt[a]++; cnt[b]++; cnt[c]++; cnt[d]++;
    const double fact[10] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
    double num = 1; int n = 0;
    for (int i = 1; i < 7; i++) { num *= fact[cnt[i]]; n += cnt[i]; }
    return 2.0 * num / fact[n + 2];
}

__global__ void tri_robin_kernel(long long nn, const double* __restrict__ nodes, long long ns,
                                 const int64_t* __restrict__ tri_nodes, double gre, double gim,
                                 const double2* __restrict__ U, const double* __restrict__ dpts, int npts,
                                 double2* __restrict__ blocks, double2* __restrict__ bvec, int* status) {
    __shared__ double ac[625];
    for (int i = threadIdx.x; i < 625; i += blockDim.x) ac[i] = area_coeff(i / 125, (i / 25) % 5, (i / 5) % 5, i % 5);
    __syncthreads();
    long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= ns) return;
    double gv[3][3];  // [coord][vertex]
    for (int v = 0; v < 3; v++) {
        int64_t id = tri_nodes[v * ns + it];
        if (id < 0 || id >= nn) { flag(status, DEV_BAD_INDEX); id = 0; }
        gv[0][v] = nodes[id]; gv[1][v] = nodes[nn + id]; gv[2][v] = nodes[2 * nn + id];
    }
    double o[3] = {gv[0][0], gv[1][0], gv[2][0]};
    double e1[3] = {gv[0][1] - o[0], gv[1][1] - o[1], gv[2][1] - o[2]};
    double e2[3] = {gv[0][2] - o[0], gv[1][2] - o[1], gv[2][2] - o[2]};
    double zh[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double n = sqrt(zh[0] * zh[0] + zh[1] * zh[1] + zh[2] * zh[2]);
    for (int i = 0; i < 3; i++) zh[i] /= n;
    n = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    double xh[3] = {e1[0] / n, e1[1] / n, e1[2] / n};
    double yh[3] = {zh[1] * xh[2] - zh[2] * xh[1], zh[2] * xh[0] - zh[0] * xh[2], zh[0] * xh[1] - zh[1] * xh[0]};
    n = sqrt(yh[0] * yh[0] + yh[1] * yh[1] + yh[2] * yh[2]);
    for (int i = 0; i < 3; i++) yh[i] /= n;
    double xs[3], ys[3];
    for (int v = 0; v < 3; v++) {
        double d0 = gv[0][v] - o[0], d1 = gv[1][v] - o[1], d2 = gv[2][v] - o[2];
        xs[v] = xh[0] * d0 + xh[1] * d1 + xh[2] * d2;
        ys[v] = yh[0] * d0 + yh[1] * d1 + yh[2] * d2;
    }
    double x1 = xs[0], x2 = xs[1], x3 = xs[2], y1 = ys[0], y2 = ys[1], y3 = ys[2];
    double As[3] = {x2 * y3 - y2 * x3, x3 * y1 - y3 * x1, x1 * y2 - y1 * x2};
    double Bs[3] = {y2 - y3, y3 - y1, y1 - y2};
    double Cs[3] = {x3 - x2, x1 - x3, x2 - x1};
    double Ds[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            Ds[i][j] = sqrt((xs[i] - xs[j]) * (xs[i] - xs[j]) + (ys[i] - ys[j]) * (ys[i] - ys[j]));
    double sg = (x1 - x3) * (y2 - y1) - (x1 - x2) * (y3 - y1);
    double Area = 0.5 * fabs(sg);
    if (!(Area > 0)) flag(status, DEV_DEGENERATE);
    double signA = sg > 0 ? -1.0 : (sg < 0 ? 1.0 : 0.0);
    const int tA = 1, tB = 2, tC = 3;
    double Lt1 = Ds[2][0], Lt2 = Ds[1][0];
    auto AC = [&](int a, int b, int c, int d) { return ac[((a * 5 + b) * 5 + c) * 5 + d] * Area; };
    auto dot2 = [&](int i, int j) { return Bs[i] * Bs[j] + Cs[i] * Cs[j]; };
    double Bm[64];
    for (int i = 0; i < 64; i++) Bm[i] = 0.0;
    cd bv[8];
    for (int i = 0; i < 8; i++) bv[i] = mk(0, 0);
    const int lem0[3] = {0, 1, 0}, lem1[3] = {1, 2, 2};
    const bool excited = U != nullptr;
    // rotate the incident field into the local frame
    double uxr[MAX_NPTS], uxi[MAX_NPTS], uyr[MAX_NPTS], uyi[MAX_NPTS], px[MAX_NPTS], py[MAX_NPTS];
    if (excited) {
        for (int p = 0; p < npts; p++) {
            double2 u0 = U[(0 * npts + p) * ns + it], u1 = U[(1 * npts + p) * ns + it], u2 = U[(2 * npts + p) * ns + it];
            uxr[p] = xh[0] * u0.x + xh[1] * u1.x + xh[2] * u2.x;
            uxi[p] = xh[0] * u0.y + xh[1] * u1.y + xh[2] * u2.y;
            uyr[p] = yh[0] * u0.x + yh[1] * u1.x + yh[2] * u2.x;
            uyi[p] = yh[0] * u0.y + yh[1] * u1.y + yh[2] * u2.y;
            px[p] = x1 * dpts[npts + p] + x2 * dpts[2 * npts + p] + x3 * dpts[3 * npts + p];
            py[p] = y1 * dpts[npts + p] + y2 * dpts[2 * npts + p] + y3 * dpts[3 * npts + p];
        }
    }
    for (int ei = 0; ei < 3; ei++) {
        int a = lem0[ei], b = lem1[ei];
        double Li = Ds[a][b];
        int A = a + 1, B = b + 1;
        for (int ej = 0; ej < 3; ej++) {
            int c = lem0[ej], d = lem1[ej];
            double Lj = Ds[c][d];
            int C = c + 1, D = d + 1;
            double DAC = dot2(a, c), DAD = dot2(a, d), DBC = dot2(b, c), DBD = dot2(b, d);
            double LL = Li * Lj;
            Bm[ei * 8 + ej] += LL * (AC(A, B, C, D) * DAC - AC(A, B, C, C) * DAD - AC(A, A, C, D) * DBC + AC(A, A, C, C) * DBD);
            Bm[ei * 8 + ej + 4] += LL * (AC(A, B, D, D) * DAC - AC(A, B, C, D) * DAD - AC(A, A, D, D) * DBC + AC(A, A, C, D) * DBD);
            Bm[(ei + 4) * 8 + ej] += LL * (AC(B, B, C, D) * DAC - AC(B, B, C, C) * DAD - AC(A, B, C, D) * DBC + AC(A, B, C, C) * DBD);
            Bm[(ei + 4) * 8 + ej + 4] += LL * (AC(B, B, D, D) * DAC - AC(B, B, C, D) * DAD - AC(A, B, D, D) * DBC + AC(A, B, C, D) * DBD);
        }
        double FA = dot2(a, 2), FB = dot2(a, 0), FC = dot2(b, 2), FD = dot2(b, 0), FE = dot2(a, 1), FF = dot2(b, 1);
        Bm[ei * 8 + 3] += Li * Lt1 * (AC(A, B, tA, tB) * FA - AC(A, B, tB, tC) * FB - AC(A, A, tA, tB) * FC + AC(A, A, tB, tC) * FD);
        Bm[ei * 8 + 7] += Li * Lt2 * (AC(A, B, tB, tC) * FB - AC(A, B, tC, tA) * FE - AC(A, A, tB, tC) * FD + AC(A, A, tC, tA) * FF);
        Bm[3 * 8 + ei] += Lt1 * Li * (AC(tA, tB, A, B) * FA - AC(tA, tB, A, A) * FC - AC(tB, tC, A, B) * FB + AC(tB, tC, A, A) * FD);
        Bm[7 * 8 + ei] += Lt2 * Li * (AC(tB, tC, A, B) * FB - AC(tB, tC, A, A) * FD - AC(tC, tA, A, B) * FE + AC(tC, tA, A, A) * FF);
        Bm[(ei + 4) * 8 + 3] += Li * Lt1 * (AC(B, B, tA, tB) * FA - AC(B, B, tB, tC) * FB - AC(A, B, tA, tB) * FC + AC(A, B, tB, tC) * FD);
        Bm[(ei + 4) * 8 + 7] += Li * Lt2 * (AC(B, B, tB, tC) * FB - AC(B, B, tC, tA) * FE - AC(A, B, tB, tC) * FD + AC(A, B, tC, tA) * FF);
        Bm[3 * 8 + ei + 4] += Lt1 * Li * (AC(tA, tB, B, B) * FA - AC(tA, tB, A, B) * FC - AC(tB, tC, B, B) * FB + AC(tB, tC, A, B) * FD);
        Bm[7 * 8 + ei + 4] += Lt2 * Li * (AC(tB, tC, B, B) * FB - AC(tB, tC, A, B) * FD - AC(tC, tA, B, B) * FE + AC(tC, tA, A, B) * FF);
        if (excited) {
            double A1 = As[a], A2 = As[b], B1 = Bs[a], B2 = Bs[b], C1 = Cs[a], C2 = Cs[b];
            double A4 = 4.0 * Area * Area, Ar2 = 1.0 / (2.0 * Area);
            cd s1 = mk(0, 0), s2 = mk(0, 0);
            for (int p = 0; p < npts; p++) {
                double Q = A2 + B2 * px[p] + C2 * py[p], Z = A1 + B1 * px[p] + C1 * py[p];
                double Q2 = Q / A4, Z2 = Z / A4;
                double ex1 = (B1 * Q2 - B2 * Z2) * Z * Ar2, ey1 = (C1 * Q2 - C2 * Z2) * Z * Ar2;
                double ex2 = (B1 * Q2 - B2 * Z2) * Q * Ar2, ey2 = (C1 * Q2 - C2 * Z2) * Q * Ar2;
                double w = dpts[p];
                s1 += w * mk(ex1 * uxr[p] + ey1 * uyr[p], ex1 * uxi[p] + ey1 * uyi[p]);
                s2 += w * mk(ex2 * uxr[p] + ey2 * uyr[p], ex2 * uxi[p] + ey2 * uyi[p]);
            }
            bv[ei] += (signA * Area * Li) * s1;
            bv[ei + 4] += (signA * Area * Li) * s2;
        }
    }
    double H1 = dot2(0, 2), H2 = dot2(0, 0), H3 = dot2(0, 1);
    Bm[3 * 8 + 3] += Lt1 * Lt1 * (AC(tA, tB, tA, tB) * dot2(2, 2) - AC(tA, tB, tB, tC) * H1 - AC(tB, tC, tA, tB) * H1 + AC(tB, tC, tB, tC) * H2);
    Bm[3 * 8 + 7] += Lt1 * Lt2 * (AC(tA, tB, tB, tC) * H1 - AC(tA, tB, tC, tA) * dot2(1, 2) - AC(tB, tC, tB, tC) * H2 + AC(tB, tC, tC, tA) * H3);
    Bm[7 * 8 + 3] += Lt2 * Lt1 * (AC(tB, tC, tA, tB) * H1 - AC(tB, tC, tB, tC) * H2 - AC(tC, tA, tA, tB) * dot2(1, 2) + AC(tC, tA, tB, tC) * H3);
    Bm[7 * 8 + 7] += Lt2 * Lt2 * (AC(tB, tC, tB, tC) * H2 - AC(tB, tC, tC, tA) * H3 - AC(tC, tA, tB, tC) * H3 + AC(tC, tA, tC, tA) * dot2(1, 1));
    if (excited) {
        double FAr = 8.0 * Area * Area * Area;
        cd s1 = mk(0, 0), s2 = mk(0, 0);
        for (int p = 0; p < npts; p++) {
            double x = px[p], y = py[p];
            double Q = As[1] + Bs[1] * x + Cs[1] * y, Z = As[0] + Bs[0] * x + Cs[0] * y;
            double W = (As[2] + Bs[2] * x + Cs[2] * y) / FAr, W2 = Q * W;
            double f1x = Lt1 * (-Bs[0] * W2 + Bs[2] * Z * Q / FAr), f1y = Lt1 * (-Cs[0] * W2 + Cs[2] * Z * Q / FAr);
            double f2x = Lt2 * (Bs[0] * W2 - Bs[1] * Z * W), f2y = Lt2 * (Cs[0] * W2 - Cs[1] * Z * W);
            double w = dpts[p];
            s1 += w * mk(f1x * uxr[p] + f1y * uyr[p], f1x * uxi[p] + f1y * uyi[p]);
            s2 += w * mk(f2x * uxr[p] + f2y * uyr[p], f2x * uxi[p] + f2y * uyi[p]);
        }
        bv[3] += (signA * Area) * s1;
        bv[7] += (signA * Area) * s2;
        for (int k = 0; k < 8; k++) bvec[it * 8 + k] = make_double2(bv[k].x, bv[k].y);
    }
    // COEFF = gamma / (2A)^2
    double den = (2.0 * Area) * (2.0 * Area);
    cd coeff = mk(gre / den, gim / den);
    for (int k = 0; k < 64; k++) {
        cd v = Bm[k] * coeff;
        blocks[it * 64 + k] = make_double2(v.x, v.y);
    }
}

}  // namespace emfem

using namespace emfem;

extern "C" int emfem_ned2_tri_robin(emfem_handle h, int64_t n_nodes, const double* nodes, int64_t n_sel,
                                    const int64_t* tri_nodes, double gamma_re, double gamma_im, const void* U,
                                    const double* dpts, int npts, void* blocks, void* bvec) {
    EMFEM_REQUIRE(h && nodes && tri_nodes && blocks && n_sel >= 0, "emfem_ned2_tri_robin: bad argument");
    EMFEM_REQUIRE(U == nullptr || (dpts != nullptr && bvec != nullptr && npts > 0 && npts <= MAX_NPTS),
                  "emfem_ned2_tri_robin: an excited port needs dpts, bvec and 1 <= npts <= %d", MAX_NPTS);
    if (n_sel == 0) return EMFEM_OK;
    tri_robin_kernel<<<grid_for(n_sel, 128), 128, 0, h->h.stream>>>(
        n_nodes, nodes, n_sel, tri_nodes, gamma_re, gamma_im, (const double2*)U, dpts, U ? npts : 0,
        (double2*)blocks, (double2*)bvec, h->h.dev_status);
    EMFEM_LAUNCH("tri_robin_kernel");
    return EMFEM_OK;
}

// ---- second-order absorbing boundary correction ------------------------------------------------
// Restates abc_order_2_terms (ASM/robin_abc_order2.py:192-327): per triangle, in its plane frame
// (x along the first edge, z the normal), cf * L_i L_j * (int curl_t N_i curl_t N_j - int div_t N_i div_t N_j) * |A|
// over the 6-point rule that module carries (8-digit weights and points, :190-193).  The triangle's
// nodes are in sorted order, so its edges are (0,1), (1,2), (0,2) (Mesh3D tri_to_edge order).
__constant__ double ABC2_DPTS[4][6] = {
    {0.22338159, 0.22338159, 0.22338159, 0.10995174, 0.10995174, 0.10995174},
    {0.10810302, 0.44594849, 0.44594849, 0.81684757, 0.09157621, 0.09157621},
    {0.44594849, 0.44594849, 0.10810302, 0.09157621, 0.09157621, 0.81684757},
    {0.44594849, 0.10810302, 0.44594849, 0.09157621, 0.81684757, 0.09157621}};

__global__ void tri_abc2_kernel(long long n_nodes, const double* __restrict__ nodes, long long n_sel,
                                const int64_t* __restrict__ tri_nodes, double cf_re, double cf_im,
                                double2* __restrict__ blocks, int* status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_sel) return;
    double v[3][3];
    for (int k = 0; k < 3; k++) {
        long long id = tri_nodes[k * n_sel + t];
        if (id < 0 || id >= n_nodes) { flag(status, DEV_BAD_INDEX); return; }
        for (int d = 0; d < 3; d++) v[d][k] = nodes[d * n_nodes + id];
    }
    double e1[3], e2[3], z[3], xh[3], yh[3];
    for (int d = 0; d < 3; d++) { e1[d] = v[d][1] - v[d][0]; e2[d] = v[d][2] - v[d][0]; }
    z[0] = e1[1] * e2[2] - e1[2] * e2[1]; z[1] = e1[2] * e2[0] - e1[0] * e2[2]; z[2] = e1[0] * e2[1] - e1[1] * e2[0];
    double nz = sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]), ne = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    if (!(nz > 0) || !(ne > 0)) { flag(status, DEV_DEGENERATE); return; }
    for (int d = 0; d < 3; d++) { z[d] /= nz; xh[d] = e1[d] / ne; }
    yh[0] = z[1] * xh[2] - z[2] * xh[1]; yh[1] = z[2] * xh[0] - z[0] * xh[2]; yh[2] = z[0] * xh[1] - z[1] * xh[0];
    double ny = sqrt(yh[0] * yh[0] + yh[1] * yh[1] + yh[2] * yh[2]);
    for (int d = 0; d < 3; d++) yh[d] /= ny;
    double xp[3], yp[3];
    for (int k = 0; k < 3; k++) {
        double r0 = v[0][k] - v[0][0], r1 = v[1][k] - v[1][0], r2 = v[2][k] - v[2][0];
        xp[k] = xh[0] * r0 + xh[1] * r1 + xh[2] * r2;
        yp[k] = yh[0] * r0 + yh[1] * r1 + yh[2] * r2;
    }
    double D[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = sqrt((xp[i] - xp[j]) * (xp[i] - xp[j]) + (yp[i] - yp[j]) * (yp[i] - yp[j]));
    double a[3] = {xp[1] * yp[2] - yp[1] * xp[2], xp[2] * yp[0] - yp[2] * xp[0], xp[0] * yp[1] - yp[0] * xp[1]};
    double b[3] = {yp[1] - yp[2], yp[2] - yp[0], yp[0] - yp[1]};
    double c[3] = {xp[2] - xp[1], xp[0] - xp[2], xp[1] - xp[0]};
    double sA = 0.5 * ((xp[0] - xp[2]) * (yp[1] - yp[0]) - (xp[0] - xp[1]) * (yp[2] - yp[0]));
    double A = fabs(sA), sg = sA > 0 ? 1.0 : (sA < 0 ? -1.0 : 0.0);
    if (!(A > 0)) { flag(status, DEV_DEGENERATE); return; }
    for (int k = 0; k < 3; k++) { a[k] = a[k] * sg / (2 * A); b[k] = b[k] * sg / (2 * A); c[k] = c[k] * sg / (2 * A); }
    // curl_t and div_t of the 8 DOFs [e1 x3, f1, e2 x3, f2] at the 6 points
    double cu[8][6], dv[8][6];
    const int EI[3] = {0, 1, 0}, EJ[3] = {1, 2, 2};
    for (int p = 0; p < 6; p++) {
        double x = xp[0] * ABC2_DPTS[1][p] + xp[1] * ABC2_DPTS[2][p] + xp[2] * ABC2_DPTS[3][p];
        double y = yp[0] * ABC2_DPTS[1][p] + yp[1] * ABC2_DPTS[2][p] + yp[2] * ABC2_DPTS[3][p];
        for (int k = 0; k < 3; k++) {
            int i = EI[k], j = EJ[k];
            double a1 = a[i], b1 = b[i], c1 = c[i], a2 = a[j], b2 = b[j], c2 = c[j];
            double L1 = a1 + b1 * x + c1 * y, L2 = a2 + b2 * x + c2 * y;
            cu[k][p] = -3 * a1 * b1 * c2 + 3 * a1 * b2 * c1 - 3 * b1 * b1 * c2 * x + 3 * b1 * b2 * c1 * x
                       - 3 * b1 * c1 * c2 * y + 3 * b2 * c1 * c1 * y;
            cu[k + 4][p] = -3 * a2 * b1 * c2 + 3 * a2 * b2 * c1 - 3 * b1 * b2 * c2 * x - 3 * b1 * c2 * c2 * y
                           + 3 * b2 * b2 * c1 * x + 3 * b2 * c1 * c2 * y;
            dv[k][p] = b1 * (b1 * L2 - b2 * L1) + c1 * (c1 * L2 - c2 * L1);
            dv[k + 4][p] = b2 * (b1 * L2 - b2 * L1) + c2 * (c1 * L2 - c2 * L1);
        }
        double L1 = a[0] + b[0] * x + c[0] * y, L2 = a[1] + b[1] * x + c[1] * y, L3 = a[2] + b[2] * x + c[2] * y;
        cu[3][p] = -b[1] * (c[0] * L3 - c[2] * L1) + c[1] * (b[0] * L3 - b[2] * L1) + 2 * (b[0] * c[2] - b[2] * c[0]) * L2;
        cu[7][p] = b[2] * (c[0] * L2 - c[1] * L1) - c[2] * (b[0] * L2 - b[1] * L1) - 2 * (b[0] * c[1] - b[1] * c[0]) * L3;
        dv[3][p] = -b[1] * (b[0] * L3 - b[2] * L1) - c[1] * (c[0] * L3 - c[2] * L1);
        dv[7][p] = b[2] * (b[0] * L2 - b[1] * L1) + c[2] * (c[0] * L2 - c[1] * L1);
    }
    double Lr[8];
    for (int k = 0; k < 3; k++) Lr[k] = Lr[k + 4] = D[EI[k]][EJ[k]];
    Lr[3] = D[0][2];
    Lr[7] = D[0][1];
    for (int r = 0; r < 8; r++)
        for (int q = 0; q < 8; q++) {
            double sc = 0, sd = 0;
            for (int p = 0; p < 6; p++) {
                sc += cu[r][p] * cu[q][p] * ABC2_DPTS[0][p];
                sd += dv[r][p] * dv[q][p] * ABC2_DPTS[0][p];
            }
            double m = Lr[r] * Lr[q] * (sc - sd) * A;
            blocks[t * 64 + r * 8 + q] = make_double2(cf_re * m, cf_im * m);
        }
}

extern "C" int emfem_ned2_tri_abc2(emfem_handle h, int64_t n_nodes, const double* nodes, int64_t n_sel,
                                   const int64_t* tri_nodes, double cf_re, double cf_im, void* blocks) {
    EMFEM_REQUIRE(h && nodes && tri_nodes && blocks && n_sel >= 0 && n_nodes > 0, "emfem_ned2_tri_abc2: bad argument");
    if (n_sel == 0) return EMFEM_OK;
    tri_abc2_kernel<<<grid_for(n_sel, 128), 128, 0, h->h.stream>>>(n_nodes, nodes, n_sel, tri_nodes, cf_re, cf_im,
                                                                   (double2*)blocks, h->h.dev_status);
    EMFEM_LAUNCH("tri_abc2_kernel");
    return EMFEM_OK;
}
