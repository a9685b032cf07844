// Port-face overlap integrals for S-parameter extraction on the device.
//
// The reference interpolates each solved field at the Dunavant points of a port face
// (Nedelec2.interpolate_Ef -> ned2_tet_interp, src/emerge/_emerge/elements/ned2_interp.py:142-300)
// and integrates its overlap with the port mode (sparam_field_power / sparam_mode_power,
// src/emerge/_emerge/physics/microwave/sparam.py:71-138, surface_integral in mth/integrals.py:60-100),
// then S[q, p] = field_power / mode_power / sqrt(P_p) (microwave_3d.py:1180-1230).
//
// Here one thread per (port triangle, system) evaluates the field at the triangle's quadrature
// points inside the tet that owns the (boundary) triangle — the only tet containing interior face
// points, which is the tet the reference's point search selects — using the reference's
// interpolation formulas, and accumulates
//   F[t, s] = c_t A_t sum_p W_p E_s(x_p) . conj(m(x_p))      (m = unit-amplitude mode shape)
//   N[t]    = c_t A_t sum_p W_p |m(x_p)|^2
// per triangle; a second kernel sums triangles in order.  The host forms
// S = (F / (scale(k0) N) - [q == p]) / sqrt(P), which is field_power / mode_power of the reference
// with the common factor 1/(2 Z_mode) and the mode amplitude scale(k0) divided out.
#include "emfem_internal.cuh"

namespace emfem {

constexpr int SP_MAX_NPTS = 16;

__device__ __forceinline__ double tet_det3(double ax, double ay, double az, double bx, double by, double bz,
                                           double cx, double cy, double cz) {
    return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
}

// det of [[1,p_j,q_j],[1,p_k,q_k],[1,p_l,q_l]]
__device__ __forceinline__ double sp_det1(double pj, double qj, double pk, double qk, double pl, double ql) {
    return (pk * ql - pl * qk) - (pj * ql - pl * qj) + (pj * qk - pk * qj);
}

__device__ __forceinline__ double sp_dist(const double* xs, const double* ys, const double* zs, int i, int j) {
    double dx = xs[i] - xs[j], dy = ys[i] - ys[j], dz = zs[i] - zs[j];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Interpolation data of one tet (tet_coefficients, ned2_interp.py:59-77) and the field at a point
// in it (ned2_tet_interp, ned2_interp.py:230-295), with the local orientation taken from the global
// node order (local_mapping of the sorted edge / triangle lists).
struct TetInterp {
    double xs[4], ys[4], zs[4], a[4], b[4], c[4], d[4], V1;
    int rank[4];
};

__device__ __forceinline__ bool load_tet_interp(long long nn, const double* __restrict__ nodes, long long nt,
                                                const int64_t* __restrict__ tets, long long T, TetInterp& ti) {
    int64_t vid[4];
    for (int i = 0; i < 4; i++) {
        int64_t id = tets[i * nt + T];
        if (id < 0 || id >= nn) return false;
        vid[i] = id;
        ti.xs[i] = nodes[id]; ti.ys[i] = nodes[nn + id]; ti.zs[i] = nodes[2 * nn + id];
    }
    const double *xs = ti.xs, *ys = ti.ys, *zs = ti.zs;
    for (int i = 0; i < 4; i++) {
        int j = i == 0 ? 1 : 0, k = i <= 1 ? 2 : 1, l = i <= 2 ? 3 : 2;
        double sgn = (i % 2 == 0) ? 1.0 : -1.0;
        ti.a[i] = sgn * tet_det3(xs[j], ys[j], zs[j], xs[k], ys[k], zs[k], xs[l], ys[l], zs[l]);
        ti.b[i] = -sgn * sp_det1(ys[j], zs[j], ys[k], zs[k], ys[l], zs[l]);
        ti.c[i] = sgn * sp_det1(xs[j], zs[j], xs[k], zs[k], xs[l], zs[l]);
        ti.d[i] = -sgn * sp_det1(xs[j], ys[j], xs[k], ys[k], xs[l], ys[l]);
    }
    double V = fabs(tet_det3(xs[1] - xs[0], ys[1] - ys[0], zs[1] - zs[0], xs[2] - xs[0], ys[2] - ys[0], zs[2] - zs[0],
                             xs[3] - xs[0], ys[3] - ys[0], zs[3] - zs[0])) / 6.0;
    ti.V1 = 216.0 * V * V * V;
    for (int i = 0; i < 4; i++) {
        int r = 0;
        for (int j = 0; j < 4; j++) r += vid[j] < vid[i];
        ti.rank[i] = r;
    }
    return true;
}

__device__ __forceinline__ void eval_field(const TetInterp& ti, const double2 dof[20], double px, double py,
                                           double pz, double Er[3], double Ei[3]) {
    const int ep[6] = {0, 0, 0, 1, 3, 2}, eq[6] = {1, 2, 3, 2, 1, 3};
    const int fv[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 2, 3}};
    const double *xs = ti.xs, *ys = ti.ys, *zs = ti.zs, *b = ti.b, *c = ti.c, *d = ti.d;
    const double V1 = ti.V1;
    double Fv[4];
    for (int i = 0; i < 4; i++) Fv[i] = ti.a[i] + b[i] * px + c[i] * py + d[i] * pz;
    for (int q = 0; q < 3; q++) { Er[q] = 0; Ei[q] = 0; }
    for (int e = 0; e < 6; e++) {
        int v1 = ep[e], v2 = eq[e];
        if (ti.rank[v2] < ti.rank[v1]) { int t = v1; v1 = v2; v2 = t; }
        double L = sp_dist(xs, ys, zs, v1, v2);
        double2 m1 = dof[e], m2 = dof[10 + e];
        double wr = m1.x * Fv[v1] + m2.x * Fv[v2], wi = m1.y * Fv[v1] + m2.y * Fv[v2];
        double gg[3] = {b[v1] * Fv[v2] - b[v2] * Fv[v1], c[v1] * Fv[v2] - c[v2] * Fv[v1], d[v1] * Fv[v2] - d[v2] * Fv[v1]};
        for (int q = 0; q < 3; q++) { Er[q] += L * wr * gg[q] / V1; Ei[q] += L * wi * gg[q] / V1; }
    }
    for (int f = 0; f < 4; f++) {
        int v1 = fv[f][0], v2 = fv[f][1], v3 = fv[f][2], t;
        if (ti.rank[v2] < ti.rank[v1]) { t = v1; v1 = v2; v2 = t; }
        if (ti.rank[v3] < ti.rank[v2]) { t = v2; v2 = v3; v3 = t; }
        if (ti.rank[v2] < ti.rank[v1]) { t = v1; v1 = v2; v2 = t; }
        double L1 = sp_dist(xs, ys, zs, v1, v3), L2 = sp_dist(xs, ys, zs, v1, v2);
        double2 m1 = dof[6 + f], m2 = dof[16 + f];
        double q1r = m1.x * L1 * Fv[v2], q1i = m1.y * L1 * Fv[v2];
        double q2r = m2.x * L2 * Fv[v3], q2i = m2.y * L2 * Fv[v3];
        double g13[3] = {b[v1] * Fv[v3] - b[v3] * Fv[v1], c[v1] * Fv[v3] - c[v3] * Fv[v1], d[v1] * Fv[v3] - d[v3] * Fv[v1]};
        double g12[3] = {b[v1] * Fv[v2] - b[v2] * Fv[v1], c[v1] * Fv[v2] - c[v2] * Fv[v1], d[v1] * Fv[v2] - d[v2] * Fv[v1]};
        for (int q = 0; q < 3; q++) {
            Er[q] += (-q1r * g13[q] + q2r * g12[q]) / V1;
            Ei[q] += (-q1i * g13[q] + q2i * g12[q]) / V1;
        }
    }
}

// E . dl at given points inside given tets, for every system: out[p * nsys + s] (lumped-port voltage
// lines, microwave_3d.py:1271-1291; the caller applies the line rule's weights)
__global__ void point_field_dot_kernel(long long nn, const double* __restrict__ nodes, long long nt,
                                       const int64_t* __restrict__ tets, const int64_t* __restrict__ t2f, long long N,
                                       long long npts, const int64_t* __restrict__ pt_tet,
                                       const double* __restrict__ pts, const double* __restrict__ dl, int nsys,
                                       const double2* __restrict__ x, double2* __restrict__ out, int* status) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npts * nsys) return;
    long long p = g / nsys;
    int s = (int)(g % nsys);
    out[g] = make_double2(0, 0);
    long long T = pt_tet[p];
    TetInterp ti;
    if (T < 0 || T >= nt || !load_tet_interp(nn, nodes, nt, tets, T, ti)) { flag(status, DEV_BAD_INDEX); return; }
    double2 dof[20];
    for (int k = 0; k < 20; k++) {
        int64_t id = t2f[k * nt + T];
        if (id < 0 || id >= N) { flag(status, DEV_BAD_INDEX); return; }
        dof[k] = x[id * nsys + s];
    }
    double Er[3], Ei[3];
    eval_field(ti, dof, pts[p], pts[npts + p], pts[2 * npts + p], Er, Ei);
    const double* w = dl + 3 * p;
    out[g] = make_double2(Er[0] * w[0] + Er[1] * w[1] + Er[2] * w[2], Ei[0] * w[0] + Ei[1] * w[1] + Ei[2] * w[2]);
}

__global__ void port_overlap_kernel(long long nn, const double* __restrict__ nodes, long long nt,
                                    const int64_t* __restrict__ tets, const int64_t* __restrict__ t2f, long long N,
                                    long long ntri, const int64_t* __restrict__ tri_tet,
                                    const int64_t* __restrict__ tri_nodes, const double* __restrict__ dpts, int npts,
                                    const double2* __restrict__ shape, const double2* __restrict__ tri_const,
                                    int nsys, const double2* __restrict__ x, double2* __restrict__ F,
                                    double2* __restrict__ Nn, int* status) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntri * nsys) return;
    long long it = g / nsys;
    int s = (int)(g % nsys);
    F[it * nsys + s] = make_double2(0, 0);
    if (s == 0) Nn[it] = make_double2(0, 0);
    long long T = tri_tet[it];
    if (T < 0 || T >= nt) { flag(status, DEV_BAD_INDEX); return; }
    // triangle geometry and quadrature points (generate_int_points_tri, mth/optimized.py:157-182)
    double tx[3], ty[3], tz[3];
    for (int v = 0; v < 3; v++) {
        int64_t id = tri_nodes[v * ntri + it];
        if (id < 0 || id >= nn) { flag(status, DEV_BAD_INDEX); return; }
        tx[v] = nodes[id]; ty[v] = nodes[nn + id]; tz[v] = nodes[2 * nn + id];
    }
    double e1x = tx[1] - tx[0], e1y = ty[1] - ty[0], e1z = tz[1] - tz[0];
    double e2x = tx[2] - tx[0], e2y = ty[2] - ty[0], e2z = tz[2] - tz[0];
    double cxp = e1y * e2z - e1z * e2y, cyp = e1z * e2x - e1x * e2z, czp = e1x * e2y - e1y * e2x;
    double area = sqrt(cxp * cxp + cyp * cyp + czp * czp) / 2;
    // owning tet: interpolation data (tet_coefficients, ned2_interp.py:59-77) and its 20 DOFs
    TetInterp ti;
    if (!load_tet_interp(nn, nodes, nt, tets, T, ti)) { flag(status, DEV_BAD_INDEX); return; }
    double2 dof[20];
    for (int k = 0; k < 20; k++) {
        int64_t id = t2f[k * nt + T];
        if (id < 0 || id >= N) { flag(status, DEV_BAD_INDEX); return; }
        dof[k] = x[id * nsys + s];
    }
    double2 accF = make_double2(0, 0);
    double accN = 0;
    for (int p = 0; p < npts; p++) {
        double px = tx[0] * dpts[npts + p] + tx[1] * dpts[2 * npts + p] + tx[2] * dpts[3 * npts + p];
        double py = ty[0] * dpts[npts + p] + ty[1] * dpts[2 * npts + p] + ty[2] * dpts[3 * npts + p];
        double pz = tz[0] * dpts[npts + p] + tz[1] * dpts[2 * npts + p] + tz[2] * dpts[3 * npts + p];
        double Er[3], Ei[3];
        eval_field(ti, dof, px, py, pz, Er, Ei);
        const double2* m = shape + (long long)(p * ntri + it);  // shape (3, npts, ntri)
        double2 mx = m[0], my = m[(long long)npts * ntri], mz = m[2LL * npts * ntri];
        // E . conj(m)
        double dr = Er[0] * mx.x + Ei[0] * mx.y + Er[1] * my.x + Ei[1] * my.y + Er[2] * mz.x + Ei[2] * mz.y;
        double di = Ei[0] * mx.x - Er[0] * mx.y + Ei[1] * my.x - Er[1] * my.y + Ei[2] * mz.x - Er[2] * mz.y;
        double w = dpts[p];
        accF.x += w * dr;
        accF.y += w * di;
        accN += w * (mx.x * mx.x + mx.y * mx.y + my.x * my.x + my.y * my.y + mz.x * mz.x + mz.y * mz.y);
    }
    double2 cst = tri_const[it];
    F[it * nsys + s] = make_double2((cst.x * accF.x - cst.y * accF.y) * area, (cst.x * accF.y + cst.y * accF.x) * area);
    if (s == 0) Nn[it] = make_double2(cst.x * accN * area, cst.y * accN * area);
}

// triangle sums in triangle order: thread s < nsys sums F[:, s], thread nsys sums N
__global__ void overlap_sum_kernel(long long ntri, int nsys, const double2* __restrict__ F, const double2* __restrict__ Nn,
                                   double2* __restrict__ outF, double2* __restrict__ outN) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > nsys) return;
    double2 acc = make_double2(0, 0);
    if (s == nsys) {
        for (long long t = 0; t < ntri; t++) { acc.x += Nn[t].x; acc.y += Nn[t].y; }
        *outN = acc;
        return;
    }
    for (long long t = 0; t < ntri; t++) { acc.x += F[t * nsys + s].x; acc.y += F[t * nsys + s].y; }
    outF[s] = acc;
}

}  // namespace emfem

using namespace emfem;

extern "C" int emfem_port_overlap(emfem_handle h, int64_t n_nodes, const double* nodes, int64_t n_tets,
                                  const int64_t* tets, const int64_t* tet_to_field, int64_t n_field, int64_t n_tri,
                                  const int64_t* tri_tet, const int64_t* tri_nodes, const double* dpts, int npts,
                                  const void* shape, const void* tri_const, int nsys, const void* x,
                                  void* work, void* overlap, void* mode_norm) {
    EMFEM_REQUIRE(h && nodes && tets && tet_to_field && tri_tet && tri_nodes && dpts && shape && tri_const && x && work &&
                  overlap && mode_norm, "emfem_port_overlap: null argument");
    EMFEM_REQUIRE(n_tri > 0 && nsys > 0 && n_field > 0 && npts > 0 && npts <= SP_MAX_NPTS,
                  "emfem_port_overlap: bad sizes");
    double2* F = (double2*)work;
    double2* Nn = F + n_tri * nsys;
    port_overlap_kernel<<<grid_for(n_tri * nsys, 128), 128, 0, h->h.stream>>>(
        n_nodes, nodes, n_tets, tets, tet_to_field, n_field, n_tri, tri_tet, tri_nodes, dpts, npts,
        (const double2*)shape, (const double2*)tri_const, nsys, (const double2*)x, F, Nn, h->h.dev_status);
    EMFEM_LAUNCH("port_overlap_kernel");
    overlap_sum_kernel<<<grid_for(nsys + 1, 64), 64, 0, h->h.stream>>>(n_tri, nsys, F, Nn, (double2*)overlap,
                                                                        (double2*)mode_norm);
    EMFEM_LAUNCH("overlap_sum_kernel");
    return EMFEM_OK;
}

extern "C" int emfem_point_field_dot(emfem_handle h, int64_t n_nodes, const double* nodes, int64_t n_tets,
                                     const int64_t* tets, const int64_t* tet_to_field, int64_t n_field, int64_t npts,
                                     const int64_t* pt_tet, const double* pts, const double* dl, int nsys,
                                     const void* x, void* out) {
    EMFEM_REQUIRE(h && nodes && tets && tet_to_field && pt_tet && pts && dl && x && out && npts >= 0 && nsys >= 1,
                  "emfem_point_field_dot: bad argument");
    if (npts == 0) return EMFEM_OK;
    point_field_dot_kernel<<<grid_for(npts * nsys, 128), 128, 0, h->h.stream>>>(
        n_nodes, nodes, n_tets, tets, tet_to_field, n_field, npts, pt_tet, pts, dl, nsys, (const double2*)x,
        (double2*)out, h->h.dev_status);
    EMFEM_LAUNCH("point_field_dot_kernel");
    return EMFEM_OK;
}
