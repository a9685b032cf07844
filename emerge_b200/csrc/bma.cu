// Boundary-mode analysis (port-mode) element matrices on the device.
//
// Replaces generalized_matrix_GQ / _matrix_builder
// (src/emerge/_emerge/physics/microwave/assembly/generalized_eigen_hb.py:257-458): for every triangle
// of a port face, the 14x14 complex blocks A and B of the mixed Nedelec-2 (transverse E) /
// Lagrange-2 (E_z) element, DOF order [e1 e2 e3 f | e1' e2' e3' f' | v1 v2 v3 | m1 m2 m3]
// (elements/nedleg2.py:140-150).
//
// Layout: one thread per (triangle, element row); a block holds 16 triangles x 14 rows.  Each
// thread evaluates the 8 transverse basis vectors, their curls and the 6 Lagrange functions with
// gradients at the 6 quadrature points of its triangle and accumulates its row of A and B, so the
// output rows are written once, row-major, exactly like the reference's dataE/dataB slices.
//
// Basis (barycentrics L_i = a_i + b_i x + c_i y in the port's local frame, tri_coefficients :202-226;
// W_ij = L_i grad L_j - L_j grad L_i; (i, j) the local slots of the global edge's nodes):
//   edge:  W_ij, W_ij (L_i - L_j); curls 2 k_ij and grad(L_i - L_j) x W_ij + 2 k_ij (L_i - L_j)
//   face:  L_2 W_13 + L_1 W_23 and -(L_3 W_12 + L_2 W_13) with their curls
//   Lagrange: L(2L - 1), 4 L_i L_j and gradients.
// Blocks: A = [[Att - k0^2 Btt, 0], [0, 0]], B = [[Dtt, Dzt^T], [Dzt, Dzz1 - k0^2 Dzz2]], times the
// area.  As in the reference, face rows of Att/Btt/Dtt take the value of the mirrored face column
// (:375-398), the face-face entries of Dtt stay zero, and no edge-length scaling is applied (:433).
#include "emfem_internal.cuh"
#include "ned2_math.cuh"

using namespace emfem;

namespace {

// 6-point Dunavant rule as the reference tabulates it (8 digits; :232-235): [W, L1, L2, L3]
__constant__ double BMA_DPTS[4][6] = {
    {0.22338159, 0.22338159, 0.22338159, 0.10995174, 0.10995174, 0.10995174},
    {0.10810302, 0.44594849, 0.44594849, 0.81684757, 0.09157621, 0.09157621},
    {0.44594849, 0.44594849, 0.10810302, 0.09157621, 0.09157621, 0.81684757},
    {0.44594849, 0.10810302, 0.44594849, 0.09157621, 0.81684757, 0.09157621}};

constexpr int BMA_NE = 14;
constexpr int BMA_TRIS_PER_BLOCK = 16;

__device__ __forceinline__ bool is_face(int i) { return i == 3 || i == 7; }

// w * (u . (M v)) for real 2-vectors u, v and a complex 2x2 M (row-major m[0..3])
__device__ __forceinline__ cd wdot(double w, const double* u, const cd* m, const double* v) {
    cd mv0 = m[0] * v[0] + m[1] * v[1];
    cd mv1 = m[2] * v[0] + m[3] * v[1];
    return (u[0] * mv0 + u[1] * mv1) * w;
}

// (u * (m v)) * w for real scalars u, v and complex m
__device__ __forceinline__ cd wsdot(double w, double u, cd m, double v) { return (u * (m * v)) * w; }

__global__ void __launch_bounds__(BMA_TRIS_PER_BLOCK * BMA_NE) bma_tri_kernel(
    long long n_nodes, const double* __restrict__ lnodes, long long n_tris, const int64_t* __restrict__ tris,
    long long n_edges, const int64_t* __restrict__ edges, const int64_t* __restrict__ tri_to_edge,
    const double2* __restrict__ er, const double2* __restrict__ ur, double k0, double2* __restrict__ A,
    double2* __restrict__ B, int* status) {
    const int lt = threadIdx.x / BMA_NE, r = threadIdx.x - lt * BMA_NE;
    const long long t = (long long)blockIdx.x * BMA_TRIS_PER_BLOCK + lt;
    if (t >= n_tris) return;

    int64_t v[3];
    double x[3], y[3];
    for (int k = 0; k < 3; k++) {
        v[k] = tris[k * n_tris + t];
        if (v[k] < 0 || v[k] >= n_nodes) { flag(status, DEV_BAD_INDEX); return; }
        x[k] = lnodes[v[k]];
        y[k] = lnodes[n_nodes + v[k]];
    }
    // local slots of each edge's two global nodes (local_tri_to_edgeid :30-33)
    int ei[3], ej[3];
    for (int e = 0; e < 3; e++) {
        int64_t id = tri_to_edge[e * n_tris + t];
        if (id < 0 || id >= n_edges) { flag(status, DEV_BAD_INDEX); return; }
        int64_t n0 = edges[id], n1 = edges[n_edges + id];
        ei[e] = n0 == v[0] ? 0 : n0 == v[1] ? 1 : n0 == v[2] ? 2 : -1;
        ej[e] = n1 == v[0] ? 0 : n1 == v[1] ? 1 : n1 == v[2] ? 2 : -1;
        if (ei[e] < 0 || ej[e] < 0) { flag(status, DEV_BAD_INDEX); return; }
    }
    // tri_coefficients (:202-226), scaled by 1/(2 area)
    double a[3], b[3], c[3];
    a[0] = x[1] * y[2] - y[1] * x[2]; a[1] = x[2] * y[0] - y[2] * x[0]; a[2] = x[0] * y[1] - y[0] * x[1];
    b[0] = y[1] - y[2]; b[1] = y[2] - y[0]; b[2] = y[0] - y[1];
    c[0] = x[2] - x[1]; c[1] = x[0] - x[2]; c[2] = x[1] - x[0];
    const double sA = 0.5 * ((x[0] - x[2]) * (y[1] - y[0]) - (x[0] - x[1]) * (y[2] - y[0]));
    const double area = fabs(sA);
    if (!(area > 0.0)) { flag(status, sA == sA ? DEV_DEGENERATE : DEV_NONFINITE); return; }
    const double sg = sA > 0 ? 1.0 : -1.0;
    for (int i = 0; i < 3; i++) {
        a[i] = a[i] * sg / (2 * area);
        b[i] = b[i] * sg / (2 * area);
        c[i] = c[i] * sg / (2 * area);
    }
    // materials: Mm = er, Ms = ur^-1 (matinv, mth/optimized.py:342-370)
    cd Mm[9], Mu[9], Ms[9];
    for (int k = 0; k < 9; k++) {
        double2 e = er[k * n_tris + t], u = ur[k * n_tris + t];
        Mm[k] = mk(e.x, e.y);
        Mu[k] = mk(u.x, u.y);
    }
    matinv3(Mu, Ms);
    const cd Ms2[4] = {Ms[0], Ms[1], Ms[3], Ms[4]};
    const cd Mm2[4] = {Mm[0], Mm[1], Mm[3], Mm[4]};
    const cd Msz = Ms[8], Mmz = Mm[8];

    cd acc0[8], acc1[8], acc2[8], accz[6], accz2[6];
    for (int j = 0; j < 8; j++) acc0[j] = acc1[j] = acc2[j] = mk(0, 0);
    for (int s = 0; s < 6; s++) accz[s] = accz2[s] = mk(0, 0);

    for (int p = 0; p < 6; p++) {
        const double w = BMA_DPTS[0][p];
        const double xs = x[0] * BMA_DPTS[1][p] + x[1] * BMA_DPTS[2][p] + x[2] * BMA_DPTS[3][p];
        const double ys = y[0] * BMA_DPTS[1][p] + y[1] * BMA_DPTS[2][p] + y[2] * BMA_DPTS[3][p];
        double L[3];
        for (int i = 0; i < 3; i++) L[i] = a[i] + b[i] * xs + c[i] * ys;
        double N[8][2], cu[8], lag[6], gl[6][2];
        for (int e = 0; e < 3; e++) {
            const int i = ei[e], j = ej[e];
            const double Wx = L[i] * b[j] - L[j] * b[i], Wy = L[i] * c[j] - L[j] * c[i];
            const double kk = b[i] * c[j] - b[j] * c[i], dL = L[i] - L[j];
            N[e][0] = Wx; N[e][1] = Wy;
            N[4 + e][0] = Wx * dL; N[4 + e][1] = Wy * dL;
            cu[e] = 2 * kk;
            cu[4 + e] = (b[i] - b[j]) * Wy - (c[i] - c[j]) * Wx + 2 * kk * dL;
            lag[3 + e] = 4 * L[i] * L[j];
            gl[3 + e][0] = 4 * (b[i] * L[j] + b[j] * L[i]);
            gl[3 + e][1] = 4 * (c[i] * L[j] + c[j] * L[i]);
            lag[e] = L[e] * (2 * L[e] - 1);
            gl[e][0] = b[e] * (4 * L[e] - 1);
            gl[e][1] = c[e] * (4 * L[e] - 1);
        }
        {
            const double W13x = L[0] * b[2] - L[2] * b[0], W13y = L[0] * c[2] - L[2] * c[0];
            const double W23x = L[1] * b[2] - L[2] * b[1], W23y = L[1] * c[2] - L[2] * c[1];
            const double W12x = L[0] * b[1] - L[1] * b[0], W12y = L[0] * c[1] - L[1] * c[0];
            const double k13 = b[0] * c[2] - b[2] * c[0], k23 = b[1] * c[2] - b[2] * c[1], k12 = b[0] * c[1] - b[1] * c[0];
            N[3][0] = L[1] * W13x + L[0] * W23x;
            N[3][1] = L[1] * W13y + L[0] * W23y;
            N[7][0] = -(L[2] * W12x + L[1] * W13x);
            N[7][1] = -(L[2] * W12y + L[1] * W13y);
            cu[3] = (b[1] * W13y - c[1] * W13x) + 2 * L[1] * k13 + (b[0] * W23y - c[0] * W23x) + 2 * L[0] * k23;
            cu[7] = -((b[2] * W12y - c[2] * W12x) + 2 * L[2] * k12 + (b[1] * W13y - c[1] * W13x) + 2 * L[1] * k13);
        }
        if (r < 8) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const bool mirror = is_face(r) && !is_face(j);
                const int ii = mirror ? j : r, jj = mirror ? r : j;
                acc0[j] += wsdot(w, cu[ii], Msz, cu[jj]);                // Att
                acc1[j] += wdot(w, N[ii], Mm2, N[jj]);                   // Btt
                if (!(is_face(r) && is_face(j))) acc2[j] += wdot(w, N[ii], Ms2, N[jj]);   // Dtt
            }
#pragma unroll
            for (int s = 0; s < 6; s++) accz[s] += wdot(w, gl[s], Ms2, N[r]);         // Dzt^T
        } else {
            const int s = r - 8;
#pragma unroll
            for (int j = 0; j < 8; j++) acc0[j] += wdot(w, gl[s], Ms2, N[j]);         // Dzt
#pragma unroll
            for (int q = 0; q < 6; q++) {
                accz[q] += wdot(w, gl[s], Ms2, gl[q]);                                  // Dzz1
                accz2[q] += wsdot(w, lag[s], Mmz, lag[q]);                              // Dzz2
            }
        }
    }
    const double kk0 = k0 * k0;
    double2* Ar = A + t * (BMA_NE * BMA_NE) + r * BMA_NE;
    double2* Br = B + t * (BMA_NE * BMA_NE) + r * BMA_NE;
    if (r < 8) {
        for (int j = 0; j < 8; j++) {
            cd va = (acc0[j] - acc1[j] * kk0) * area, vb = acc2[j] * area;
            Ar[j] = make_double2(va.x, va.y);
            Br[j] = make_double2(vb.x, vb.y);
        }
        for (int s = 0; s < 6; s++) {
            cd vb = accz[s] * area;
            Ar[8 + s] = make_double2(0.0, 0.0);
            Br[8 + s] = make_double2(vb.x, vb.y);
        }
    } else {
        for (int j = 0; j < 8; j++) {
            cd vb = acc0[j] * area;
            Ar[j] = make_double2(0.0, 0.0);
            Br[j] = make_double2(vb.x, vb.y);
        }
        for (int q = 0; q < 6; q++) {
            cd vb = (accz[q] - accz2[q] * kk0) * area;
            Ar[8 + q] = make_double2(0.0, 0.0);
            Br[8 + q] = make_double2(vb.x, vb.y);
        }
    }
}

// E (what = 0) or the curl form H / (j / (k0 c0 mu0)) (what = 1) of one port-mode vector at points
// given per triangle: ned2_tri_interp_full (elements/ned2_interp.py:616-685) and
// ned2_tri_interp_curl (:687-760) with the same basis as bma_tri_kernel.  For H:
//   (d_y E_z - j beta E_y, -d_x E_z + j beta E_x, curl_t E_t) times the diagonal of the triangle's
// diadic (ur^-1).  One thread per (point, triangle); pts (2, npts, n_tris) local coordinates of
// points inside their triangle; out (3, npts, n_tris) in the port's local frame.
__global__ void tri_field_kernel(long long n_nodes, const double* __restrict__ lnodes, long long n_tris,
                                 const int64_t* __restrict__ tris, long long n_edges, const int64_t* __restrict__ edges,
                                 const int64_t* __restrict__ tri_to_edge, const int64_t* __restrict__ t2f,
                                 long long n_field, const double2* __restrict__ x, int npts,
                                 const double* __restrict__ pts, int what, double beta_re, double beta_im,
                                 const double2* __restrict__ diadic, double2* __restrict__ out, int* status) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)npts * n_tris) return;
    const long long t = i % n_tris;
    int64_t v[3];
    double xv[3], yv[3];
    for (int k = 0; k < 3; k++) {
        v[k] = tris[k * n_tris + t];
        if (v[k] < 0 || v[k] >= n_nodes) { flag(status, DEV_BAD_INDEX); return; }
        xv[k] = lnodes[v[k]];
        yv[k] = lnodes[n_nodes + v[k]];
    }
    int ei[3], ej[3];
    for (int e = 0; e < 3; e++) {
        int64_t id = tri_to_edge[e * n_tris + t];
        if (id < 0 || id >= n_edges) { flag(status, DEV_BAD_INDEX); return; }
        int64_t n0 = edges[id], n1 = edges[n_edges + id];
        ei[e] = n0 == v[0] ? 0 : n0 == v[1] ? 1 : n0 == v[2] ? 2 : -1;
        ej[e] = n1 == v[0] ? 0 : n1 == v[1] ? 1 : n1 == v[2] ? 2 : -1;
        if (ei[e] < 0 || ej[e] < 0) { flag(status, DEV_BAD_INDEX); return; }
    }
    cd e[BMA_NE];
    for (int k = 0; k < BMA_NE; k++) {
        int64_t id = t2f[k * n_tris + t];
        if (id < 0 || id >= n_field) { flag(status, DEV_BAD_INDEX); return; }
        double2 q = x[id];
        e[k] = mk(q.x, q.y);
    }
    double a[3], b[3], c[3];
    a[0] = xv[1] * yv[2] - yv[1] * xv[2]; a[1] = xv[2] * yv[0] - yv[2] * xv[0]; a[2] = xv[0] * yv[1] - yv[0] * xv[1];
    b[0] = yv[1] - yv[2]; b[1] = yv[2] - yv[0]; b[2] = yv[0] - yv[1];
    c[0] = xv[2] - xv[1]; c[1] = xv[0] - xv[2]; c[2] = xv[1] - xv[0];
    const double sA = 0.5 * ((xv[0] - xv[2]) * (yv[1] - yv[0]) - (xv[0] - xv[1]) * (yv[2] - yv[0]));
    const double area = fabs(sA);
    if (!(area > 0.0)) { flag(status, sA == sA ? DEV_DEGENERATE : DEV_NONFINITE); return; }
    const double sg = sA > 0 ? 1.0 : -1.0;
    for (int k = 0; k < 3; k++) {
        a[k] = a[k] * sg / (2 * area);
        b[k] = b[k] * sg / (2 * area);
        c[k] = c[k] * sg / (2 * area);
    }
    const long long pi = i / n_tris;
    const double px = pts[pi * n_tris + t], py = pts[((long long)npts + pi) * n_tris + t];
    double L[3];
    for (int k = 0; k < 3; k++) L[k] = a[k] + b[k] * px + c[k] * py;
    cd Ex = mk(0, 0), Ey = mk(0, 0), Ez = mk(0, 0), cz = mk(0, 0), gx = mk(0, 0), gy = mk(0, 0);
    for (int k = 0; k < 3; k++) {
        const int p = ei[k], q = ej[k];
        const double Wx = L[p] * b[q] - L[q] * b[p], Wy = L[p] * c[q] - L[q] * c[p];
        const double kk = b[p] * c[q] - b[q] * c[p], dL = L[p] - L[q];
        Ex += e[k] * Wx + e[4 + k] * (Wx * dL);
        Ey += e[k] * Wy + e[4 + k] * (Wy * dL);
        cz += e[k] * (2 * kk) + e[4 + k] * ((b[p] - b[q]) * Wy - (c[p] - c[q]) * Wx + 2 * kk * dL);
        // E_z: vertex k and edge k Lagrange functions
        Ez += e[8 + k] * (L[k] * (2 * L[k] - 1)) + e[11 + k] * (4 * L[p] * L[q]);
        gx += e[8 + k] * (b[k] * (4 * L[k] - 1)) + e[11 + k] * (4 * (b[p] * L[q] + b[q] * L[p]));
        gy += e[8 + k] * (c[k] * (4 * L[k] - 1)) + e[11 + k] * (4 * (c[p] * L[q] + c[q] * L[p]));
    }
    {
        const double W13x = L[0] * b[2] - L[2] * b[0], W13y = L[0] * c[2] - L[2] * c[0];
        const double W23x = L[1] * b[2] - L[2] * b[1], W23y = L[1] * c[2] - L[2] * c[1];
        const double W12x = L[0] * b[1] - L[1] * b[0], W12y = L[0] * c[1] - L[1] * c[0];
        const double k13 = b[0] * c[2] - b[2] * c[0], k23 = b[1] * c[2] - b[2] * c[1], k12 = b[0] * c[1] - b[1] * c[0];
        Ex += e[3] * (L[1] * W13x + L[0] * W23x) + e[7] * (-(L[2] * W12x + L[1] * W13x));
        Ey += e[3] * (L[1] * W13y + L[0] * W23y) + e[7] * (-(L[2] * W12y + L[1] * W13y));
        cz += e[3] * ((b[1] * W13y - c[1] * W13x) + 2 * L[1] * k13 + (b[0] * W23y - c[0] * W23x) + 2 * L[0] * k23);
        cz += e[7] * (-((b[2] * W12y - c[2] * W12x) + 2 * L[2] * k12 + (b[1] * W13y - c[1] * W13x) + 2 * L[1] * k13));
    }
    cd o0, o1, o2;
    if (what == 0) {
        o0 = Ex; o1 = Ey; o2 = Ez;
    } else {
        const cd jb = mk(-beta_im, beta_re);                  // j beta
        o0 = gy - jb * Ey;
        o1 = -gx + jb * Ex;
        o2 = cz;
        if (diadic) {
            double2 d0 = diadic[t], d1 = diadic[n_tris + t], d2 = diadic[2 * n_tris + t];
            o0 = o0 * mk(d0.x, d0.y);
            o1 = o1 * mk(d1.x, d1.y);
            o2 = o2 * mk(d2.x, d2.y);
        }
    }
    const long long plane = (long long)npts * n_tris;
    out[i] = make_double2(o0.x, o0.y);
    out[plane + i] = make_double2(o1.x, o1.y);
    out[2 * plane + i] = make_double2(o2.x, o2.y);
}

}  // namespace

extern "C" int emfem_ned2_bma_tri_matrices(emfem_handle h, int64_t n_nodes, const double* local_nodes,
                                           int64_t n_tris, const int64_t* tris, int64_t n_edges,
                                           const int64_t* edges, const int64_t* tri_to_edge, const void* er,
                                           const void* ur, double k0, void* A, void* B) {
    EMFEM_REQUIRE(h && local_nodes && tris && edges && tri_to_edge && er && ur && A && B && n_nodes > 0 &&
                      n_tris >= 0 && n_edges > 0,
                  "emfem_ned2_bma_tri_matrices: bad argument");
    if (n_tris == 0) return EMFEM_OK;
    const long long blocks = (n_tris + BMA_TRIS_PER_BLOCK - 1) / BMA_TRIS_PER_BLOCK;
    EMFEM_REQUIRE(blocks < (1LL << 31), "emfem_ned2_bma_tri_matrices: too many triangles");
    bma_tri_kernel<<<(unsigned)blocks, BMA_TRIS_PER_BLOCK * BMA_NE, 0, h->h.stream>>>(
        n_nodes, local_nodes, n_tris, tris, n_edges, edges, tri_to_edge, (const double2*)er, (const double2*)ur, k0,
        (double2*)A, (double2*)B, h->h.dev_status);
    EMFEM_LAUNCH("bma_tri_kernel");
    return EMFEM_OK;
}

extern "C" int emfem_ned2_tri_field(emfem_handle h, int64_t n_nodes, const double* local_nodes, int64_t n_tris,
                                    const int64_t* tris, int64_t n_edges, const int64_t* edges,
                                    const int64_t* tri_to_edge, const int64_t* tri_to_field, int64_t n_field,
                                    const void* x, int npts, const double* pts, int what, double beta_re,
                                    double beta_im, const void* diadic, void* out) {
    EMFEM_REQUIRE(h && local_nodes && tris && edges && tri_to_edge && tri_to_field && x && pts && out &&
                      n_nodes > 0 && n_tris >= 0 && n_edges > 0 && n_field > 0 && npts > 0 && (what == 0 || what == 1),
                  "emfem_ned2_tri_field: bad argument");
    if (n_tris == 0) return EMFEM_OK;
    const long long n = (long long)npts * n_tris;
    tri_field_kernel<<<grid_for(n, 128), 128, 0, h->h.stream>>>(
        n_nodes, local_nodes, n_tris, tris, n_edges, edges, tri_to_edge, tri_to_field, n_field, (const double2*)x,
        npts, pts, what, beta_re, beta_im, (const double2*)diadic, (double2*)out, h->h.dev_status);
    EMFEM_LAUNCH("tri_field_kernel");
    return EMFEM_OK;
}
