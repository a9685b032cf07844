// Auxiliary nodal space of the Nedelec-2 field and the learned auxiliary-space preconditioner.
//
// The reference solves every frequency with a direct factorisation (SolverSuperLU,
// src/emerge/_emerge/solver.py:535-572) and has no preconditioner of its own.  Iterative solves of
// K = E - k0^2 B + R stall on the near-kernel of the curl-curl operator: gradient fields, on which
// E vanishes and K = -k0^2 B is small and of the wrong sign.  Block Jacobi cannot see them.  This
// file builds the space of those gradients and a correction through it (Hiptmair-Xu style
// auxiliary-space preconditioning):
//
//   M r = BJ r + G N( D_a^-1 G^T r )
//
// * G (N x N_a) is the exact discrete gradient from the second-order nodal space (one aux node per
//   mesh vertex: hat L_v; one per mesh edge: L_a L_b) into the reference's Nedelec-2 basis
//   (edge functions l L_a W_ab, l L_b W_ab; face functions -l_ac L_b W_ac, l_ab L_c W_ab with
//   W_ij = L_j grad L_i - L_i grad L_j, src/emerge/_emerge/elements/ned2_interp.py:248-295).  Its
//   entries depend only on an entity's sorted node ids and edge lengths, so G is built per entity
//   without touching tets: an edge row has 3 entries (2 vertices + the edge), a face row 6.
// * D_a = diag(G^T K G) per system; N is the identity (aux-space Jacobi) or a learned network: a
//   4-layer message-passing network over the vertex-edge incidence graph of the mesh with 32
//   complex (64 real) channels and real weights, linear in its input, so M is a fixed linear
//   operator per system and BiCGStab's theory holds.  The network's skip term is its input.
//
// Every reduction is a fixed-order gather or a fixed-order sum of per-block partials (no atomics
// on values), so results are reproducible.
#include "emfem_internal.cuh"

#include <mma.h>

#include <utility>
#include <vector>

namespace emfem {

constexpr int AB = 256;
constexpr int NN_C = EMFEM_MPNN_CHANNELS;   // complex channels
constexpr int NN_L = EMFEM_MPNN_LAYERS;

// parameter offsets (float): w_in[2][C], per layer W[2][C][C] then U[2][C][C], w_out[2][C]
__host__ __device__ constexpr int nn_off_win() { return 0; }
__host__ __device__ constexpr int nn_off_W(int l) { return 2 * NN_C + l * 4 * NN_C * NN_C; }
__host__ __device__ constexpr int nn_off_U(int l) { return nn_off_W(l) + 2 * NN_C * NN_C; }
__host__ __device__ constexpr int nn_off_wout() { return 2 * NN_C + NN_L * 4 * NN_C * NN_C; }
__host__ __device__ constexpr int nn_nparams() { return nn_off_wout() + 2 * NN_C; }
static_assert(nn_nparams() == EMFEM_MPNN_NPARAMS, "parameter layout");

// ---- discrete gradient ---------------------------------------------------------------------
// ELL rows of G: gcol[i*6 + k] (aux id or -1), gval[i*6 + k].  Aux ids: vertex v -> v, edge e -> N_n + e.
__global__ void aux_grad_kernel(long long nn, long long ne, long long nf, const int64_t* __restrict__ edges,
                                const int64_t* __restrict__ tris, const int64_t* __restrict__ tri_to_edge,
                                const double* __restrict__ elen, int* __restrict__ gcol, double* __restrict__ gval,
                                int* status) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long H = ne + nf;
    if (q >= H) return;
    int c[2][6];
    double v[2][6];
    for (int k = 0; k < 6; k++) { c[0][k] = c[1][k] = -1; v[0][k] = v[1][k] = 0.0; }
    if (q < ne) {
        long long a = edges[q], b = edges[ne + q];
        double l = elen[q];
        if (a < 0 || a >= nn || b < 0 || b >= nn || !(l > 0)) { flag(status, DEV_BAD_INDEX); return; }
        double il = 1.0 / l;
        // e1 = l L_a W'_ab, e2 = l L_b W'_ab with W'_ab = L_b grad L_a - L_a grad L_b (a < b):
        // grad L_a -> (+1, +1)/l, grad L_b -> (-1, -1)/l, grad (L_a L_b) -> (-1, +1)/l
        c[0][0] = c[1][0] = (int)a; v[0][0] = il;  v[1][0] = il;
        c[0][1] = c[1][1] = (int)b; v[0][1] = -il; v[1][1] = -il;
        c[0][2] = c[1][2] = (int)(nn + q); v[0][2] = -il; v[1][2] = il;
    } else {
        long long t = q - ne;
        long long a = tris[t], b = tris[nf + t], cc = tris[2 * nf + t];
        long long eab = tri_to_edge[t], ebc = tri_to_edge[nf + t], eac = tri_to_edge[2 * nf + t];
        if (a < 0 || a >= nn || b < 0 || b >= nn || cc < 0 || cc >= nn || eab < 0 || eab >= ne || ebc < 0 ||
            ebc >= ne || eac < 0 || eac >= ne) { flag(status, DEV_BAD_INDEX); return; }
        double lab = elen[eab], lac = elen[eac];
        if (!(lab > 0) || !(lac > 0)) { flag(status, DEV_DEGENERATE); return; }
        double iab = 1.0 / lab, iac = 1.0 / lac;
        // f1 = -l_ac L_b W'_ac, f2 = l_ab L_c W'_ab (a < b < c).  With L_c W'_ab = f2/l_ab,
        // L_b W'_ac = -f1/l_ac and L_a W'_bc = -f1/l_ac - f2/l_ab, the face parts of
        // grad L_v = sum_u W'_vu and grad (L_x L_y) = L_x grad L_y + L_y grad L_x are:
        const long long ids[6] = {a, b, cc, nn + eab, nn + eac, nn + ebc};
        const double f1[6] = {-iac, -iac, 2 * iac, -2 * iac, iac, iac};
        const double f2[6] = {iab, -2 * iab, iab, -iab, 2 * iab, -iab};
        for (int k = 0; k < 6; k++) {
            c[0][k] = c[1][k] = (int)ids[k];
            v[0][k] = f1[k];
            v[1][k] = f2[k];
        }
    }
    for (int half = 0; half < 2; half++) {
        long long row = q + half * H;
        for (int k = 0; k < 6; k++) {
            gcol[row * 6 + k] = c[half][k];
            gval[row * 6 + k] = v[half][k];
        }
    }
}

__global__ void ell_count_kernel(long long n, const int* __restrict__ gcol, int* __restrict__ cnt) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 6; k++) {
        int c = gcol[i * 6 + k];
        if (c >= 0) atomicAdd(&cnt[c], 1);
    }
}

__global__ void ell_fill_kernel(long long n, const int* __restrict__ gcol, const double* __restrict__ gval,
                                const int* __restrict__ ptr, int* __restrict__ cur, int* __restrict__ row,
                                double* __restrict__ val) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 6; k++) {
        int c = gcol[i * 6 + k];
        if (c < 0) continue;
        int p = ptr[c] + atomicAdd(&cur[c], 1);
        row[p] = (int)i;
        val[p] = gval[i * 6 + k];
    }
}

// sort each CSR row by column (values travel along): rows are short
__global__ void csr_sort_rows_kernel(long long nr, const int* __restrict__ ptr, int* __restrict__ col,
                                     double* __restrict__ val) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
    int b = ptr[r], e = ptr[r + 1];
    for (int i = b + 1; i < e; i++) {
        int c = col[i];
        double v = val ? val[i] : 0.0;
        int j = i - 1;
        while (j >= b && col[j] > c) { col[j + 1] = col[j]; if (val) val[j + 1] = val[j]; j--; }
        col[j + 1] = c;
        if (val) val[j + 1] = v;
    }
}

// incidence graph: vertex v -> edges containing v (as aux ids), edge e -> its two vertices
__global__ void inc_count_kernel(long long nn, long long ne, const int64_t* __restrict__ edges, int* __restrict__ cnt) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    atomicAdd(&cnt[edges[e]], 1);
    atomicAdd(&cnt[edges[ne + e]], 1);
    cnt[nn + e] = 2;
}

__global__ void inc_fill_kernel(long long nn, long long ne, const int64_t* __restrict__ edges, const int* __restrict__ ptr,
                                int* __restrict__ cur, int* __restrict__ nbr) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    long long a = edges[e], b = edges[ne + e];
    nbr[ptr[a] + atomicAdd(&cur[a], 1)] = (int)(nn + e);
    nbr[ptr[b] + atomicAdd(&cur[b], 1)] = (int)(nn + e);
    nbr[ptr[nn + e]] = (int)a;
    nbr[ptr[nn + e] + 1] = (int)b;
}

__global__ void inv_deg_type_kernel(long long nn, long long na, const int* ptr, float* inv_deg, uint8_t* atype) {
    long long y = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= na) return;
    int d = ptr[y + 1] - ptr[y];
    inv_deg[y] = d > 0 ? 1.0f / (float)d : 0.0f;
    atype[y] = (uint8_t)(y >= nn);
}

// ---- aux operator diagonal and usable-node mask -----------------------------------------------
// d_X[y] = sum_{i, j in supp(y)} G_iy X_ij G_jy for X = E, B (shared CSR pattern) and every Robin
// patch port; amask[y] = 1 iff every DOF of supp(y) is free.  One warp per aux node; the support
// (G^T row y) is sorted, so X_ij's column j is found by binary search.
__device__ __forceinline__ int find_sorted(const int* a, int n, int key) {
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = a[mid];
        if (v == key) return mid;
        if (v < key) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

__global__ void aux_diag_kernel(long long na, const int* __restrict__ gt_ptr, const int* __restrict__ gt_row,
                                const double* __restrict__ gt_val, const int* __restrict__ indptr,
                                const int* __restrict__ indices, const double2* __restrict__ E,
                                const double2* __restrict__ B, const int* __restrict__ patch_of_row,
                                const int* __restrict__ prowptr, const int* __restrict__ pcols,
                                const double2* __restrict__ pvals, const int* __restrict__ pport, int nports,
                                const uint8_t* __restrict__ mask, double2* __restrict__ dE, double2* __restrict__ dB,
                                double2* __restrict__ dR, uint8_t* __restrict__ amask) {
    long long y = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (y >= na) return;
    int b = gt_ptr[y], nsup = gt_ptr[y + 1] - b;
    const int* sup = gt_row + b;
    const double* sval = gt_val + b;
    double er = 0, ei = 0, br = 0, bi = 0;
    double rr[EMFEM_MAX_PORTS], ri[EMFEM_MAX_PORTS];
#pragma unroll
    for (int p = 0; p < EMFEM_MAX_PORTS; p++) rr[p] = ri[p] = 0;
    int ok = 1;
    for (int k = lane; k < nsup; k += 32) {
        int i = sup[k];
        double gi = sval[k];
        if (!mask[i]) ok = 0;
        double ser = 0, sei = 0, sbr = 0, sbi = 0;
        for (int jj = indptr[i]; jj < indptr[i + 1]; jj++) {
            int q = find_sorted(sup, nsup, indices[jj]);
            if (q < 0) continue;
            double gj = sval[q];
            double2 ev = E[jj], bv = B[jj];
            ser += ev.x * gj; sei += ev.y * gj;
            sbr += bv.x * gj; sbi += bv.y * gj;
        }
        er += gi * ser; ei += gi * sei; br += gi * sbr; bi += gi * sbi;
        if (patch_of_row) {
            int pr = patch_of_row[i];
            if (pr >= 0) {
                // a patch row may hold entries of several ports: the port is per entry
                for (int jj = prowptr[pr]; jj < prowptr[pr + 1]; jj++) {
                    int q = find_sorted(sup, nsup, pcols[jj]);
                    if (q < 0) continue;
                    int port = pport[jj];
                    double wr = gi * pvals[jj].x * sval[q], wi = gi * pvals[jj].y * sval[q];
#pragma unroll
                    for (int p = 0; p < EMFEM_MAX_PORTS; p++)
                        if (p == port) { rr[p] += wr; ri[p] += wi; }
                }
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        er += __shfl_down_sync(0xffffffffu, er, off);
        ei += __shfl_down_sync(0xffffffffu, ei, off);
        br += __shfl_down_sync(0xffffffffu, br, off);
        bi += __shfl_down_sync(0xffffffffu, bi, off);
#pragma unroll
        for (int p = 0; p < EMFEM_MAX_PORTS; p++) {
            rr[p] += __shfl_down_sync(0xffffffffu, rr[p], off);
            ri[p] += __shfl_down_sync(0xffffffffu, ri[p], off);
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        dE[y] = make_double2(er, ei);
        dB[y] = make_double2(br, bi);
#pragma unroll
        for (int p = 0; p < EMFEM_MAX_PORTS; p++)
            if (p < nports) dR[(long long)p * na + y] = make_double2(rr[p], ri[p]);
        amask[y] = (uint8_t)(ok && nsup > 0);
    }
}

// ---- kernels used inside the Krylov iterations and by training ------------------------------
// dinv[y][s] = amask ? 1 / (dE - k0_s^2 dB + sum_p gamma_{s,p} dR_p) : 0; in a grouped solve column s
// of aux node y is system agroup[y] * S + s of k0sq and gamma
template <typename T>
__global__ void aux_dinv_kernel(long long na, int S, int nsys, const uint8_t* __restrict__ amask,
                                const double2* __restrict__ dE, const double2* __restrict__ dB,
                                const double2* __restrict__ dR, int nports, const double* __restrict__ k0sq,
                                const double* __restrict__ gamma, T* __restrict__ dinv,
                                const int* __restrict__ agroup = nullptr) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= na * S) return;
    long long y = g / S;
    int s = (int)(g % S);
    double dr = 0, di = 0;
    if (s < nsys && amask[y]) {
        const int sy = agroup ? agroup[y] * S + s : s;
        double k2 = k0sq[sy];
        dr = dE[y].x - k2 * dB[y].x;
        di = dE[y].y - k2 * dB[y].y;
        for (int p = 0; p < nports; p++) {
            double gr = gamma[2 * (sy * nports + p)], gi = gamma[2 * (sy * nports + p) + 1];
            double2 r = dR[(long long)p * na + y];
            dr += gr * r.x - gi * r.y;
            di += gr * r.y + gi * r.x;
        }
    }
    double m2 = dr * dr + di * di;
    T o;
    if (m2 > 0) { o.x = dr / m2; o.y = -di / m2; } else { o.x = 0; o.y = 0; }
    dinv[g] = o;
}

// x[y][s] = dinv[y][s] * sum_i G_iy v[i][s]   (dinv null: no scaling)
template <typename TV, typename TX>
__global__ void aux_restrict_kernel(long long na, int S, const int* __restrict__ gt_ptr, const int* __restrict__ gt_row,
                                    const double* __restrict__ gt_val, const TX* __restrict__ dinv,
                                    const TV* __restrict__ v, TX* __restrict__ x) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= na * S) return;
    long long y = g / S;
    int s = (int)(g % S);
    double ar = 0, ai = 0;
    int k = gt_ptr[y], ke = gt_ptr[y + 1];
    for (; k + 4 <= ke; k += 4) {        // loads of four entries in flight, summed in order
        int rr[4];
        double gv[4];
        TV vv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) { rr[u] = gt_row[k + u]; gv[u] = gt_val[k + u]; }
#pragma unroll
        for (int u = 0; u < 4; u++) vv[u] = v[(long long)rr[u] * S + s];
#pragma unroll
        for (int u = 0; u < 4; u++) { ar += gv[u] * (double)vv[u].x; ai += gv[u] * (double)vv[u].y; }
    }
    for (; k < ke; k++) {
        double gv = gt_val[k];
        TV vv = v[(long long)gt_row[k] * S + s];
        ar += gv * (double)vv.x;
        ai += gv * (double)vv.y;
    }
    TX o;
    if (dinv) {
        TX d = dinv[g];
        o.x = ar * (double)d.x - ai * (double)d.y;
        o.y = ar * (double)d.y + ai * (double)d.x;
    } else {
        o.x = ar; o.y = ai;
    }
    x[g] = o;
}

// z[i][s] (+)= sum_k G_i,k za[col_k][s] on free rows (mask null: all rows)
template <typename TZ, typename TA>
__global__ void aux_prolong_kernel(long long n, int S, const int* __restrict__ gcol, const double* __restrict__ gval,
                                   const TA* __restrict__ za, const uint8_t* __restrict__ mask, TZ* __restrict__ z,
                                   int accumulate) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * S) return;
    long long i = g / S;
    int s = (int)(g % S);
    double ar = 0, ai = 0;
    if (!mask || mask[i]) {
        for (int k = 0; k < 6; k++) {
            int c = gcol[i * 6 + k];
            if (c < 0) continue;
            TA a = za[(long long)c * S + s];
            double gv = gval[i * 6 + k];
            ar += gv * (double)a.x;
            ai += gv * (double)a.y;
        }
    }
    TZ o;
    if (accumulate) { o = z[g]; o.x += ar; o.y += ai; } else { o.x = ar; o.y = ai; }
    z[g] = o;
}

// ---- network forward ------------------------------------------------------------------------
// One warp per (aux node y, system s); lane c holds channel c.  Layer l (0-based):
//   in_y   = l == 0 ? x_y w_in[t_y] : H_l[y]            (complex channels, real weights)
//   m_y    = inv_deg_y * sum_{j in N(y)} in_j
//   out_y  = in_y W_l[t_y] + m_y U_l[t_y]               (t = type: 0 vertex, 1 edge)
// Layer 0 recomputes in_j = x_j w_in[t_j] on the fly.  The last layer optionally writes
// za_y = x_y + sum_c out_y[c] w_out[t_y][c].
template <typename TX>
__global__ void __launch_bounds__(AB) mpnn_layer_kernel(long long na, int S, int layer, const float* __restrict__ P,
                                                        const int* __restrict__ nptr, const int* __restrict__ nbr,
                                                        const float* __restrict__ inv_deg, const uint8_t* __restrict__ atype,
                                                        const TX* __restrict__ x, const float2* __restrict__ Hin,
                                                        float2* __restrict__ Hout, TX* __restrict__ za) {
    __shared__ float sW[2][NN_C][NN_C + 1], sU[2][NN_C][NN_C + 1];
    __shared__ float sWin[2][NN_C], sWout[2][NN_C];
    for (int k = threadIdx.x; k < 2 * NN_C * NN_C; k += blockDim.x) {
        int t = k / (NN_C * NN_C), r = (k / NN_C) % NN_C, c = k % NN_C;
        sW[t][r][c] = P[nn_off_W(layer) + k];
        sU[t][r][c] = P[nn_off_U(layer) + k];
    }
    for (int k = threadIdx.x; k < 2 * NN_C; k += blockDim.x) {
        sWin[k / NN_C][k % NN_C] = P[nn_off_win() + k];
        sWout[k / NN_C][k % NN_C] = P[nn_off_wout() + k];
    }
    __syncthreads();
    int lane = threadIdx.x & 31;
    long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < na * S; w += nw) {
    long long y = w / S;
    int s = (int)(w % S);
    int t = atype[y];
    float2 in, m = make_float2(0.f, 0.f);
    if (layer == 0) {
        TX xv = x[w];
        in = make_float2((float)xv.x * sWin[t][lane], (float)xv.y * sWin[t][lane]);
        for (int k = nptr[y]; k < nptr[y + 1]; k++) {
            long long j = nbr[k];
            TX xj = x[j * S + s];
            float wj = sWin[atype[j]][lane];
            m.x += (float)xj.x * wj;
            m.y += (float)xj.y * wj;
        }
    } else {
        in = Hin[w * NN_C + lane];
        for (int k = nptr[y]; k < nptr[y + 1]; k++) {
            float2 hj = Hin[((long long)nbr[k] * S + s) * NN_C + lane];
            m.x += hj.x;
            m.y += hj.y;
        }
    }
    float idg = inv_deg[y];
    m.x *= idg; m.y *= idg;
    float2 o = make_float2(0.f, 0.f);
#pragma unroll 8
    for (int k = 0; k < NN_C; k++) {
        float ix = __shfl_sync(0xffffffffu, in.x, k), iy = __shfl_sync(0xffffffffu, in.y, k);
        float mx = __shfl_sync(0xffffffffu, m.x, k), my = __shfl_sync(0xffffffffu, m.y, k);
        float wv = sW[t][k][lane], uv = sU[t][k][lane];
        o.x += ix * wv + mx * uv;
        o.y += iy * wv + my * uv;
    }
    if (Hout) Hout[w * NN_C + lane] = o;
    if (za) {
        float zr = o.x * sWout[t][lane], zi = o.y * sWout[t][lane];
        for (int off = 16; off > 0; off >>= 1) {
            zr += __shfl_down_sync(0xffffffffu, zr, off);
            zi += __shfl_down_sync(0xffffffffu, zi, off);
        }
        if (lane == 0) {
            TX xv = x[w], r;
            r.x = xv.x + zr;
            r.y = xv.y + zi;
            za[w] = r;
        }
    }
    }
}

// persistent grid for the warp-per-row network kernels: the weights are staged once per block
static unsigned warp_grid(long long rows) {
    long long blocks = (rows + (AB / 32) - 1) / (AB / 32);
    long long cap = 148LL * 8;
    return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

// Tensor-core layer for inference inside the solve (TF32 inputs, FP32 accumulation, via wmma).
// A warp takes 8 rows (y, s) at a time.  It gathers in_y and m_y into shared memory with lanes over
// channels (coalesced), as 16 matrix rows (re and im of each row) x 32 channels.  It multiplies them
// by W_l[t] and U_l[t] for both node types on the tensor cores, then writes each row's result for its
// own type, lanes over channels again.  Real weights act on the re and im rows alike, so this is the
// same complex-linear layer as mpnn_layer_kernel, rounded to TF32 on input.
constexpr int TC_LD = 40;                // padded row stride (floats) of the shared tiles
constexpr int TC_WARPS = 4;

template <typename TX>
__global__ void __launch_bounds__(TC_WARPS * 32) mpnn_layer_tc_kernel(
    long long na, int S, int layer, const float* __restrict__ P, const int* __restrict__ nptr,
    const int* __restrict__ nbr, const float* __restrict__ inv_deg, const uint8_t* __restrict__ atype,
    const TX* __restrict__ x, const float2* __restrict__ Hin, float2* __restrict__ Hout, TX* __restrict__ za) {
    using namespace nvcuda;
    __shared__ __align__(32) float sWU[4][NN_C * TC_LD];          // W0, W1, U0, U1 as [k][c]
    __shared__ __align__(32) float sA[TC_WARPS][16 * TC_LD], sM[TC_WARPS][16 * TC_LD];
    __shared__ float sWin[2][NN_C], sWout[2][NN_C];
    for (int i = threadIdx.x; i < 4 * NN_C * NN_C; i += blockDim.x) {
        int m = i / (NN_C * NN_C), r = i % (NN_C * NN_C), k = r / NN_C, c = r % NN_C;
        int t = m & 1, isU = m >> 1;
        float v = P[(isU ? nn_off_U(layer) : nn_off_W(layer)) + t * NN_C * NN_C + r];
        sWU[m][k * TC_LD + c] = wmma::__float_to_tf32(v);
    }
    for (int k = threadIdx.x; k < 2 * NN_C; k += blockDim.x) {
        sWin[k / NN_C][k % NN_C] = P[nn_off_win() + k];
        sWout[k / NN_C][k % NN_C] = P[nn_off_wout() + k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    float* A = sA[wl];
    float* M = sM[wl];
    const long long total = na * S;
    const long long ntiles = (total + 7) / 8;
    // S a multiple of 8: the 8 rows of a tile are systems s0..s0+7 of one node y, so the neighbour
    // list is read once and each neighbour's 8 rows are loaded together (8 loads in flight instead
    // of one dependent index-then-row chain per row).  Each row still sums its neighbours in list
    // order, so the result is the same as the row-by-row gather below.
    const bool same_node = (S & 7) == 0;
    for (long long tile = (long long)blockIdx.x * TC_WARPS + wl; tile < ntiles; tile += (long long)gridDim.x * TC_WARPS) {
        const long long w0 = tile * 8;
        bool has[2] = {false, false};
        if (same_node) {
            const long long y = w0 / S;
            const int t = atype[y], k0 = nptr[y], k1 = nptr[y + 1];
            has[t] = true;
            float2 in[8], m[8];
            if (layer == 0) {
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    TX xv = x[w0 + r];
                    in[r] = make_float2((float)xv.x * sWin[t][lane], (float)xv.y * sWin[t][lane]);
                    m[r] = make_float2(0.f, 0.f);
                }
                for (int k = k0; k < k1; k++) {
                    const long long j = nbr[k];
                    const float wj = sWin[atype[j]][lane];
                    const TX* xj = x + j * S + (w0 - y * S);
                    TX v[8];
#pragma unroll
                    for (int r = 0; r < 8; r++) v[r] = xj[r];
#pragma unroll
                    for (int r = 0; r < 8; r++) {
                        m[r].x += (float)v[r].x * wj;
                        m[r].y += (float)v[r].y * wj;
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    in[r] = Hin[(w0 + r) * NN_C + lane];
                    m[r] = make_float2(0.f, 0.f);
                }
                for (int k = k0; k < k1; k++) {
                    const float2* hj = Hin + ((long long)nbr[k] * S + (w0 - y * S)) * NN_C + lane;
                    float2 v[8];
#pragma unroll
                    for (int r = 0; r < 8; r++) v[r] = hj[r * NN_C];
#pragma unroll
                    for (int r = 0; r < 8; r++) {
                        m[r].x += v[r].x;
                        m[r].y += v[r].y;
                    }
                }
            }
            const float idg = inv_deg[y];
#pragma unroll
            for (int r = 0; r < 8; r++) {
                A[(2 * r) * TC_LD + lane] = wmma::__float_to_tf32(in[r].x);
                A[(2 * r + 1) * TC_LD + lane] = wmma::__float_to_tf32(in[r].y);
                M[(2 * r) * TC_LD + lane] = wmma::__float_to_tf32(m[r].x * idg);
                M[(2 * r + 1) * TC_LD + lane] = wmma::__float_to_tf32(m[r].y * idg);
            }
        } else
        for (int r = 0; r < 8; r++) {
            long long w = w0 + r;
            float2 in = make_float2(0.f, 0.f), m = make_float2(0.f, 0.f);
            if (w < total) {
                long long y = w / S;
                int s = (int)(w % S), t = atype[y];
                has[t] = true;
                if (layer == 0) {
                    TX xv = x[w];
                    in = make_float2((float)xv.x * sWin[t][lane], (float)xv.y * sWin[t][lane]);
                    for (int k = nptr[y]; k < nptr[y + 1]; k++) {
                        long long j = nbr[k];
                        TX xj = x[j * S + s];
                        float wj = sWin[atype[j]][lane];
                        m.x += (float)xj.x * wj;
                        m.y += (float)xj.y * wj;
                    }
                } else {
                    in = Hin[w * NN_C + lane];
                    for (int k = nptr[y]; k < nptr[y + 1]; k++) {
                        float2 hj = Hin[((long long)nbr[k] * S + s) * NN_C + lane];
                        m.x += hj.x;
                        m.y += hj.y;
                    }
                }
                float idg = inv_deg[y];
                m.x *= idg; m.y *= idg;
            }
            A[(2 * r) * TC_LD + lane] = wmma::__float_to_tf32(in.x);
            A[(2 * r + 1) * TC_LD + lane] = wmma::__float_to_tf32(in.y);
            M[(2 * r) * TC_LD + lane] = wmma::__float_to_tf32(m.x);
            M[(2 * r + 1) * TC_LD + lane] = wmma::__float_to_tf32(m.y);
        }
        __syncwarp();
        wmma::fragment<wmma::accumulator, 16, 16, 8, float> acc[2][2];
        for (int t = 0; t < 2; t++)
            for (int n = 0; n < 2; n++) wmma::fill_fragment(acc[t][n], 0.0f);
        for (int kk = 0; kk < NN_C; kk += 8) {
            wmma::fragment<wmma::matrix_a, 16, 16, 8, wmma::precision::tf32, wmma::row_major> fa, fm;
            wmma::load_matrix_sync(fa, A + kk, TC_LD);
            wmma::load_matrix_sync(fm, M + kk, TC_LD);
            for (int t = 0; t < 2; t++) {
                if (!__any_sync(0xffffffffu, has[t])) continue;
                for (int n = 0; n < 2; n++) {
                    wmma::fragment<wmma::matrix_b, 16, 16, 8, wmma::precision::tf32, wmma::row_major> fw, fu;
                    wmma::load_matrix_sync(fw, sWU[t] + kk * TC_LD + 16 * n, TC_LD);
                    wmma::load_matrix_sync(fu, sWU[2 + t] + kk * TC_LD + 16 * n, TC_LD);
                    wmma::mma_sync(acc[t][n], fa, fw, acc[t][n]);
                    wmma::mma_sync(acc[t][n], fm, fu, acc[t][n]);
                }
            }
        }
        __syncwarp();
        // type-0 results into A, type-1 results into M (the inputs are consumed)
        for (int n = 0; n < 2; n++) {
            wmma::store_matrix_sync(A + 16 * n, acc[0][n], TC_LD, wmma::mem_row_major);
            wmma::store_matrix_sync(M + 16 * n, acc[1][n], TC_LD, wmma::mem_row_major);
        }
        __syncwarp();
        for (int r = 0; r < 8; r++) {
            long long w = w0 + r;
            if (w >= total) break;
            int t = atype[w / S];
            const float* src = t ? M : A;
            float2 o = make_float2(src[(2 * r) * TC_LD + lane], src[(2 * r + 1) * TC_LD + lane]);
            if (Hout) Hout[w * NN_C + lane] = o;
            if (za) {
                float zr = o.x * sWout[t][lane], zi = o.y * sWout[t][lane];
                for (int off = 16; off > 0; off >>= 1) {
                    zr += __shfl_down_sync(0xffffffffu, zr, off);
                    zi += __shfl_down_sync(0xffffffffu, zi, off);
                }
                if (lane == 0) {
                    TX xv = x[w], rr;
                    rr.x = xv.x + zr;
                    rr.y = xv.y + zi;
                    za[w] = rr;
                }
            }
        }
        __syncwarp();
    }
}

template <typename TX>
int mpnn_forward_tc(const emfem_aux_s* a, int S, const float* P, const TX* x, float2* H0, float2* H1, TX* za,
                    cudaStream_t s) {
    long long na = a->na;
    long long tiles = (na * S + 7) / 8;
    long long blocks = (tiles + TC_WARPS - 1) / TC_WARPS;
    unsigned grid = (unsigned)(blocks < 148LL * 16 ? (blocks > 0 ? blocks : 1) : 148LL * 16);
    const float2* hin = nullptr;
    for (int l = 0; l < NN_L; l++) {
        float2* hout = (l % 2 == 0) ? H0 : H1;
        bool last = l == NN_L - 1;
        mpnn_layer_tc_kernel<TX><<<grid, TC_WARPS * 32, 0, s>>>(na, S, l, P, a->inc_ptr, a->inc, a->inv_deg,
                                                                a->atype, x, hin, last ? nullptr : hout,
                                                                last ? za : nullptr);
        hin = hout;
    }
    return check_cuda(cudaGetLastError(), "mpnn_layer_tc_kernel");
}

// Hstore non-null: every layer's output is kept (training); else layers alternate H0/H1 and the
// last layer writes only za.
template <typename TX>
int mpnn_forward(const emfem_aux_s* a, int S, const float* P, const TX* x, float2* H0, float2* H1, float2* Hstore,
                 TX* za, cudaStream_t s) {
    long long na = a->na;
    unsigned grid = warp_grid(na * S);
    const float2* hin = nullptr;
    for (int l = 0; l < NN_L; l++) {
        float2* hout = Hstore ? Hstore + (size_t)l * na * S * NN_C : ((l % 2 == 0) ? H0 : H1);
        bool last = l == NN_L - 1;
        mpnn_layer_kernel<TX><<<grid, AB, 0, s>>>(na, S, l, P, a->inc_ptr, a->inc, a->inv_deg, a->atype, x, hin,
                                                  (last && !Hstore) ? nullptr : hout, last ? za : nullptr);
        hin = hout;
    }
    return check_cuda(cudaGetLastError(), "mpnn_layer_kernel");
}

// ---- network backward ------------------------------------------------------------------------
// With d = dL/dRe + i dL/dIm for every complex quantity and real weights, per layer in reverse:
//   dW[t][k][c] += Re(conj(in_y[k]) dOut_y[c]),  dU[t][k][c] += Re(conj(m_y[k]) dOut_y[c])
//   dIn_y[k]     = sum_c W[t_y][k][c] dOut_y[c] + sum_{j in N(y)} inv_deg_j sum_c U[t_j][k][c] dOut_j[c]
// (the incidence graph is symmetric); the last layer's dOut = w_out[t] dza, and the first layer's
// dIn gives dw_in.  Weight gradients: each of WG_BLOCKS blocks sums a fixed contiguous range of
// rows into one partial row, then the partial rows are added in block order.
constexpr int WG_BLOCKS = 296;

__global__ void __launch_bounds__(AB) mpnn_bwd_dm_kernel(long long na, int S, int layer, const float* __restrict__ P,
                                                         const float* __restrict__ inv_deg,
                                                         const uint8_t* __restrict__ atype,
                                                         const float2* __restrict__ dOut, float2* __restrict__ dM) {
    __shared__ float sU[2][NN_C][NN_C + 1];
    for (int k = threadIdx.x; k < 2 * NN_C * NN_C; k += blockDim.x) {
        int t = k / (NN_C * NN_C), r = (k / NN_C) % NN_C, c = k % NN_C;
        sU[t][r][c] = P[nn_off_U(layer) + k];
    }
    __syncthreads();
    int lane = threadIdx.x & 31;
    long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < na * S; w += nw) {
        long long y = w / S;
        int t = atype[y];
        float2 d = dOut[w * NN_C + lane];
        float2 o = make_float2(0.f, 0.f);
#pragma unroll 8
        for (int c = 0; c < NN_C; c++) {
            float dx = __shfl_sync(0xffffffffu, d.x, c), dy = __shfl_sync(0xffffffffu, d.y, c);
            float u = sU[t][lane][c];
            o.x += u * dx;
            o.y += u * dy;
        }
        float idg = inv_deg[y];
        dM[w * NN_C + lane] = make_float2(o.x * idg, o.y * idg);
    }
}

__global__ void __launch_bounds__(AB) mpnn_bwd_din_kernel(long long na, int S, int layer, const float* __restrict__ P,
                                                          const int* __restrict__ nptr, const int* __restrict__ nbr,
                                                          const uint8_t* __restrict__ atype,
                                                          const float2* __restrict__ dOut, const float2* __restrict__ dM,
                                                          float2* __restrict__ dIn) {
    __shared__ float sW[2][NN_C][NN_C + 1];
    for (int k = threadIdx.x; k < 2 * NN_C * NN_C; k += blockDim.x) {
        int t = k / (NN_C * NN_C), r = (k / NN_C) % NN_C, c = k % NN_C;
        sW[t][r][c] = P[nn_off_W(layer) + k];
    }
    __syncthreads();
    int lane = threadIdx.x & 31;
    long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < na * S; w += nw) {
        long long y = w / S;
        int s = (int)(w % S);
        int t = atype[y];
        float2 d = dOut[w * NN_C + lane];
        float2 o = make_float2(0.f, 0.f);
#pragma unroll 8
        for (int c = 0; c < NN_C; c++) {
            float dx = __shfl_sync(0xffffffffu, d.x, c), dy = __shfl_sync(0xffffffffu, d.y, c);
            float wv = sW[t][lane][c];
            o.x += wv * dx;
            o.y += wv * dy;
        }
        for (int k = nptr[y]; k < nptr[y + 1]; k++) {
            float2 m = dM[((long long)nbr[k] * S + s) * NN_C + lane];
            o.x += m.x;
            o.y += m.y;
        }
        dIn[w * NN_C + lane] = o;
    }
}

template <typename TX>
__device__ __forceinline__ float2 layer_in(int layer, const float* sWin, const uint8_t* atype, const TX* x,
                                           const float2* Hin, long long j, int S, int s, int k) {
    if (layer == 0) {
        TX xv = x[j * S + s];
        float w = sWin[atype[j] * NN_C + k];
        return make_float2((float)xv.x * w, (float)xv.y * w);
    }
    return Hin[(j * S + s) * NN_C + k];
}

// partial row per block: [2 types][2 mats (W, U)][C][C]
template <typename TX>
__global__ void __launch_bounds__(AB) mpnn_bwd_wgrad_kernel(long long na, int S, int layer, const float* __restrict__ P,
                                                            const int* __restrict__ nptr, const int* __restrict__ nbr,
                                                            const float* __restrict__ inv_deg,
                                                            const uint8_t* __restrict__ atype, const TX* __restrict__ x,
                                                            const float2* __restrict__ Hin,
                                                            const float2* __restrict__ dOut, float* __restrict__ partial) {
    __shared__ float sWin[2 * NN_C];
    __shared__ float2 sIn[8][NN_C], sM[8][NN_C], sD[8][NN_C];
    __shared__ int sT[8];
    for (int k = threadIdx.x; k < 2 * NN_C; k += blockDim.x) sWin[k] = P[nn_off_win() + k];
    // thread owns outputs (k = tid / 8, c = 4 (tid % 8) .. +3) for both types and both matrices
    int kk = threadIdx.x >> 3, c0 = (threadIdx.x & 7) * 4;
    float accW[2][4], accU[2][4];
    for (int t = 0; t < 2; t++)
        for (int q = 0; q < 4; q++) accW[t][q] = accU[t][q] = 0.f;
    long long rows = na * S;
    long long per = (rows + gridDim.x - 1) / gridDim.x;
    long long r0 = blockIdx.x * per, r1 = min(rows, r0 + per);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    for (long long base = r0; base < r1; base += 8) {
        long long w = base + warp;
        if (w < r1) {
            long long y = w / S;
            int s = (int)(w % S);
            float2 in = layer_in<TX>(layer, sWin, atype, x, Hin, y, S, s, lane);
            float2 m = make_float2(0.f, 0.f);
            for (int k = nptr[y]; k < nptr[y + 1]; k++) {
                float2 v = layer_in<TX>(layer, sWin, atype, x, Hin, nbr[k], S, s, lane);
                m.x += v.x; m.y += v.y;
            }
            float idg = inv_deg[y];
            sIn[warp][lane] = in;
            sM[warp][lane] = make_float2(m.x * idg, m.y * idg);
            sD[warp][lane] = dOut[w * NN_C + lane];
            if (lane == 0) sT[warp] = atype[y];
        } else {
            sIn[warp][lane] = make_float2(0.f, 0.f);
            sM[warp][lane] = make_float2(0.f, 0.f);
            sD[warp][lane] = make_float2(0.f, 0.f);
            if (lane == 0) sT[warp] = 0;
        }
        __syncthreads();
        for (int r = 0; r < 8; r++) {
            int t = sT[r];
            float2 iv = sIn[r][kk], mv = sM[r][kk];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float2 d = sD[r][c0 + q];
                float gw = iv.x * d.x + iv.y * d.y, gu = mv.x * d.x + mv.y * d.y;
                if (t == 0) { accW[0][q] += gw; accU[0][q] += gu; }
                else { accW[1][q] += gw; accU[1][q] += gu; }
            }
        }
        __syncthreads();
    }
    float* out = partial + (long long)blockIdx.x * 4 * NN_C * NN_C;
    for (int t = 0; t < 2; t++)
        for (int q = 0; q < 4; q++) {
            out[(t * 2 + 0) * NN_C * NN_C + kk * NN_C + c0 + q] = accW[t][q];
            out[(t * 2 + 1) * NN_C * NN_C + kk * NN_C + c0 + q] = accU[t][q];
        }
}

// dw_in[t][c] = sum Re(conj(x_y) dIn0_y[c]), dw_out[t][c] = sum Re(conj(out_L,y[c]) dza_y) over y of
// type t; partial row per block: [win t0 | win t1 | wout t0 | wout t1] (4 C)
template <typename TX>
__global__ void __launch_bounds__(AB) mpnn_bwd_vec_kernel(long long na, int S, const uint8_t* __restrict__ atype,
                                                          const TX* __restrict__ x, const float2* __restrict__ dIn0,
                                                          const float2* __restrict__ outL, const TX* __restrict__ dza,
                                                          float* __restrict__ partial) {
    __shared__ float red[AB / 32][4 * NN_C];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    long long rows = na * S;
    long long per = (rows + gridDim.x - 1) / gridDim.x;
    long long r0 = blockIdx.x * per, r1 = min(rows, r0 + per);
    for (long long w = r0 + warp; w < r1; w += AB / 32) {
        long long y = w / S;
        int t = atype[y];
        TX xv = x[w];
        float2 di = dIn0[w * NN_C + lane];
        TX dz = dza[w];
        float2 o = outL[w * NN_C + lane];
        acc[t] += (float)xv.x * di.x + (float)xv.y * di.y;
        acc[2 + t] += o.x * (float)dz.x + o.y * (float)dz.y;
    }
    for (int q = 0; q < 4; q++) red[warp][q * NN_C + lane] = acc[q];
    __syncthreads();
    if (warp == 0) {
        for (int q = 0; q < 4; q++) {
            float v = 0.f;
            for (int r = 0; r < AB / 32; r++) v += red[r][q * NN_C + lane];
            partial[(long long)blockIdx.x * 4 * NN_C + q * NN_C + lane] = v;
        }
    }
}

// out[c] = sum_r partial[r * stride + c] for c < count, rows added in order
__global__ void partial_sum_kernel(int nrows, int stride, int count, const float* __restrict__ partial,
                                   float* __restrict__ out) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    float v = 0.f;
    for (int r = 0; r < nrows; r++) v += partial[(long long)r * stride + c];
    out[c] = v;
}

template <typename TX>
__global__ void mpnn_bwd_out_kernel(long long na, int S, const float* __restrict__ P, const uint8_t* __restrict__ atype,
                                    const TX* __restrict__ dza, float2* __restrict__ dOut) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= na * S * NN_C) return;
    long long w = g / NN_C;
    int c = (int)(g % NN_C);
    long long y = w / S;
    float wo = P[nn_off_wout() + atype[y] * NN_C + c];
    TX d = dza[w];
    dOut[g] = make_float2(wo * (float)d.x, wo * (float)d.y);
}

__global__ void adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            float wd) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i] + wd * p[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---- Krylov-side entry points (sweep_solve.cu) -----------------------------------------------
// kbuf layout for S systems (byte offsets, sized for FP64 so FP32 solves fit too):
// ra [0, vb), za [vb, 2 vb), dinv [2 vb, 3 vb), then H0 and H1 (na S C float2 each)
size_t aux_solve_bytes(const emfem_aux_s* a, int S) {
    return (size_t)a->na * S * (3 * sizeof(double2) + 2 * NN_C * sizeof(float2));
}

void* aux_dinv_buffer(const emfem_aux_s* a, int S) {
    return (char*)a->kbuf + 2 * (size_t)a->na * S * sizeof(double2);
}

// z += G N(dinv . G^T v) on free rows (N = identity or the network)
template <typename T>
int aux_correct(const emfem_aux_s* a, int S, bool learned, const T* dinv, const T* v, const uint8_t* mask, T* z,
                cudaStream_t s) {
    char* base = (char*)a->kbuf;
    size_t vb = (size_t)a->na * S * sizeof(double2);
    T* ra = (T*)base;
    T* za = (T*)(base + vb);
    float2* H0 = (float2*)(base + 3 * vb);
    float2* H1 = H0 + (size_t)a->na * S * NN_C;
    aux_restrict_kernel<T, T><<<grid_for(a->na * S, AB), AB, 0, s>>>(a->na, S, a->gt_ptr, a->gt_row, a->gt_val, dinv,
                                                                     v, ra);
    const T* zsrc = ra;
    if (learned) {
        EMFEM_TRY(mpnn_forward_tc<T>(a, S, a->params, ra, H0, H1, za, s));
        zsrc = za;
    }
    aux_prolong_kernel<T, T><<<grid_for(a->n * S, AB), AB, 0, s>>>(a->n, S, a->gcol, a->gval, zsrc, mask, z, 1);
    return check_cuda(cudaGetLastError(), "aux_correct");
}

template <typename T>
int aux_setup_dinv(const emfem_aux_s* a, int S, int nsys, const double* k0sq, const double* gamma, T* dinv,
                   cudaStream_t s) {
    aux_dinv_kernel<T><<<grid_for(a->na * S, AB), AB, 0, s>>>(a->na, S, nsys, a->amask, a->dE, a->dB, a->dR, a->nports,
                                                            k0sq, gamma, dinv, a->agroup);
    return check_cuda(cudaGetLastError(), "aux_dinv_kernel");
}

template int aux_correct<double2>(const emfem_aux_s*, int, bool, const double2*, const double2*, const uint8_t*,
                                  double2*, cudaStream_t);
template int aux_correct<float2>(const emfem_aux_s*, int, bool, const float2*, const float2*, const uint8_t*,
                                 float2*, cudaStream_t);
template int aux_setup_dinv<double2>(const emfem_aux_s*, int, int, const double*, const double*, double2*,
                                     cudaStream_t);
template int aux_setup_dinv<float2>(const emfem_aux_s*, int, int, const double*, const double*, float2*, cudaStream_t);

}  // namespace emfem

using namespace emfem;

static void aux_free(emfem_aux a) {
    if (!a) return;
    cudaFree(a->gcol); cudaFree(a->gval); cudaFree(a->gt_ptr); cudaFree(a->gt_row); cudaFree(a->gt_val);
    cudaFree(a->inc_ptr); cudaFree(a->inc); cudaFree(a->inv_deg); cudaFree(a->atype); cudaFree(a->amask);
    cudaFree(a->dE); cudaFree(a->dB); cudaFree(a->dR); cudaFree(a->kbuf); cudaFree(a->agroup);
    delete a;
}

// Row relabelling for a grouped (multi-mesh) solve: G row r of the aux space's own numbering becomes
// row new_of_old[r] of an n_new-row system (rows not reached stay empty), and G^T's row indices follow.
__global__ void aux_move_rows_kernel(long long n_old, long long n_new, const int64_t* __restrict__ new_of_old,
                                     const int* __restrict__ gcol, const double* __restrict__ gval,
                                     int* __restrict__ gcol_new, double* __restrict__ gval_new, int* status) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_old) return;
    long long q = new_of_old[r];
    if (q < 0 || q >= n_new) { flag(status, DEV_BAD_INDEX); return; }
    for (int k = 0; k < 6; k++) {
        gcol_new[q * 6 + k] = gcol[r * 6 + k];
        gval_new[q * 6 + k] = gval[r * 6 + k];
    }
}

__global__ void aux_relabel_kernel(long long nnz, long long n_old, const int64_t* __restrict__ new_of_old,
                                   int* __restrict__ gt_row, int* status) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    int r = gt_row[k];
    if (r < 0 || r >= n_old) { flag(status, DEV_BAD_INDEX); return; }
    gt_row[k] = (int)new_of_old[r];
}

extern "C" {

int emfem_aux_create(emfem_handle hd, int64_t n_nodes, int64_t n_edges, int64_t n_tris, const int64_t* edges,
                     const int64_t* tris, const int64_t* tri_to_edge, const double* edge_lengths, emfem_aux* out) {
    EMFEM_REQUIRE(hd && edges && tris && tri_to_edge && edge_lengths && out && n_nodes > 0 && n_edges > 0 && n_tris > 0,
                  "emfem_aux_create: bad argument");
    EMFEM_REQUIRE(12 * (n_edges + n_tris) < (1LL << 31) && n_nodes + n_edges < (1LL << 31),
                  "emfem_aux_create: mesh too large for int32 indexing");
    Handle* h = &hd->h;
    cudaStream_t s = h->stream;
    emfem_aux a = new emfem_aux_s();
    a->h = h; a->nn = n_nodes; a->ne = n_edges; a->nf = n_tris;
    a->n = 2 * (n_edges + n_tris); a->na = n_nodes + n_edges;
    long long n = a->n, na = a->na;
    int *cnt = nullptr, *cur = nullptr, *scratch = nullptr;
    int st = EMFEM_OK;
#define ATRY(x) do { st = (x); if (st != EMFEM_OK) goto fail; } while (0)
    ATRY(check_cuda(cudaMemsetAsync(h->dev_status, 0, sizeof(int), s), "memset"));
    ATRY(check_cuda(cudaMalloc(&a->gcol, n * 6 * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->gval, n * 6 * sizeof(double)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->gt_ptr, (na + 1) * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->inc_ptr, (na + 1) * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->inv_deg, na * sizeof(float)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->atype, na), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->amask, na), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->dE, na * sizeof(double2)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->dB, na * sizeof(double2)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->dR, EMFEM_MAX_PORTS * na * sizeof(double2)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&cnt, na * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&cur, na * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&scratch, scan_scratch_ints(na) * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMemsetAsync(a->amask, 0, na, s), "memset"));
    aux_grad_kernel<<<grid_for(n_edges + n_tris, AB), AB, 0, s>>>(n_nodes, n_edges, n_tris, edges, tris, tri_to_edge,
                                                                  edge_lengths, a->gcol, a->gval, h->dev_status);
    ATRY(check_cuda(cudaGetLastError(), "aux_grad_kernel"));
    {
        int dstat = 0;
        ATRY(check_cuda(cudaMemcpyAsync(&dstat, h->dev_status, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        ATRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        if (dstat) {
            set_error("emfem_aux_create: bad edge/triangle node id or non-positive edge length");
            cudaMemsetAsync(h->dev_status, 0, sizeof(int), s);
            st = EMFEM_ERR_DEVICE_CHECK;
            goto fail;
        }
    }
    // G^T in CSR (rows = aux nodes, sorted DOF columns)
    ATRY(check_cuda(cudaMemsetAsync(cnt, 0, na * sizeof(int), s), "memset"));
    ATRY(check_cuda(cudaMemsetAsync(cur, 0, na * sizeof(int), s), "memset"));
    ell_count_kernel<<<grid_for(n, AB), AB, 0, s>>>(n, a->gcol, cnt);
    ATRY(exclusive_scan_i32(h, cnt, a->gt_ptr, na, scratch));
    {
        int tot = 0;
        ATRY(check_cuda(cudaMemcpyAsync(&tot, a->gt_ptr + na, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        ATRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        a->nnz_gt = tot;
    }
    ATRY(check_cuda(cudaMalloc(&a->gt_row, a->nnz_gt * sizeof(int)), "cudaMalloc"));
    ATRY(check_cuda(cudaMalloc(&a->gt_val, a->nnz_gt * sizeof(double)), "cudaMalloc"));
    ell_fill_kernel<<<grid_for(n, AB), AB, 0, s>>>(n, a->gcol, a->gval, a->gt_ptr, cur, a->gt_row, a->gt_val);
    csr_sort_rows_kernel<<<grid_for(na, AB), AB, 0, s>>>(na, a->gt_ptr, a->gt_row, a->gt_val);
    ATRY(check_cuda(cudaGetLastError(), "G^T"));
    // vertex-edge incidence graph
    ATRY(check_cuda(cudaMemsetAsync(cnt, 0, na * sizeof(int), s), "memset"));
    ATRY(check_cuda(cudaMemsetAsync(cur, 0, na * sizeof(int), s), "memset"));
    inc_count_kernel<<<grid_for(n_edges, AB), AB, 0, s>>>(n_nodes, n_edges, edges, cnt);
    ATRY(exclusive_scan_i32(h, cnt, a->inc_ptr, na, scratch));
    a->nnz_inc = 4 * n_edges;
    ATRY(check_cuda(cudaMalloc(&a->inc, a->nnz_inc * sizeof(int)), "cudaMalloc"));
    inc_fill_kernel<<<grid_for(n_edges, AB), AB, 0, s>>>(n_nodes, n_edges, edges, a->inc_ptr, cur, a->inc);
    csr_sort_rows_kernel<<<grid_for(na, AB), AB, 0, s>>>(na, a->inc_ptr, a->inc, nullptr);
    inv_deg_type_kernel<<<grid_for(na, AB), AB, 0, s>>>(n_nodes, na, a->inc_ptr, a->inv_deg, a->atype);
    ATRY(check_cuda(cudaGetLastError(), "incidence graph"));
    ATRY(check_cuda(cudaStreamSynchronize(s), "sync"));
    cudaFree(cnt); cudaFree(cur); cudaFree(scratch);
    *out = a;
    return EMFEM_OK;
fail:
    cudaFree(cnt); cudaFree(cur); cudaFree(scratch);
    aux_free(a);
    return st;
#undef ATRY
}

int emfem_aux_info(emfem_aux a, int64_t* n_aux, int64_t* nnz_gt, int64_t* nnz_graph) {
    EMFEM_REQUIRE(a, "emfem_aux_info: null");
    if (n_aux) *n_aux = a->na;
    if (nnz_gt) *nnz_gt = a->nnz_gt;
    if (nnz_graph) *nnz_graph = a->nnz_inc;
    return EMFEM_OK;
}

int emfem_aux_export(emfem_aux a, int32_t* gcol, double* gval, int32_t* gt_ptr, int32_t* gt_row, double* gt_val,
                     int32_t* graph_ptr, int32_t* graph_nbr) {
    EMFEM_REQUIRE(a, "emfem_aux_export: null");
    cudaStream_t s = a->h->stream;
    if (gcol) EMFEM_CUDA(cudaMemcpyAsync(gcol, a->gcol, a->n * 6 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (gval) EMFEM_CUDA(cudaMemcpyAsync(gval, a->gval, a->n * 6 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (gt_ptr) EMFEM_CUDA(cudaMemcpyAsync(gt_ptr, a->gt_ptr, (a->na + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (gt_row) EMFEM_CUDA(cudaMemcpyAsync(gt_row, a->gt_row, a->nnz_gt * sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (gt_val) EMFEM_CUDA(cudaMemcpyAsync(gt_val, a->gt_val, a->nnz_gt * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (graph_ptr) EMFEM_CUDA(cudaMemcpyAsync(graph_ptr, a->inc_ptr, (a->na + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (graph_nbr) EMFEM_CUDA(cudaMemcpyAsync(graph_nbr, a->inc, a->nnz_inc * sizeof(int), cudaMemcpyDeviceToDevice, s));
    return EMFEM_OK;
}

int emfem_aux_set_operator(emfem_aux a, int64_t n, const int32_t* indptr, const int32_t* indices, const void* E_vals,
                           const void* B_vals, int64_t n_patch_rows, const int32_t* patch_rows,
                           const int32_t* patch_rowptr, const int32_t* patch_cols, const void* patch_vals,
                           const int32_t* patch_port, int n_ports, const uint8_t* free_mask, void* diag_out,
                           uint8_t* mask_out) {
    EMFEM_REQUIRE(a && indptr && indices && E_vals && B_vals && free_mask && n == a->n,
                  "emfem_aux_set_operator: bad argument (n must equal the aux space's field size)");
    EMFEM_REQUIRE(n_ports >= 0 && n_ports <= EMFEM_MAX_PORTS, "emfem_aux_set_operator: too many ports");
    EMFEM_REQUIRE(n_patch_rows == 0 || (patch_rows && patch_rowptr && patch_cols && patch_vals && patch_port),
                  "emfem_aux_set_operator: patch arrays missing");
    cudaStream_t s = a->h->stream;
    int* pmap = nullptr;
    if (n_patch_rows > 0) {
        EMFEM_CUDA(cudaMallocAsync(&pmap, sizeof(int) * n, s));
        EMFEM_CUDA(cudaMemsetAsync(pmap, 0xff, sizeof(int) * n, s));
        launch_patch_map(n_patch_rows, patch_rows, pmap, s);
    }
    EMFEM_CUDA(cudaMemsetAsync(a->dR, 0, EMFEM_MAX_PORTS * a->na * sizeof(double2), s));
    aux_diag_kernel<<<grid_for(a->na * 32, AB), AB, 0, s>>>(
        a->na, a->gt_ptr, a->gt_row, a->gt_val, indptr, indices, (const double2*)E_vals, (const double2*)B_vals, pmap,
        patch_rowptr, patch_cols, (const double2*)patch_vals, patch_port, n_ports, free_mask, a->dE, a->dB, a->dR,
        a->amask);
    EMFEM_LAUNCH("aux_diag_kernel");
    if (pmap) EMFEM_CUDA(cudaFreeAsync(pmap, s));
    a->nports = n_ports;
    a->have_operator = true;
    if (diag_out) {
        // [dE | dB | dR_0 .. dR_{P-1}], complex, n_aux each
        double2* o = (double2*)diag_out;
        EMFEM_CUDA(cudaMemcpyAsync(o, a->dE, a->na * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        EMFEM_CUDA(cudaMemcpyAsync(o + a->na, a->dB, a->na * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        if (n_ports > 0)
            EMFEM_CUDA(cudaMemcpyAsync(o + 2 * a->na, a->dR, n_ports * a->na * sizeof(double2),
                                       cudaMemcpyDeviceToDevice, s));
    }
    if (mask_out) EMFEM_CUDA(cudaMemcpyAsync(mask_out, a->amask, a->na, cudaMemcpyDeviceToDevice, s));
    return EMFEM_OK;
}

int emfem_aux_reserve(emfem_aux a, int nsys) {
    EMFEM_REQUIRE(a && nsys >= 1 && nsys <= 64, "emfem_aux_reserve: 1 <= nsys <= 64");
    int S = 1;
    while (S < nsys) S <<= 1;
    size_t need = aux_solve_bytes(a, S);
    if (need > a->kbuf_bytes) {
        EMFEM_CUDA(cudaStreamSynchronize(a->h->stream));
        cudaFree(a->kbuf);
        a->kbuf = nullptr;
        a->kbuf_bytes = 0;
        EMFEM_CUDA(cudaMalloc(&a->kbuf, need));
        a->kbuf_bytes = need;
    }
    return EMFEM_OK;
}

int emfem_aux_set_network(emfem_aux a, const float* params) {
    EMFEM_REQUIRE(a, "emfem_aux_set_network: null");
    a->params = (float*)params;
    return EMFEM_OK;
}

int emfem_aux_set_rows(emfem_aux a, int64_t n_new, const int64_t* new_of_old, int ngroups, const int32_t* aux_group) {
    EMFEM_REQUIRE(a && new_of_old && n_new >= a->n && n_new < (1LL << 31) && (n_new % 2) == 0,
                  "emfem_aux_set_rows: bad argument (n_new must be even, >= the current rows, < 2^31)");
    EMFEM_REQUIRE(ngroups >= 1 && (ngroups == 1 || aux_group), "emfem_aux_set_rows: aux_group required for ngroups > 1");
    cudaStream_t st = a->h->stream;
    int* gcol_new = nullptr;
    double* gval_new = nullptr;
    int* grp = nullptr;
    int rc = EMFEM_OK;
    if ((rc = check_cuda(cudaMalloc(&gcol_new, n_new * 6 * sizeof(int)), "cudaMalloc")) != EMFEM_OK) return rc;
    if ((rc = check_cuda(cudaMalloc(&gval_new, n_new * 6 * sizeof(double)), "cudaMalloc")) != EMFEM_OK) {
        cudaFree(gcol_new);
        return rc;
    }
    if (ngroups > 1 && (rc = check_cuda(cudaMalloc(&grp, a->na * sizeof(int)), "cudaMalloc")) != EMFEM_OK) {
        cudaFree(gcol_new); cudaFree(gval_new);
        return rc;
    }
    cudaMemsetAsync(gcol_new, 0xff, n_new * 6 * sizeof(int), st);
    cudaMemsetAsync(gval_new, 0, n_new * 6 * sizeof(double), st);
    aux_move_rows_kernel<<<grid_for(a->n, AB), AB, 0, st>>>(a->n, n_new, new_of_old, a->gcol, a->gval, gcol_new, gval_new,
                                                            a->h->dev_status);
    if (a->nnz_gt > 0)
        aux_relabel_kernel<<<grid_for(a->nnz_gt, AB), AB, 0, st>>>(a->nnz_gt, a->n, new_of_old, a->gt_row, a->h->dev_status);
    if (grp) cudaMemcpyAsync(grp, aux_group, a->na * sizeof(int), cudaMemcpyDeviceToDevice, st);
    rc = check_cuda(cudaStreamSynchronize(st), "emfem_aux_set_rows");
    if (rc != EMFEM_OK) { cudaFree(gcol_new); cudaFree(gval_new); cudaFree(grp); return rc; }
    cudaFree(a->gcol); cudaFree(a->gval); cudaFree(a->agroup);
    a->gcol = gcol_new; a->gval = gval_new; a->agroup = grp;
    a->n = n_new;
    a->ngroups = ngroups;
    a->have_operator = false;
    return EMFEM_OK;
}

int emfem_aux_destroy(emfem_aux a) {
    aux_free(a);
    return EMFEM_OK;
}

int emfem_aux_dinv(emfem_aux a, int nsys, const double* k0sq_dev, const double* gamma_dev, void* dinv) {
    EMFEM_REQUIRE(a && k0sq_dev && dinv && nsys >= 1 && a->have_operator, "emfem_aux_dinv: bad argument or no operator");
    EMFEM_REQUIRE(a->nports == 0 || gamma_dev, "emfem_aux_dinv: gamma missing");
    aux_dinv_kernel<double2><<<grid_for(a->na * nsys, AB), AB, 0, a->h->stream>>>(
        a->na, nsys, nsys, a->amask, a->dE, a->dB, a->dR, a->nports, k0sq_dev, gamma_dev, (double2*)dinv);
    EMFEM_LAUNCH("aux_dinv_kernel");
    return EMFEM_OK;
}

int emfem_aux_restrict(emfem_aux a, int nsys, const void* dinv, const void* v, void* x) {
    EMFEM_REQUIRE(a && v && x && nsys >= 1, "emfem_aux_restrict: bad argument");
    aux_restrict_kernel<double2, double2><<<grid_for(a->na * nsys, AB), AB, 0, a->h->stream>>>(
        a->na, nsys, a->gt_ptr, a->gt_row, a->gt_val, (const double2*)dinv, (const double2*)v, (double2*)x);
    EMFEM_LAUNCH("aux_restrict_kernel");
    return EMFEM_OK;
}

int emfem_aux_prolong(emfem_aux a, int nsys, const void* za, const uint8_t* free_mask, void* z, int accumulate) {
    EMFEM_REQUIRE(a && za && z && nsys >= 1, "emfem_aux_prolong: bad argument");
    aux_prolong_kernel<double2, double2><<<grid_for(a->n * nsys, AB), AB, 0, a->h->stream>>>(
        a->n, nsys, a->gcol, a->gval, (const double2*)za, free_mask, (double2*)z, accumulate);
    EMFEM_LAUNCH("aux_prolong_kernel");
    return EMFEM_OK;
}

int emfem_mpnn_nparams(void) { return EMFEM_MPNN_NPARAMS; }

int emfem_mpnn_workspace_floats(emfem_aux a, int nsys, int64_t* activation_floats, int64_t* scratch_floats) {
    EMFEM_REQUIRE(a && nsys >= 1, "emfem_mpnn_workspace_floats: bad argument");
    int64_t act = (int64_t)a->na * nsys * NN_C * 2;
    if (activation_floats) *activation_floats = NN_L * act;
    if (scratch_floats) *scratch_floats = 3 * act + (int64_t)WG_BLOCKS * 4 * NN_C * NN_C;
    return EMFEM_OK;
}

int emfem_mpnn_forward(emfem_aux a, int nsys, const float* params, const void* x, float* act, void* za) {
    EMFEM_REQUIRE(a && params && x && act && za && nsys >= 1, "emfem_mpnn_forward: bad argument");
    return mpnn_forward<float2>(a, nsys, params, (const float2*)x, nullptr, nullptr, (float2*)act, (float2*)za,
                                a->h->stream);
}

int emfem_mpnn_infer(emfem_aux a, int nsys, const float* params, const void* x, float* work, void* za) {
    EMFEM_REQUIRE(a && params && x && work && za && nsys >= 1, "emfem_mpnn_infer: bad argument");
    float2* H0 = (float2*)work;
    float2* H1 = H0 + (size_t)a->na * nsys * NN_C;
    return mpnn_forward_tc<float2>(a, nsys, params, (const float2*)x, H0, H1, (float2*)za, a->h->stream);
}

int emfem_mpnn_backward(emfem_aux a, int nsys, const float* params, const void* x, const float* act, const void* dza,
                        float* grad, float* scratch) {
    EMFEM_REQUIRE(a && params && x && act && dza && grad && scratch && nsys >= 1, "emfem_mpnn_backward: bad argument");
    cudaStream_t s = a->h->stream;
    long long na = a->na, rows = na * nsys;
    size_t actn = (size_t)rows * NN_C;
    float2* dOut = (float2*)scratch;
    float2* dM = dOut + actn;
    float2* dIn = dM + actn;
    float* partial = (float*)(dIn + actn);
    const float2* A = (const float2*)act;
    unsigned gw = warp_grid(rows);
    mpnn_bwd_out_kernel<float2><<<grid_for(rows * NN_C, AB), AB, 0, s>>>(na, nsys, params, a->atype,
                                                                         (const float2*)dza, dOut);
    // w_out gradient from dza and the last layer's output, before dOut is overwritten
    mpnn_bwd_vec_kernel<float2><<<WG_BLOCKS, AB, 0, s>>>(na, nsys, a->atype, (const float2*)x, dOut,
                                                         A + (size_t)(NN_L - 1) * actn, (const float2*)dza, partial);
    partial_sum_kernel<<<1, 2 * NN_C, 0, s>>>(WG_BLOCKS, 4 * NN_C, 2 * NN_C, partial + 2 * NN_C, grad + nn_off_wout());
    for (int l = NN_L - 1; l >= 0; l--) {
        const float2* Hin = l > 0 ? A + (size_t)(l - 1) * actn : nullptr;
        mpnn_bwd_wgrad_kernel<float2><<<WG_BLOCKS, AB, 0, s>>>(na, nsys, l, params, a->inc_ptr, a->inc, a->inv_deg,
                                                               a->atype, (const float2*)x, Hin, dOut, partial);
        // partial rows are [t][mat][C][C]; grad holds W_l[t][C][C] then U_l[t][C][C]
        for (int t = 0; t < 2; t++)
            for (int mat = 0; mat < 2; mat++) {
                float* dst = grad + (mat == 0 ? nn_off_W(l) : nn_off_U(l)) + t * NN_C * NN_C;
                partial_sum_kernel<<<grid_for(NN_C * NN_C, AB), AB, 0, s>>>(
                    WG_BLOCKS, 4 * NN_C * NN_C, NN_C * NN_C, partial + (t * 2 + mat) * NN_C * NN_C, dst);
            }
        mpnn_bwd_dm_kernel<<<gw, AB, 0, s>>>(na, nsys, l, params, a->inv_deg, a->atype, dOut, dM);
        mpnn_bwd_din_kernel<<<gw, AB, 0, s>>>(na, nsys, l, params, a->inc_ptr, a->inc, a->atype, dOut, dM, dIn);
        std::swap(dOut, dIn);   // dIn of layer l is dOut of layer l - 1
    }
    EMFEM_LAUNCH("mpnn backward");
    // dOut now holds dL/d in_0 = dL/d(x w_in) per channel: w_in gradient
    mpnn_bwd_vec_kernel<float2><<<WG_BLOCKS, AB, 0, s>>>(na, nsys, a->atype, (const float2*)x, dOut,
                                                         A + (size_t)(NN_L - 1) * actn, (const float2*)dza, partial);
    partial_sum_kernel<<<1, 2 * NN_C, 0, s>>>(WG_BLOCKS, 4 * NN_C, 2 * NN_C, partial, grad + nn_off_win());
    EMFEM_LAUNCH("mpnn backward vectors");
    return EMFEM_OK;
}

int emfem_adam_step(emfem_handle hd, int64_t n, float* params, const float* grad, float* m, float* v, float lr,
                    float beta1, float beta2, float eps, float weight_decay, int step) {
    EMFEM_REQUIRE(hd && params && grad && m && v && n > 0 && step >= 1, "emfem_adam_step: bad argument");
    float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(n, AB), AB, 0, hd->h.stream>>>(n, params, grad, m, v, lr, beta1, beta2, eps, c1, c2,
                                                         weight_decay);
    EMFEM_LAUNCH("adam_kernel");
    return EMFEM_OK;
}

}  // extern "C"
