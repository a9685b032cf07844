// Frequency-sweep operator and batched Krylov solvers (COCG and BiCGStab).
//
// Replaces the per-frequency direct solve (SolverSuperLU, src/emerge/_emerge/solver.py:535-572,
// through SolveRoutine.solve :1241-1326) for the systems K_f = E - k0_f^2 B + sum_p gamma_{f,p} R_p
// that Assembler.assemble_freq_matrix builds (ASM/assembler.py:255, :314-350).  All systems of a
// batch share one CSR pattern; vectors are DOF-major (n, S) so one pass over the pattern's column
// indices and E/B values serves every system, and the S entries of a gathered column are
// contiguous.  PEC elimination (SolveRoutine's A[ids, ids], solver.py:1266-1269) is a free-DOF
// mask: eliminated rows produce 0 and eliminated entries of every Krylov vector stay 0.
//
// Methods.  COCG (van der Vorst & Melissen 1990) is CG with the unconjugated form x^T y and is
// exact for complex-symmetric A.  The reference's mass matrix is not symmetric: its face-face
// block uses coefficient tables whose index lists differ between (i, j) and (j, i)
// (ASM/curlcurl.py:348-357, e.g. VBCDE = VOLUME_COEFF_CACHE[B,C,D,F]), about 0.5 % of ||B||, and
// COCG stalls near 1e-5 on it.  The default is therefore right-preconditioned BiCGStab
// (van der Vorst 1992), the general-matrix member of the same BiCG family, with the same batched
// operator and preconditioner.  Every reduction is a fixed-order tree, so runs are
// bit-reproducible.  Iterations run in CUDA-graph chunks with all scalars on the device; the host
// reads only the per-system active flags between chunks.
#include "emfem_internal.cuh"

#include <vector>
#include <algorithm>
#include <cmath>

namespace emfem {

template <typename R> struct V2;
template <> struct V2<double> { typedef double2 T; };
template <> struct V2<float> { typedef float2 T; };

template <typename R, typename T = typename V2<R>::T>
__device__ __forceinline__ T mk2(R x, R y) { T v; v.x = x; v.y = y; return v; }

constexpr int VB = 256;  // threads per block for vector/SpMV kernels

// relative tolerance of each FP32 inner solve in the mixed-precision refinement (compile-time)
#ifndef EMFEM_INNER_TOL
#define EMFEM_INNER_TOL 1e-4
#endif

struct SysState;

struct OpArgs {
    long long n;
    int S;                          // padded systems (power of two, divides VB)
    const int* indptr;
    const int* indices;
    const void* E;                  // value arrays (precision of the kernel)
    const void* B;                  // may be null
    const double* k0sq;             // [S]
    const int* patch_of_row;        // [n], -1 or index into patch rows
    const int* patch_rowptr;
    const int* patch_cols;
    const void* patch_vals;         // complex of kernel precision
    const int* patch_port;
    int n_ports;
    const double* gamma;            // [S][n_ports] complex (interleaved)
    const uint8_t* mask;            // [n]
    // grouped systems (emfem_krylov_solve_grouped): group of every DOF pair i < hh, or null.  Row i
    // (or i - hh) of system column s then belongs to system pg[i] * S + s of the per-system arrays.
    const int* pg;
    long long hh;
    // inside a Krylov iteration: the per-system state; rows of systems that are no longer active are
    // skipped (their scalars are zero, so these vectors are not used again).  Null elsewhere.
    const SysState* skip;
};

__device__ __forceinline__ bool sys_active(const SysState* st, int sy);

__device__ __forceinline__ int sys_of_row(const int* pg, long long hh, long long i, int S, int s) {
    return pg ? pg[i < hh ? i : i - hh] * S + s : s;
}

template <typename T>
__device__ __forceinline__ double2 dotu(T a, T b) {  // a^T b contribution (unconjugated)
    return make_double2((double)a.x * b.x - (double)a.y * b.y, (double)a.x * b.y + (double)a.y * b.x);
}
template <typename T>
__device__ __forceinline__ double2 dotc(T a, T b) {  // conj(a) b
    return make_double2((double)a.x * b.x + (double)a.y * b.y, (double)a.x * b.y - (double)a.y * b.x);
}
template <typename T>
__device__ __forceinline__ double nrm2(T a) { return (double)a.x * a.x + (double)a.y * a.y; }

enum DotMode { DOT_NONE = 0, DOT_XY = 1, DOT_CONJW_Y = 2, DOT_CONJY_W_YY = 3 };

// Block-level fixed-order tree reduction of up to three components per thread (two complex, one
// real); thread s < S stores component c of this block at partial[(c * nblocks + block) * S + s].
__device__ __forceinline__ void block_store3(double2 v0, double2 v1, double v2, int ncomp, int S, double2* partial) {
    __shared__ double2 r0[VB], r1[VB];
    __shared__ double r2[VB];
    r0[threadIdx.x] = v0;
    r1[threadIdx.x] = v1;
    r2[threadIdx.x] = v2;
    __syncthreads();
    for (int off = VB / 2; off >= S; off >>= 1) {
        if (threadIdx.x < off) {
            r0[threadIdx.x].x += r0[threadIdx.x + off].x; r0[threadIdx.x].y += r0[threadIdx.x + off].y;
            r1[threadIdx.x].x += r1[threadIdx.x + off].x; r1[threadIdx.x].y += r1[threadIdx.x + off].y;
            r2[threadIdx.x] += r2[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x < S) {
        partial[(long long)blockIdx.x * S + threadIdx.x] = r0[threadIdx.x];
        if (ncomp > 1) partial[((long long)gridDim.x + blockIdx.x) * S + threadIdx.x] = r1[threadIdx.x];
        if (ncomp > 2) partial[(2LL * gridDim.x + blockIdx.x) * S + threadIdx.x] = make_double2(r2[threadIdx.x], 0.0);
    }
}
__device__ __forceinline__ void block_store2(double2 v0, double2 v1, int ncomp, int S, double2* partial) {
    block_store3(v0, v1, 0.0, ncomp, S, partial);
}

// y = A x for all systems, one thread per (row, system); optional dot-product epilogue (DotMode).
// The operator values (E, B, Robin patch) are always FP64 and every row is accumulated in FP64;
// R is the precision of the Krylov vectors only (FP32 in the mixed-precision inner solve), so the
// inner iterations see the exact operator and only the vectors are rounded.  Rounding E and B to
// FP32 separately would lose the cancellation in E - k0^2 B near resonances.
template <typename R>
__global__ void __launch_bounds__(VB) spmv_kernel(OpArgs a, const typename V2<R>::T* __restrict__ x,
                                                   typename V2<R>::T* __restrict__ y, double2* __restrict__ partial,
                                                   int dotmode, const typename V2<R>::T* __restrict__ w) {
    typedef typename V2<R>::T T;
    const int S = a.S;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 c0 = make_double2(0.0, 0.0), c1 = c0;
    double c2 = 0.0;
    const int sy = i < a.n ? sys_of_row(a.pg, a.hh, i, S, s) : 0;
    bool act = i < a.n && (!a.skip || sys_active(a.skip, sy));
    // S >= 32: the 32 lanes of a warp are 32 systems of one row and stage that row's entries together
    // (warp-synchronous below), so the warp skips the row only when none of its systems is active.
    // Every lane reaches this vote, and the row index is the same for the whole warp.
    if (S >= 32) act = __any_sync(0xffffffffu, act);
    if (act) {
        double yr = 0, yi = 0;
        if (a.mask[i]) {
            const double2* Ev = (const double2*)a.E;
            const double2* Bv = (const double2*)a.B;
            double er = 0, ei = 0, br = 0, bi = 0;
            int jb = a.indptr[i], je = a.indptr[i + 1];
            int j = jb;
            if (S >= 32) {
                // a warp holds 32 systems of one row: it stages 32 consecutive (column, E, B) entries
                // with one coalesced load per lane and reads them back as shared-memory broadcasts;
                // the products are summed in column order as below
                __shared__ int s_c[VB / 32][32];
                __shared__ double2 s_e[VB / 32][32], s_b[VB / 32][32];
                const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
                for (int base = jb; base < je; base += 32) {
                    int jj = base + lane;
                    if (jj < je) {
                        s_c[wl][lane] = a.indices[jj];
                        s_e[wl][lane] = Ev[jj];
                        s_b[wl][lane] = Bv ? Bv[jj] : make_double2(0.0, 0.0);
                    }
                    __syncwarp();
                    const int cnt = min(32, je - base);
                    int u = 0;
                    for (; u + 4 <= cnt; u += 4) {
                        T xv[4];
#pragma unroll
                        for (int t = 0; t < 4; t++) xv[t] = x[(long long)s_c[wl][u + t] * S + s];
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            double2 e = s_e[wl][u + t], b = s_b[wl][u + t];
                            double xr = xv[t].x, xi = xv[t].y;
                            er += e.x * xr - e.y * xi;
                            ei += e.x * xi + e.y * xr;
                            if (Bv) {
                                br += b.x * xr - b.y * xi;
                                bi += b.x * xi + b.y * xr;
                            }
                        }
                    }
                    for (; u < cnt; u++) {
                        T xv = x[(long long)s_c[wl][u] * S + s];
                        double2 e = s_e[wl][u], b = s_b[wl][u];
                        double xr = xv.x, xi = xv.y;
                        er += e.x * xr - e.y * xi;
                        ei += e.x * xi + e.y * xr;
                        if (Bv) {
                            br += b.x * xr - b.y * xi;
                            bi += b.x * xi + b.y * xr;
                        }
                    }
                    __syncwarp();
                }
                j = je;
            }
            // four entries' loads are issued before their products are summed (in column order, so
            // the sums are the same as the one-at-a-time loop): the row walk is latency-bound
            for (; j + 4 <= je; j += 4) {
                int cc[4];
                T xv[4];
                double2 e[4], b[4];
#pragma unroll
                for (int u = 0; u < 4; u++) cc[u] = a.indices[j + u];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    xv[u] = x[(long long)cc[u] * S + s];
                    e[u] = Ev[j + u];
                    b[u] = Bv ? Bv[j + u] : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    double xr = xv[u].x, xi = xv[u].y;
                    er += e[u].x * xr - e[u].y * xi;
                    ei += e[u].x * xi + e[u].y * xr;
                    if (Bv) {
                        br += b[u].x * xr - b[u].y * xi;
                        bi += b[u].x * xi + b[u].y * xr;
                    }
                }
            }
            for (; j < je; j++) {
                int c = a.indices[j];
                T xv = x[(long long)c * S + s];
                double xr = xv.x, xi = xv.y;
                double2 e = Ev[j];
                er += e.x * xr - e.y * xi;
                ei += e.x * xi + e.y * xr;
                if (Bv) {
                    double2 b = Bv[j];
                    br += b.x * xr - b.y * xi;
                    bi += b.x * xi + b.y * xr;
                }
            }
            double k2 = a.k0sq[sy];
            yr = er - k2 * br;
            yi = ei - k2 * bi;
            int pr = a.patch_of_row ? a.patch_of_row[i] : -1;
            if (pr >= 0) {
                const double2* Pv = (const double2*)a.patch_vals;
                for (int q = 0; q < a.n_ports; q++) {
                    double pr_ = 0, pi_ = 0;
                    for (int j = a.patch_rowptr[pr]; j < a.patch_rowptr[pr + 1]; j++) {
                        if (a.patch_port[j] != q) continue;
                        T xv = x[(long long)a.patch_cols[j] * S + s];
                        double2 v = Pv[j];
                        pr_ += v.x * xv.x - v.y * xv.y;
                        pi_ += v.x * xv.y + v.y * xv.x;
                    }
                    double gr = a.gamma[2 * (sy * a.n_ports + q)], gi = a.gamma[2 * (sy * a.n_ports + q) + 1];
                    yr += gr * pr_ - gi * pi_;
                    yi += gr * pi_ + gi * pr_;
                }
            }
        }
        y[i * S + s] = mk2<R>((R)yr, (R)yi);
        if (dotmode == DOT_XY) {
            T xi = x[i * S + s];
            c0 = make_double2((double)xi.x * yr - (double)xi.y * yi, (double)xi.x * yi + (double)xi.y * yr);
        } else if (dotmode == DOT_CONJW_Y) {
            T wi = w[i * S + s];
            c0 = make_double2((double)wi.x * yr + (double)wi.y * yi, (double)wi.x * yi - (double)wi.y * yr);
        } else if (dotmode == DOT_CONJY_W_YY) {
            T wi = w[i * S + s];
            c0 = make_double2(yr * wi.x + yi * wi.y, yr * wi.y - yi * wi.x);
            c1 = make_double2(yr * yr + yi * yi, 0.0);
            c2 = nrm2(wi);
        }
    }
    if (dotmode != DOT_NONE) block_store3(c0, c1, c2, dotmode == DOT_CONJY_W_YY ? 3 : 1, S, partial);
}

// Solver state per system (device).
struct SysState {
    double2 rho;      // COCG: r^T z;   BiCGStab: (r_hat, r)
    double2 alpha;
    double2 beta;
    double2 omega;
    double rn2;       // ||r||^2 (conjugated)
    double bn2;       // ||b||^2
    double tol2;      // tol^2 * bn2
    double rh2;       // BiCGStab: ||r_hat||^2 (shadow residual)
    int active;
    int iters;
    int status;       // 0 converged, 1 cap, 2 breakdown
    int restart;      // BiCGStab: take r_hat = r at the next p update
};

__device__ __forceinline__ bool sys_active(const SysState* st, int sy) { return st[sy].active != 0; }

__device__ __forceinline__ double2 cdiv2(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

enum UpdateMode { UPD_INIT = 0, UPD_SET_RHO = 1, UPD_COCG_ALPHA = 2, UPD_COCG_BETA = 3,
                  UPD_BICG_ALPHA = 4, UPD_BICG_OMEGA = 5, UPD_BICG_RHO = 6 };

__device__ void stop(SysState& q, int status) {
    q.active = 0; q.status = status;
    q.alpha = make_double2(0, 0); q.omega = make_double2(0, 0); q.beta = make_double2(0, 0);
}

// One block per system: fixed-order sum of the block partials, then the scalar recurrences.
// Grouped systems (G > 1): block sys = g S + s sums only group g's blocks, gblk[g] .. gblk[g + 1] of
// a DOF-pair launch (nbh blocks), and for a launch over all rows also the same range in the second
// half (two_halves).
__global__ void reduce_update_kernel(const double2* __restrict__ partial, int nblocks, int S, int ncomp,
                                     SysState* st, int mode, int maxit, double tol, int nsys, int G = 1,
                                     const int* __restrict__ gblk = nullptr, int two_halves = 0, int nbh = 0) {
    __shared__ double2 red[VB];
    __shared__ double2 sums[3];
    const int sys = blockIdx.x;
    const int s = G > 1 ? sys % S : sys;
    int b0 = 0, cnt = nblocks, total = nblocks;
    if (G > 1) {
        b0 = gblk[sys / S];
        cnt = gblk[sys / S + 1] - b0;
        total = two_halves ? 2 * cnt : cnt;
    }
    for (int comp = 0; comp < ncomp; comp++) {
        double2 acc = make_double2(0, 0);
        for (int k = threadIdx.x; k < total; k += VB) {
            int b = k < cnt ? b0 + k : nbh + b0 + (k - cnt);
            double2 v = partial[((long long)comp * nblocks + b) * S + s];
            acc.x += v.x; acc.y += v.y;
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int off = VB / 2; off > 0; off >>= 1) {
            if (threadIdx.x < off) { red[threadIdx.x].x += red[threadIdx.x + off].x; red[threadIdx.x].y += red[threadIdx.x + off].y; }
            __syncthreads();
        }
        if (threadIdx.x == 0) sums[comp] = red[0];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    SysState& q = st[sys];
    double2 c0 = sums[0], c1 = ncomp > 1 ? sums[1] : make_double2(0, 0);
    double c2 = ncomp > 2 ? sums[2].x : 0.0;
    switch (mode) {
    case UPD_INIT: {  // c0 = ||b||^2, c1 = ||r||^2
        SysState z;
        z.rho = z.alpha = z.beta = z.omega = make_double2(0, 0);
        z.alpha.x = 1.0; z.omega.x = 1.0;
        z.bn2 = c0.x; z.rn2 = c1.x; z.tol2 = tol * tol * c0.x;
        z.iters = 0; z.status = 0; z.restart = 0; z.rh2 = 0;
        z.active = (s < nsys) && (z.bn2 > 0) && (z.rn2 > z.tol2);
        st[sys] = z;
        break;
    }
    case UPD_SET_RHO:
        q.rho = c0;
        q.rh2 = c0.x;
        break;
    case UPD_COCG_ALPHA:
        if (!q.active) { q.alpha = make_double2(0, 0); break; }
        if (!(cabs1(c0) > 0) || !isfinite(cabs1(c0))) { stop(q, 2); break; }
        q.alpha = cdiv2(q.rho, c0);
        break;
    case UPD_COCG_BETA:
        if (!q.active) { q.beta = make_double2(0, 0); break; }
        q.rn2 = c1.x;
        q.iters += 1;
        if (q.rn2 <= q.tol2) { stop(q, 0); break; }
        if (!isfinite(q.rn2)) { stop(q, 2); break; }
        if (q.iters >= maxit) { stop(q, 1); break; }
        if (!(cabs1(q.rho) > 0)) { stop(q, 2); break; }
        q.beta = cdiv2(c0, q.rho);
        q.rho = c0;
        break;
    case UPD_BICG_ALPHA:
        q.restart = 0;
        if (!q.active) { q.alpha = make_double2(0, 0); break; }
        if (!(cabs1(c0) > 0) || !isfinite(cabs1(c0))) { stop(q, 2); break; }
        q.alpha = cdiv2(q.rho, c0);
        break;
    case UPD_BICG_OMEGA: {
        // c0 = (t, s), c1 = ||t||^2, c2 = ||s||^2.  Minimal-residual omega, enlarged when t and s are
        // nearly orthogonal (Sleijpen & van der Vorst 1995, "maintaining convergence properties of
        // BiCGstab methods in finite precision arithmetic": |cos| >= 0.7).
        if (!q.active) { q.omega = make_double2(0, 0); break; }
        if (!(c1.x > 0)) { q.omega = make_double2(0, 0); break; }
        q.omega = make_double2(c0.x / c1.x, c0.y / c1.x);
        double cosang = sqrt(c0.x * c0.x + c0.y * c0.y) / sqrt(c1.x * c2);
        if (cosang > 0 && cosang < 0.7) { double f = 0.7 / cosang; q.omega.x *= f; q.omega.y *= f; }
        break;
    }
    case UPD_BICG_RHO: {
        if (!q.active) { q.beta = make_double2(0, 0); break; }
        q.rn2 = c1.x;
        q.iters += 1;
        if (q.rn2 <= q.tol2) { stop(q, 0); break; }
        if (!isfinite(q.rn2)) { stop(q, 2); break; }
        if (q.iters >= maxit) { stop(q, 1); break; }
        if (!(cabs1(q.rho) > 0) || !(cabs1(q.omega) > 0)) { stop(q, 2); break; }
        // restart with r_hat = r when (r_hat, r) is nearly orthogonal (tol carries the threshold)
        if (sqrt(c0.x * c0.x + c0.y * c0.y) < tol * sqrt(q.rh2 * q.rn2)) {
            q.restart = 1;
            q.rho = make_double2(q.rn2, 0.0);
            q.rh2 = q.rn2;
            q.beta = make_double2(0, 0);
            break;
        }
        q.beta = cmul2(cdiv2(c0, q.rho), cdiv2(q.alpha, q.omega));
        q.rho = c0;
        break;
    }
    }
}

// Preconditioner: z = M^-1 r on DOF pairs (i, i + h); precond 0 = identity.
template <typename R>
__device__ __forceinline__ void apply_pair(int precond, const typename V2<R>::T* __restrict__ minv, int S,
                                           long long i, int s, typename V2<R>::T a, typename V2<R>::T b,
                                           typename V2<R>::T& z_lo, typename V2<R>::T& z_hi) {
    if (precond == 0) { z_lo = a; z_hi = b; return; }
    typedef typename V2<R>::T T;
    const T* m = minv + (i * S + s) * 4;
    T m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
    z_lo = mk2<R>(m00.x * a.x - m00.y * a.y + m01.x * b.x - m01.y * b.y, m00.x * a.y + m00.y * a.x + m01.x * b.y + m01.y * b.x);
    z_hi = mk2<R>(m10.x * a.x - m10.y * a.y + m11.x * b.x - m11.y * b.y, m10.x * a.y + m10.y * a.x + m11.x * b.y + m11.y * b.x);
}


// ---- COCG vector kernels (thread per DOF pair i < h and system s) ----
template <typename R>
__global__ void __launch_bounds__(VB) cocg_init_kernel(long long h, int S, int precond, const typename V2<R>::T* __restrict__ r,
                                                       typename V2<R>::T* __restrict__ z, typename V2<R>::T* __restrict__ p,
                                                       const typename V2<R>::T* __restrict__ minv, double2* __restrict__ partial) {
    typedef typename V2<R>::T T;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 rz = make_double2(0, 0);
    if (i < h) {
        T rl = r[i * S + s], rh = r[(i + h) * S + s], zl, zh;
        apply_pair<R>(precond, minv, S, i, s, rl, rh, zl, zh);
        z[i * S + s] = zl; z[(i + h) * S + s] = zh;
        p[i * S + s] = zl; p[(i + h) * S + s] = zh;
        double2 a = dotu(rl, zl), b = dotu(rh, zh);
        rz = make_double2(a.x + b.x, a.y + b.y);
    }
    block_store2(rz, rz, 1, S, partial);
}

template <typename R>
__global__ void __launch_bounds__(VB) cocg_update_kernel(long long h, int S, int precond, const int* __restrict__ pg,
                                                         const SysState* __restrict__ st,
                                                         typename V2<R>::T* __restrict__ x, typename V2<R>::T* __restrict__ r,
                                                         typename V2<R>::T* __restrict__ z, const typename V2<R>::T* __restrict__ p,
                                                         const typename V2<R>::T* __restrict__ q, const typename V2<R>::T* __restrict__ minv,
                                                         double2* __restrict__ partial) {
    typedef typename V2<R>::T T;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 rz = make_double2(0, 0), rr = make_double2(0, 0);
    if (i < h && st[sys_of_row(pg, h, i, S, s)].active) {
        double2 al = st[sys_of_row(pg, h, i, S, s)].alpha;
        R ar = (R)al.x, ai = (R)al.y;
        T rv2[2];
#pragma unroll
        for (int half = 0; half < 2; half++) {
            long long k = (i + half * h) * S + s;
            T pv = p[k], qv = q[k], xv = x[k], rv = r[k];
            xv.x += ar * pv.x - ai * pv.y; xv.y += ar * pv.y + ai * pv.x;
            rv.x -= ar * qv.x - ai * qv.y; rv.y -= ar * qv.y + ai * qv.x;
            x[k] = xv; r[k] = rv; rv2[half] = rv;
        }
        T zl, zh;
        apply_pair<R>(precond, minv, S, i, s, rv2[0], rv2[1], zl, zh);
        z[i * S + s] = zl; z[(i + h) * S + s] = zh;
        double2 a = dotu(rv2[0], zl), b = dotu(rv2[1], zh);
        rz = make_double2(a.x + b.x, a.y + b.y);
        rr.x = nrm2(rv2[0]) + nrm2(rv2[1]);
    }
    block_store2(rz, rr, 2, S, partial);
}

template <typename R>
__global__ void cocg_pupdate_kernel(long long n, int S, const int* __restrict__ pg, const SysState* __restrict__ st,
                                    const typename V2<R>::T* __restrict__ z, typename V2<R>::T* __restrict__ p) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    const int sy = sys_of_row(pg, n / 2, g / S, S, (int)(g % S));
    if (!st[sy].active) return;
    double2 b = st[sy].beta;
    R br = (R)b.x, bi = (R)b.y;
    typename V2<R>::T zv = z[g], pv = p[g];
    p[g] = mk2<R>(zv.x + br * pv.x - bi * pv.y, zv.y + br * pv.y + bi * pv.x);
}

// ---- BiCGStab vector kernels ----
// r_hat = r, p = v = 0, partial (r_hat, r) = ||r||^2
template <typename R>
__global__ void __launch_bounds__(VB) bicg_init_kernel(long long n, int S, const typename V2<R>::T* __restrict__ r,
                                                       typename V2<R>::T* __restrict__ rh, typename V2<R>::T* __restrict__ p,
                                                       typename V2<R>::T* __restrict__ v, double2* __restrict__ partial) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    double2 c = make_double2(0, 0);
    if (g < n * S) {
        typename V2<R>::T rv = r[g];
        rh[g] = rv;
        p[g] = mk2<R>(0, 0);
        v[g] = mk2<R>(0, 0);
        c.x = nrm2(rv);
    }
    block_store2(c, c, 1, S, partial);
}

// p = r + beta (p - omega v); p_hat = M^-1 p   (thread per DOF pair)
template <typename R>
__global__ void __launch_bounds__(VB) bicg_p_kernel(long long h, int S, int precond, const int* __restrict__ pg,
                                                    const SysState* __restrict__ st,
                                                    const typename V2<R>::T* __restrict__ r, typename V2<R>::T* __restrict__ p,
                                                    const typename V2<R>::T* __restrict__ v, typename V2<R>::T* __restrict__ ph,
                                                    const typename V2<R>::T* __restrict__ minv, typename V2<R>::T* __restrict__ rh) {
    typedef typename V2<R>::T T;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    if (i >= h) return;
    const int sy = sys_of_row(pg, h, i, S, s);
    if (!st[sy].active) return;
    double2 b = st[sy].beta, w = st[sy].omega;
    R br = (R)b.x, bi = (R)b.y, wr = (R)w.x, wi = (R)w.y;
    if (st[sy].restart) {
        rh[i * S + s] = r[i * S + s];
        rh[(i + h) * S + s] = r[(i + h) * S + s];
    }
    T pn[2];
#pragma unroll
    for (int half = 0; half < 2; half++) {
        long long k = (i + half * h) * S + s;
        T rv = r[k], pv = p[k], vv = v[k];
        R tr = pv.x - (wr * vv.x - wi * vv.y), ti = pv.y - (wr * vv.y + wi * vv.x);
        pn[half] = mk2<R>(rv.x + br * tr - bi * ti, rv.y + br * ti + bi * tr);
        p[k] = pn[half];
    }
    T zl, zh;
    apply_pair<R>(precond, minv, S, i, s, pn[0], pn[1], zl, zh);
    ph[i * S + s] = zl;
    ph[(i + h) * S + s] = zh;
}

// s = r - alpha v (stored in r); s_hat = M^-1 s
template <typename R>
__global__ void __launch_bounds__(VB) bicg_s_kernel(long long h, int S, int precond, const int* __restrict__ pg,
                                                    const SysState* __restrict__ st,
                                                    typename V2<R>::T* __restrict__ r, const typename V2<R>::T* __restrict__ v,
                                                    typename V2<R>::T* __restrict__ sh, const typename V2<R>::T* __restrict__ minv) {
    typedef typename V2<R>::T T;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    if (i >= h) return;
    if (!st[sys_of_row(pg, h, i, S, s)].active) return;
    double2 a = st[sys_of_row(pg, h, i, S, s)].alpha;
    R ar = (R)a.x, ai = (R)a.y;
    T sn[2];
#pragma unroll
    for (int half = 0; half < 2; half++) {
        long long k = (i + half * h) * S + s;
        T rv = r[k], vv = v[k];
        sn[half] = mk2<R>(rv.x - (ar * vv.x - ai * vv.y), rv.y - (ar * vv.y + ai * vv.x));
        r[k] = sn[half];
    }
    T zl, zh;
    apply_pair<R>(precond, minv, S, i, s, sn[0], sn[1], zl, zh);
    sh[i * S + s] = zl;
    sh[(i + h) * S + s] = zh;
}

// x += alpha p_hat + omega s_hat; r = s - omega t; partial (r_hat, r) and ||r||^2
template <typename R>
__global__ void __launch_bounds__(VB) bicg_x_kernel(long long n, int S, const int* __restrict__ pg,
                                                    const SysState* __restrict__ st,
                                                    typename V2<R>::T* __restrict__ x, typename V2<R>::T* __restrict__ r,
                                                    const typename V2<R>::T* __restrict__ ph, const typename V2<R>::T* __restrict__ sh,
                                                    const typename V2<R>::T* __restrict__ t, const typename V2<R>::T* __restrict__ rh,
                                                    double2* __restrict__ partial) {
    typedef typename V2<R>::T T;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    double2 c0 = make_double2(0, 0), c1 = c0;
    const int sy = g < n * S ? sys_of_row(pg, n / 2, g / S, S, (int)(g % S)) : 0;
    if (g < n * S && st[sy].active) {
        double2 a = st[sy].alpha, w = st[sy].omega;
        R ar = (R)a.x, ai = (R)a.y, wr = (R)w.x, wi = (R)w.y;
        T xv = x[g], pv = ph[g], sv = sh[g], rv = r[g], tv = t[g];
        xv.x += ar * pv.x - ai * pv.y + wr * sv.x - wi * sv.y;
        xv.y += ar * pv.y + ai * pv.x + wr * sv.y + wi * sv.x;
        rv.x -= wr * tv.x - wi * tv.y;
        rv.y -= wr * tv.y + wi * tv.x;
        x[g] = xv;
        r[g] = rv;
        c0 = dotc(rh[g], rv);
        c1.x = nrm2(rv);
    }
    block_store2(c0, c1, 2, S, partial);
}

// ---- setup kernels -------------------------------------------------------------------
__global__ void mask_vec_kernel(long long n, int S, const uint8_t* mask, double2* v) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    if (!mask[g / S]) v[g] = make_double2(0, 0);
}

// r = b - Ax on free DOFs; partials ||b||^2 and ||r||^2
__global__ void __launch_bounds__(VB) residual_kernel(long long n, int S, const uint8_t* __restrict__ mask,
                                                       const double2* __restrict__ b, const double2* __restrict__ Ax,
                                                       double2* __restrict__ r, double2* __restrict__ partial) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    double2 cb = make_double2(0, 0), cr = cb;
    if (g < n * S) {
        long long i = g / S;
        double2 res = make_double2(0, 0);
        if (mask[i]) {
            double2 bv = b[g], av = Ax[g];
            res = make_double2(bv.x - av.x, bv.y - av.y);
            cb.x = bv.x * bv.x + bv.y * bv.y;
            cr.x = res.x * res.x + res.y * res.y;
        }
        r[g] = res;
    }
    block_store2(cb, cr, 2, S, partial);
}

// Operator entry (row, col) of system s (E - k0^2 B + patch), used by the preconditioner setup.
__device__ __forceinline__ double2 row_value(const OpArgs& a, long long row, long long col, int sy) {
    const double2* Ev = (const double2*)a.E;
    const double2* Bv = (const double2*)a.B;
    int lo = a.indptr[row], hi = a.indptr[row + 1] - 1;
    double2 v = make_double2(0, 0);
    if (hi >= lo) {
        while (lo < hi) { int mid = (lo + hi) >> 1; if (a.indices[mid] < col) lo = mid + 1; else hi = mid; }
        if (a.indices[lo] == col) {
            double2 e = Ev[lo];
            double k2 = a.k0sq[sy];
            v = e;
            if (Bv) { double2 b = Bv[lo]; v.x -= k2 * b.x; v.y -= k2 * b.y; }
        }
    }
    int pr = a.patch_of_row ? a.patch_of_row[row] : -1;
    if (pr >= 0) {
        const double2* Pv = (const double2*)a.patch_vals;
        for (int j = a.patch_rowptr[pr]; j < a.patch_rowptr[pr + 1]; j++) {
            if (a.patch_cols[j] != col) continue;
            int q = a.patch_port[j];
            double gr = a.gamma[2 * (sy * a.n_ports + q)], gi = a.gamma[2 * (sy * a.n_ports + q) + 1];
            double2 pv = Pv[j];
            v.x += gr * pv.x - gi * pv.y;
            v.y += gr * pv.y + gi * pv.x;
        }
    }
    return v;
}

// Inverse 2x2 pair blocks (precond 2) or inverse diagonals (precond 1); op is the FP64 operator.
template <typename R>
__global__ void precond_setup_kernel(OpArgs a, int precond, typename V2<R>::T* __restrict__ minv) {
    long long h = a.n / 2;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    int S = a.S;
    if (g >= h * S) return;
    long long i = g / S;
    int s = (int)(g % S);
    long long j = i + h;
    const int sy = sys_of_row(a.pg, h, i, S, s);
    double2 m00 = make_double2(0, 0), m01 = m00, m10 = m00, m11 = m00;
    bool fi = a.mask[i] != 0, fj = a.mask[j] != 0;
    double2 a00 = fi ? row_value(a, i, i, sy) : make_double2(1, 0);
    double2 a11 = fj ? row_value(a, j, j, sy) : make_double2(1, 0);
    double2 a01 = (fi && fj) ? row_value(a, i, j, sy) : make_double2(0, 0);
    double2 a10 = (fi && fj) ? row_value(a, j, i, sy) : make_double2(0, 0);
    auto inv1 = [](double2 v) { return cabs1(v) > 0 ? cdiv2(make_double2(1, 0), v) : make_double2(1, 0); };
    bool done = false;
    if (precond == 2) {
        double2 det = make_double2(a00.x * a11.x - a00.y * a11.y - (a01.x * a10.x - a01.y * a10.y),
                                   a00.x * a11.y + a00.y * a11.x - (a01.x * a10.y + a01.y * a10.x));
        double sc = cabs1(a00) * cabs1(a11);
        if (cabs1(det) > 1e-12 * sc && isfinite(cabs1(det))) {
            double2 id = cdiv2(make_double2(1, 0), det);
            m00 = cmul2(a11, id);
            m11 = cmul2(a00, id);
            m01 = cmul2(make_double2(-a01.x, -a01.y), id);
            m10 = cmul2(make_double2(-a10.x, -a10.y), id);
            done = true;
        }
    }
    if (!done) { m00 = inv1(a00); m11 = inv1(a11); }
    typename V2<R>::T* m = minv + (i * S + s) * 4;
    m[0] = mk2<R>((R)m00.x, (R)m00.y); m[1] = mk2<R>((R)m01.x, (R)m01.y);
    m[2] = mk2<R>((R)m10.x, (R)m10.y); m[3] = mk2<R>((R)m11.x, (R)m11.y);
}

// conversions / scaled copies for the mixed-precision refinement
// scale[q] = ||r_q|| of every system (grouped: G S of them)
__global__ void state_scale_kernel(int GS, const SysState* __restrict__ st64, double* __restrict__ scale) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < GS) scale[q] = sqrt(st64[q].rn2);
}

__global__ void to_f32_scaled_kernel(long long n, int S, const int* __restrict__ pg, const double2* __restrict__ src,
                                     const double* __restrict__ scale, float2* __restrict__ dst) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    double rn = scale[sys_of_row(pg, n / 2, g / S, S, (int)(g % S))];
    double sc = rn > 0 ? 1.0 / rn : 0.0;
    double2 v = src[g];
    dst[g] = make_float2((float)(v.x * sc), (float)(v.y * sc));
}

__global__ void add_scaled_f32_kernel(long long n, int S, const int* __restrict__ pg, const float2* __restrict__ d,
                                      const double* __restrict__ scale, const SysState* __restrict__ outer,
                                      double2* __restrict__ x) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    const int sy = sys_of_row(pg, n / 2, g / S, S, (int)(g % S));
    if (!outer[sy].active) return;
    double sc = scale[sy];
    float2 v = d[g];
    x[g].x += sc * (double)v.x;
    x[g].y += sc * (double)v.y;
}

__global__ void cast_values_kernel(long long nnz, const double2* __restrict__ src, float2* __restrict__ dst) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g < nnz) dst[g] = make_float2((float)src[g].x, (float)src[g].y);
}

// inner state for one refinement step: unit-norm rhs, relative tolerance `itol`, active = outer active
__global__ void inner_init_kernel(SysState* inner, const SysState* outer, int GS, double itol) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= GS) return;
    SysState z;
    z.rho = z.alpha = z.beta = z.omega = make_double2(0, 0);
    z.alpha.x = 1.0; z.omega.x = 1.0;
    z.active = outer[s].active;
    z.bn2 = z.active ? 1.0 : 0.0;
    z.rn2 = z.bn2;
    z.tol2 = itol * itol;
    z.iters = 0; z.status = 0; z.restart = 0; z.rh2 = 0;
    inner[s] = z;
}

__global__ void patch_map_kernel(long long np, const int* rows, int* patch_of_row) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g < np) patch_of_row[rows[g]] = (int)g;
}

void launch_patch_map(long long np, const int* rows, int* pmap, cudaStream_t s) {
    patch_map_kernel<<<grid_for(np, VB), VB, 0, s>>>(np, rows, pmap);
}

__global__ void pad_copy_kernel(long long n, int nsys, int S, const double2* __restrict__ src, double2* __restrict__ dst) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    long long i = g / S;
    int s = (int)(g % S);
    dst[g] = s < nsys ? src[i * nsys + s] : make_double2(0, 0);
}

__global__ void unpad_copy_kernel(long long n, int nsys, int S, const double2* __restrict__ src, double2* __restrict__ dst) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * nsys) return;
    long long i = g / nsys;
    int s = (int)(g % nsys);
    dst[g] = src[i * S + s];
}

__global__ void combine_kernel(long long nnz, const double2* __restrict__ E, const double2* __restrict__ B, double k0sq,
                               double2* __restrict__ K) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= nnz) return;
    double2 e = E[g], b = B[g];
    // (E - (B k0^2)) with the product rounded first, as the reference's E - B*k0**2
    double bx = __dmul_rn(b.x, k0sq), by = __dmul_rn(b.y, k0sq);
    K[g] = make_double2(__dsub_rn(e.x, bx), __dsub_rn(e.y, by));
}

__global__ void patch_add_kernel(long long np, const int* __restrict__ slot, const double2* __restrict__ vals,
                                 double gr, double gi, double2* __restrict__ K) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= np) return;
    double2 v = vals[g];
    int s = slot[g];
    K[s].x += gr * v.x - gi * v.y;
    K[s].y += gr * v.y + gi * v.x;
}

static int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ---- workspace layout ----------------------------------------------------------------------
struct Layout {
    size_t off_state, off_gamma, off_k0, off_partial, off_patchmap, off_scale, off_gblk;
    size_t off_x, off_b, off_r64, off_Ax;                  // FP64 vectors (n, S)
    size_t off_v[8];                                       // Krylov vectors of the inner precision
    size_t off_minv;
    size_t total;
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static Layout make_layout(long long n, long long nnz, long long npatch, int S, int nports, int precision, int G = 1) {
    Layout L;
    size_t o = 0;
    long long nb = (n * S + VB - 1) / VB + 1;
    size_t vec64 = (size_t)n * S * sizeof(double2);
    size_t vecw = (size_t)n * S * (precision ? sizeof(float2) : sizeof(double2));
    L.off_state = o; o = align256(o + sizeof(SysState) * 2 * S * G);
    L.off_gamma = o; o = align256(o + sizeof(double) * 2 * S * G * (nports > 0 ? nports : 1));
    L.off_k0 = o; o = align256(o + sizeof(double) * S * G);
    L.off_partial = o; o = align256(o + sizeof(double2) * 3 * nb * S);
    L.off_patchmap = o; o = align256(o + sizeof(int) * n);
    L.off_scale = o; o = align256(o + sizeof(double) * S * G);
    L.off_gblk = o; o = align256(o + sizeof(int) * (G + 1));
    L.off_x = o; o = align256(o + vec64);
    L.off_b = o; o = align256(o + vec64);
    L.off_r64 = o; o = align256(o + vec64);
    L.off_Ax = o; o = align256(o + vec64);
    for (int k = 0; k < 8; k++) { L.off_v[k] = o; o = align256(o + vecw); }
    L.off_minv = o; o = align256(o + vecw * 2);  // (n/2) * S * 4 entries
    (void)nnz; (void)npatch;
    L.total = o;
    return L;
}

// Batched Krylov solve in precision R from x = 0 with the initial residual already in r and the
// per-system state (bn2, tol2, active) in st.
template <typename R>
struct Krylov {
    typedef typename V2<R>::T T;
    int method = 1;            // 0 COCG, 1 BiCGStab
    OpArgs op;
    long long n = 0, h = 0;
    int S = 1, precond = 2, maxit = 1000, nsys = 1;
    T *x = nullptr, *r = nullptr, *minv = nullptr;
    T* v[7] = {nullptr};       // work vectors
    double2* partial = nullptr;
    SysState* st = nullptr;
    cudaStream_t s = nullptr;
    // grouped systems: G groups of S systems, group of every DOF pair, group block ranges
    int G = 1;
    const int* pg = nullptr;
    const int* gblk = nullptr;
    // auxiliary-space correction (precond 3: aux Jacobi, 4: learned network); BiCGStab only
    const emfem_aux_s* aux = nullptr;
    T* adinv = nullptr;
    // multifrontal LU of one system's operator (precond 5): M^-1 for every system of the batch
    emfem_mf_s* mf = nullptr;
    int bj() const { return precond == 5 ? 0 : (precond >= 3 ? 2 : precond); }

    unsigned nb_all() const { return grid_for(n * (long long)S, VB); }
    unsigned nb_pair() const { return grid_for(h * (long long)S, VB); }

    // restart BiCGStab's shadow residual only when (r_hat, r) is at the rounding level of the
    // vectors' precision (the dots accumulate in FP64); a looser FP32 threshold restarts so often
    // that the Krylov memory is lost
    double restart_eps = sizeof(R) == 8 ? 1e-9 : 1e-6;
    void reduce(int ncomp, unsigned nblocks, int mode) {
        reduce_update_kernel<<<G * S, VB, 0, s>>>(partial, (int)nblocks, S, ncomp, st, mode, maxit, restart_eps, nsys, G,
                                                  gblk, nblocks != nb_pair() ? 1 : 0, (int)nb_pair());
    }

    int start() {
        if (method == 0) {
            T *z = v[0], *p = v[1];
            cocg_init_kernel<R><<<nb_pair(), VB, 0, s>>>(h, S, precond, r, z, p, minv, partial);
            reduce(1, nb_pair(), UPD_SET_RHO);
        } else {
            T *rh = v[0], *p = v[1], *vv = v[2];
            bicg_init_kernel<R><<<nb_all(), VB, 0, s>>>(n, S, r, rh, p, vv, partial);
            reduce(1, nb_all(), UPD_SET_RHO);
        }
        return check_cuda(cudaGetLastError(), "krylov start");
    }

    int iteration() {
        if (method == 0) {
            T *z = v[0], *p = v[1], *q = v[2];
            spmv_kernel<R><<<nb_all(), VB, 0, s>>>(op, p, q, partial, DOT_XY, nullptr);
            reduce(1, nb_all(), UPD_COCG_ALPHA);
            cocg_update_kernel<R><<<nb_pair(), VB, 0, s>>>(h, S, precond, pg, st, x, r, z, p, q, minv, partial);
            reduce(2, nb_pair(), UPD_COCG_BETA);
            cocg_pupdate_kernel<R><<<nb_all(), VB, 0, s>>>(n, S, pg, st, z, p);
        } else {
            T *rh = v[0], *p = v[1], *vv = v[2], *ph = v[3], *sh = v[4], *t = v[5];
            bicg_p_kernel<R><<<nb_pair(), VB, 0, s>>>(h, S, bj(), pg, st, r, p, vv, ph, minv, rh);
            if (aux) EMFEM_TRY(aux_correct<T>(aux, S, precond == 4, adinv, p, op.mask, ph, s));
            if constexpr (sizeof(R) == 8) {
                if (mf) EMFEM_TRY(mf_apply(mf, S, (const double2*)p, (double2*)ph, s));
            }
            spmv_kernel<R><<<nb_all(), VB, 0, s>>>(op, ph, vv, partial, DOT_CONJW_Y, rh);
            reduce(1, nb_all(), UPD_BICG_ALPHA);
            bicg_s_kernel<R><<<nb_pair(), VB, 0, s>>>(h, S, bj(), pg, st, r, vv, sh, minv);
            if (aux) EMFEM_TRY(aux_correct<T>(aux, S, precond == 4, adinv, r, op.mask, sh, s));
            if constexpr (sizeof(R) == 8) {
                if (mf) EMFEM_TRY(mf_apply(mf, S, (const double2*)r, (double2*)sh, s));
            }
            spmv_kernel<R><<<nb_all(), VB, 0, s>>>(op, sh, t, partial, DOT_CONJY_W_YY, r);
            reduce(3, nb_all(), UPD_BICG_OMEGA);
            bicg_x_kernel<R><<<nb_all(), VB, 0, s>>>(n, S, pg, st, x, r, ph, sh, t, rh, partial);
            reduce(2, nb_all(), UPD_BICG_RHO);
        }
        return check_cuda(cudaGetLastError(), "krylov iteration");
    }

    // one eager iteration (loads every kernel before capture), then `chunk` iterations captured once
    // and replayed until no system is active or the iteration cap is reached
    int run(int chunk) {
        EMFEM_TRY(iteration());
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        EMFEM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st_cap = EMFEM_OK;
        for (int k = 0; k < chunk && st_cap == EMFEM_OK; k++) st_cap = iteration();
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st_cap != EMFEM_OK) { if (graph) cudaGraphDestroy(graph); return st_cap; }
        EMFEM_CUDA(e);
        EMFEM_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        std::vector<SysState> host((size_t)G * S);
        int rounds = (maxit + chunk - 1) / chunk + 1;
        int rc = EMFEM_OK;
        for (int it = 0; it < rounds; it++) {
            if ((rc = check_cuda(cudaGraphLaunch(exec, s), "cudaGraphLaunch")) != EMFEM_OK) break;
            if ((rc = check_cuda(cudaMemcpyAsync(host.data(), st, sizeof(SysState) * host.size(), cudaMemcpyDeviceToHost, s), "copy state")) != EMFEM_OK) break;
            if ((rc = check_cuda(cudaStreamSynchronize(s), "sync")) != EMFEM_OK) break;
            bool any = false;
            for (size_t k = 0; k < host.size(); k++) any |= host[k].active != 0;
            if (!any) break;
        }
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return rc;
    }
};

}  // namespace emfem

using namespace emfem;

static void build_op(OpArgs& a, int64_t n, int S, const int32_t* indptr, const int32_t* indices, const void* E,
                     const void* B, const double* k0dev, const int* pmap, const int32_t* prowptr, const int32_t* pcols,
                     const void* pvals, const int32_t* pport, int nports, const double* gdev, const uint8_t* mask) {
    a.n = n; a.S = S; a.indptr = indptr; a.indices = indices; a.E = E; a.B = B; a.k0sq = k0dev;
    a.patch_of_row = pmap; a.patch_rowptr = prowptr; a.patch_cols = pcols; a.patch_vals = pvals; a.patch_port = pport;
    a.n_ports = nports; a.gamma = gdev; a.mask = mask;
    a.pg = nullptr; a.hh = n / 2; a.skip = nullptr;
}

extern "C" {

int emfem_krylov_workspace_size(int64_t n, int64_t nnz, int nsys, int precision, size_t* bytes) {
    EMFEM_REQUIRE(bytes && n > 0 && nsys > 0 && nsys <= 64 && nnz >= 0, "emfem_krylov_workspace_size: bad argument");
    EMFEM_REQUIRE(precision == 0 || precision == 1, "emfem_krylov_workspace_size: precision must be 0 or 1");
    int S = pow2_at_least(nsys);
    Layout L = make_layout(n, nnz, nnz, S, 8, precision);
    *bytes = L.total;
    return EMFEM_OK;
}

int emfem_sweep_combine(emfem_handle h, int64_t nnz, const void* E_vals, const void* B_vals, double k0sq,
                        int64_t n_patch, const int32_t* patch_slot, const void* patch_vals,
                        double gamma_re, double gamma_im, void* K_vals) {
    EMFEM_REQUIRE(h && E_vals && B_vals && K_vals && nnz >= 0, "emfem_sweep_combine: bad argument");
    EMFEM_REQUIRE(n_patch == 0 || (patch_slot && patch_vals), "emfem_sweep_combine: patch arrays missing");
    if (nnz > 0) {
        combine_kernel<<<grid_for(nnz, VB), VB, 0, h->h.stream>>>(nnz, (const double2*)E_vals, (const double2*)B_vals,
                                                                  k0sq, (double2*)K_vals);
        EMFEM_LAUNCH("combine_kernel");
    }
    if (n_patch > 0) {
        patch_add_kernel<<<grid_for(n_patch, VB), VB, 0, h->h.stream>>>(n_patch, patch_slot, (const double2*)patch_vals,
                                                                        gamma_re, gamma_im, (double2*)K_vals);
        EMFEM_LAUNCH("patch_add_kernel");
    }
    return EMFEM_OK;
}

int emfem_sweep_spmv(emfem_handle h, int64_t n, const int32_t* indptr, const int32_t* indices,
                     const void* E_vals, const void* B_vals, int nsys, const double* k0sq_dev,
                     int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                     const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                     int n_ports, const double* gamma_dev, const uint8_t* free_mask, const void* x, void* y) {
    EMFEM_REQUIRE(h && indptr && indices && E_vals && k0sq_dev && free_mask && x && y && n > 0,
                  "emfem_sweep_spmv: bad argument");
    EMFEM_REQUIRE(nsys >= 1 && nsys <= 256 && (nsys & (nsys - 1)) == 0,
                  "emfem_sweep_spmv: nsys must be a power of two <= 256");
    EMFEM_REQUIRE(n_patch_rows == 0 || (patch_rows && patch_rowptr && patch_cols && patch_vals && patch_port && gamma_dev),
                  "emfem_sweep_spmv: patch arrays missing");
    int* pmap = nullptr;
    if (n_patch_rows > 0) {
        EMFEM_CUDA(cudaMallocAsync(&pmap, sizeof(int) * n, h->h.stream));
        EMFEM_CUDA(cudaMemsetAsync(pmap, 0xff, sizeof(int) * n, h->h.stream));
        patch_map_kernel<<<grid_for(n_patch_rows, VB), VB, 0, h->h.stream>>>(n_patch_rows, patch_rows, pmap);
        EMFEM_LAUNCH("patch_map_kernel");
    }
    OpArgs a;
    build_op(a, n, nsys, indptr, indices, E_vals, B_vals, k0sq_dev, pmap, patch_rowptr, patch_cols, patch_vals,
             patch_port, n_ports, gamma_dev, free_mask);
    spmv_kernel<double><<<grid_for(n * nsys, VB), VB, 0, h->h.stream>>>(a, (const double2*)x, (double2*)y, nullptr,
                                                                          DOT_NONE, nullptr);
    EMFEM_LAUNCH("spmv_kernel");
    if (pmap) EMFEM_CUDA(cudaFreeAsync(pmap, h->h.stream));
    return EMFEM_OK;
}

}  // extern "C"

// The batched solve behind emfem_krylov_solve (G = 1) and emfem_krylov_solve_grouped (G groups of
// nsys systems; row i of the (n, S) vectors belongs to group pair_group[i mod n/2]).
static int krylov_impl(emfem_handle hd, int method, int64_t n, int64_t nnz, const int32_t* indptr, const int32_t* indices,
                       const void* E_vals, const void* B_vals, int nsys, const double* k0sq,
                       int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                       const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                       int n_ports, const double* gamma, const uint8_t* free_mask, const void* rhs, void* x,
                       double tol, int maxit, int precond, int precision, void* workspace, size_t workspace_bytes,
                       int* status, int* iters, double* relres, emfem_aux aux, int G, const int32_t* pair_group,
                       emfem_mf_s* mf = nullptr) {
    EMFEM_REQUIRE(hd && indptr && indices && E_vals && k0sq && free_mask && rhs && x && workspace,
                  "emfem_krylov_solve: null argument");
    EMFEM_REQUIRE((precond == 5) == (mf != nullptr), "emfem_krylov_solve: the LU preconditioner goes with precond 5");
    EMFEM_REQUIRE(precond != 5 || (method == 1 && precision == 0 && G == 1),
                  "emfem_krylov_solve_lu: FP64 BiCGStab on one group only");
    EMFEM_REQUIRE(method == 0 || method == 1, "emfem_krylov_solve: method must be 0 (COCG) or 1 (BiCGStab)");
    EMFEM_REQUIRE(n > 0 && (n % 2) == 0, "emfem_krylov_solve: n must be even (DOF pairs i, i + n/2)");
    EMFEM_REQUIRE(nsys >= 1 && nsys <= 64, "emfem_krylov_solve: 1 <= nsys <= 64");
    EMFEM_REQUIRE(precond >= 0 && precond <= 5 && (precision == 0 || precision == 1), "emfem_krylov_solve: bad option");
    EMFEM_REQUIRE(precond < 3 || precond == 5 || (aux && method == 1 && aux->n == n && aux->have_operator && aux->nports == n_ports),
                  "emfem_krylov_solve: precond 3/4 need BiCGStab and an aux space of this field with its operator "
                  "set (emfem_aux_set_operator, same ports)");
    EMFEM_REQUIRE(precond != 4 || aux->params, "emfem_krylov_solve: precond 4 needs network parameters (emfem_aux_set_network)");
    EMFEM_REQUIRE(precond < 3 || precond == 5 || aux->ngroups == G,
                  "emfem_krylov_solve: the aux space's groups (emfem_aux_set_rows) must match the solve's groups");
    EMFEM_REQUIRE(n_ports >= 0 && n_ports <= 8, "emfem_krylov_solve: at most 8 ports");
    EMFEM_REQUIRE(n_patch_rows == 0 || (patch_rows && patch_rowptr && patch_cols && patch_vals && patch_port && gamma),
                  "emfem_krylov_solve: patch arrays missing");
    EMFEM_REQUIRE(tol > 0 && maxit > 0, "emfem_krylov_solve: tol and maxit must be positive");
    Handle* h = &hd->h;
    int S = pow2_at_least(nsys);
    int64_t npatch = 0;
    if (n_patch_rows > 0) {
        int32_t last = 0;
        EMFEM_CUDA(cudaMemcpy(&last, patch_rowptr + n_patch_rows, sizeof(int32_t), cudaMemcpyDeviceToHost));
        npatch = last;
    }
    EMFEM_REQUIRE(npatch <= nnz, "emfem_krylov_solve: more patch entries than nnz");
    EMFEM_REQUIRE(precond != 5 || mf_reserved(mf) >= S,
                  "emfem_krylov_solve_lu: call emfem_mf_reserve with at least the padded batch size first");
    EMFEM_REQUIRE(precond < 3 || precond == 5 || aux->kbuf_bytes >= aux_solve_bytes(aux, S),
                  "emfem_krylov_solve: call emfem_aux_reserve with at least nsys systems first");
    std::vector<int> hgblk(G + 1, 0);
    if (G > 1) {
        EMFEM_REQUIRE(pair_group, "emfem_krylov_solve_grouped: pair_group required");
        EMFEM_REQUIRE((n / 2) % VB == 0, "emfem_krylov_solve_grouped: n/2 must be a multiple of 256");
        std::vector<int> hp(n / 2);
        EMFEM_CUDA(cudaMemcpy(hp.data(), pair_group, sizeof(int) * (n / 2), cudaMemcpyDeviceToHost));
        // groups 0..G-1 in ascending order, none empty, each starting at a multiple of 256 pairs
        int prev = -1;
        for (long long i = 0; i < n / 2; i++) {
            int v = hp[i];
            if (v == prev) continue;
            EMFEM_REQUIRE(v == prev + 1 && v < G && i % VB == 0,
                          "emfem_krylov_solve_grouped: pair_group must run through 0..G-1 in order, each group "
                          "starting at a multiple of 256 pairs");
            hgblk[v] = (int)(i * S / VB);
            prev = v;
        }
        EMFEM_REQUIRE(prev == G - 1, "emfem_krylov_solve_grouped: every group needs at least one DOF pair");
        hgblk[G] = (int)((n / 2) * S / VB);
    }
    Layout L = make_layout(n, nnz, npatch, S, n_ports, precision, G);
    size_t need = make_layout(n, nnz, nnz, S, 8, precision, G).total;
    if (workspace_bytes < need) {
        set_error("emfem_krylov_solve: workspace of %zu bytes, %zu needed (emfem_krylov_workspace_size)", workspace_bytes, need);
        return EMFEM_ERR_WORKSPACE;
    }
    char* ws = (char*)workspace;
    cudaStream_t s = nullptr;
    EMFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(s);
        set_error("emfem_krylov_solve: cudaEventCreate failed");
        return EMFEM_ERR_CUDA;
    }
    SysState* st = (SysState*)(ws + L.off_state);
    SysState* st_outer = st + (size_t)G * S;
    int* gblk = (int*)(ws + L.off_gblk);
    const int nbh = (int)grid_for((n / 2) * (long long)S, VB);
    double* gdev = (double*)(ws + L.off_gamma);
    double* k0dev = (double*)(ws + L.off_k0);
    double2* partial = (double2*)(ws + L.off_partial);
    int* pmap = (int*)(ws + L.off_patchmap);
    double* scale = (double*)(ws + L.off_scale);
    double2* x64 = (double2*)(ws + L.off_x);
    double2* b64 = (double2*)(ws + L.off_b);
    double2* r64 = (double2*)(ws + L.off_r64);
    double2* Ax = (double2*)(ws + L.off_Ax);
    long long nS = n * (long long)S;
    unsigned gv = grid_for(nS, VB);
    std::vector<double> hk0((size_t)G * S, 0.0), hg(2 * (size_t)G * S * (n_ports > 0 ? n_ports : 1), 0.0);
    for (int g = 0; g < G; g++)
        for (int k = 0; k < nsys; k++) {
            hk0[g * S + k] = k0sq[g * nsys + k];
            for (int q = 0; q < n_ports; q++) {
                hg[2 * ((g * S + k) * n_ports + q)] = gamma[2 * ((g * nsys + k) * n_ports + q)];
                hg[2 * ((g * S + k) * n_ports + q) + 1] = gamma[2 * ((g * nsys + k) * n_ports + q) + 1];
            }
        }
    OpArgs op64;
    int rc = EMFEM_OK;
#define STRY(x) do { rc = (x); if (rc != EMFEM_OK) goto done; } while (0)
    STRY(check_cuda(cudaEventRecord(ev, h->stream), "event"));
    STRY(check_cuda(cudaStreamWaitEvent(s, ev, 0), "wait"));
    STRY(check_cuda(cudaMemcpyAsync(k0dev, hk0.data(), sizeof(double) * hk0.size(), cudaMemcpyHostToDevice, s), "copy k0"));
    STRY(check_cuda(cudaMemcpyAsync(gblk, hgblk.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, s), "copy gblk"));
    STRY(check_cuda(cudaMemcpyAsync(gdev, hg.data(), sizeof(double) * hg.size(), cudaMemcpyHostToDevice, s), "copy gamma"));
    STRY(check_cuda(cudaMemsetAsync(pmap, 0xff, sizeof(int) * n, s), "memset"));
    if (n_patch_rows > 0) {
        patch_map_kernel<<<grid_for(n_patch_rows, VB), VB, 0, s>>>(n_patch_rows, patch_rows, pmap);
        STRY(check_cuda(cudaGetLastError(), "patch_map_kernel"));
    }
    pad_copy_kernel<<<gv, VB, 0, s>>>(n, nsys, S, (const double2*)rhs, b64);
    pad_copy_kernel<<<gv, VB, 0, s>>>(n, nsys, S, (const double2*)x, x64);
    mask_vec_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, b64);
    mask_vec_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, x64);
    STRY(check_cuda(cudaGetLastError(), "setup copies"));
    build_op(op64, n, S, indptr, indices, E_vals, B_vals, k0dev, n_patch_rows ? pmap : nullptr, patch_rowptr,
             patch_cols, patch_vals, patch_port, n_ports, gdev, free_mask);
    if (G > 1) op64.pg = pair_group;
    // initial residual r64 = b - A x0 and the outer state (||b||, tolerance, active)
    spmv_kernel<double><<<gv, VB, 0, s>>>(op64, x64, Ax, nullptr, DOT_NONE, nullptr);
    residual_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial);
    reduce_update_kernel<<<G * S, VB, 0, s>>>(partial, (int)gv, S, 2, st_outer, UPD_INIT, maxit, tol, nsys, G, gblk, 1, nbh);
    STRY(check_cuda(cudaGetLastError(), "initial residual"));

    if (precision == 0) {
        Krylov<double> k;
        k.method = method; k.op = op64; k.n = n; k.h = n / 2; k.S = S; k.precond = precond; k.maxit = maxit; k.nsys = nsys;
        k.x = x64; k.r = (double2*)(ws + L.off_r64); k.minv = (double2*)(ws + L.off_minv);
        for (int q = 0; q < 7; q++) k.v[q] = (double2*)(ws + L.off_v[q]);
        k.partial = partial; k.st = st; k.s = s;
        k.op.skip = st;
        k.G = G; k.pg = G > 1 ? pair_group : nullptr; k.gblk = gblk;
        if (k.bj()) {
            precond_setup_kernel<double><<<grid_for((n / 2) * (long long)S, VB), VB, 0, s>>>(op64, k.bj(), k.minv);
            STRY(check_cuda(cudaGetLastError(), "precond_setup"));
        }
        if (precond == 3 || precond == 4) {
            k.aux = aux;
            k.adinv = (double2*)aux_dinv_buffer(aux, S);
            STRY(aux_setup_dinv<double2>(aux, S, nsys, k0dev, gdev, k.adinv, s));
        }
        k.mf = mf;
        // the recurrence tolerance is half the requested one so the FP64 true residual meets it
        reduce_update_kernel<<<G * S, VB, 0, s>>>(partial, (int)gv, S, 2, st, UPD_INIT, maxit, 0.5 * tol, nsys, G, gblk, 1,
                                                  nbh);
        STRY(check_cuda(cudaGetLastError(), "init state"));
        STRY(k.start());
        STRY(k.run(mf ? 2 : 16));     // an LU application is ~1000 launches: short captured chunks
    } else {
        OpArgs op32 = op64;  // FP64 values, FP32 vectors (see spmv_kernel)
        Krylov<float> k;
        k.method = method; k.op = op32; k.n = n; k.h = n / 2; k.S = S; k.precond = precond; k.nsys = nsys;
        float2* r32 = (float2*)(ws + L.off_v[6]);
        float2* d32 = (float2*)(ws + L.off_v[7]);
        k.x = d32; k.r = r32; k.minv = (float2*)(ws + L.off_minv);
        for (int q = 0; q < 6; q++) k.v[q] = (float2*)(ws + L.off_v[q]);
        k.partial = partial; k.st = st; k.s = s;
        k.op.skip = st;
        k.G = G; k.pg = G > 1 ? pair_group : nullptr; k.gblk = gblk;
        const int* pgk = k.pg;
        const size_t GSm = (size_t)G * S;
        if (precond) {
            precond_setup_kernel<float><<<grid_for((n / 2) * (long long)S, VB), VB, 0, s>>>(op64, k.bj(), k.minv);
            STRY(check_cuda(cudaGetLastError(), "precond_setup"));
        }
        if (precond >= 3) {
            k.aux = aux;
            k.adinv = (float2*)aux_dinv_buffer(aux, S);
            STRY(aux_setup_dinv<float2>(aux, S, nsys, k0dev, gdev, k.adinv, s));
        }
        std::vector<SysState> ho(GSm);
        int used = 0;
        for (int outer = 0; outer < 60; outer++) {
            STRY(check_cuda(cudaMemcpyAsync(ho.data(), st_outer, sizeof(SysState) * GSm, cudaMemcpyDeviceToHost, s), "copy"));
            STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
            bool any = false;
            for (size_t q = 0; q < GSm; q++) any |= ho[q].active != 0;
            if (!any || used >= maxit) break;
            state_scale_kernel<<<grid_for((long long)GSm, 64), 64, 0, s>>>((int)GSm, st_outer, scale);
            to_f32_scaled_kernel<<<gv, VB, 0, s>>>(n, S, pgk, r64, scale, r32);
            STRY(check_cuda(cudaMemsetAsync(d32, 0, sizeof(float2) * nS, s), "memset d"));
            inner_init_kernel<<<grid_for((long long)GSm, 64), 64, 0, s>>>(st, st_outer, (int)GSm, EMFEM_INNER_TOL);
            k.maxit = std::max(1, maxit - used);
            STRY(k.start());
            STRY(k.run(16));
            std::vector<SysState> hin(GSm);
            STRY(check_cuda(cudaMemcpyAsync(hin.data(), st, sizeof(SysState) * GSm, cudaMemcpyDeviceToHost, s), "copy"));
            STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
            int mx = 1;
            for (size_t q = 0; q < GSm; q++) if (ho[q].active) mx = std::max(mx, hin[q].iters);
            used += mx;
            add_scaled_f32_kernel<<<gv, VB, 0, s>>>(n, S, pgk, d32, scale, st_outer, x64);
            spmv_kernel<double><<<gv, VB, 0, s>>>(op64, x64, Ax, nullptr, DOT_NONE, nullptr);
            residual_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial);
            // the inner state array is free now: reuse it to reduce ||b||^2, ||r||^2 of the new residual
            reduce_update_kernel<<<G * S, VB, 0, s>>>(partial, (int)gv, S, 2, st, UPD_INIT, maxit, 1.0, S, G, gblk, 1, nbh);
            STRY(check_cuda(cudaGetLastError(), "refinement"));
            std::vector<SysState> hr(GSm);
            STRY(check_cuda(cudaMemcpyAsync(hr.data(), st, sizeof(SysState) * GSm, cudaMemcpyDeviceToHost, s), "copy"));
            STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
            // a correction that did not lower the FP64 residual is reverted and the system stops
            std::vector<double> rev(GSm, 0.0);
            bool any_rev = false;
            for (size_t q = 0; q < GSm; q++) {
                if (!ho[q].active) continue;
                ho[q].iters += hin[q].iters;
                double prev = ho[q].rn2;
                if (!std::isfinite(hr[q].rn2) || hr[q].rn2 >= prev) {
                    rev[q] = -std::sqrt(prev);
                    any_rev = true;
                    ho[q].active = 0; ho[q].status = 2;
                    continue;
                }
                ho[q].rn2 = hr[q].rn2;
                if (ho[q].rn2 <= ho[q].tol2) { ho[q].active = 0; ho[q].status = 0; }
                else if (ho[q].rn2 >= 0.98 * prev) { ho[q].active = 0; ho[q].status = 2; }
            }
            if (any_rev) {
                STRY(check_cuda(cudaMemcpyAsync(scale, rev.data(), sizeof(double) * GSm, cudaMemcpyHostToDevice, s), "copy"));
                add_scaled_f32_kernel<<<gv, VB, 0, s>>>(n, S, pgk, d32, scale, st_outer, x64);
                STRY(check_cuda(cudaGetLastError(), "revert"));
            }
            STRY(check_cuda(cudaMemcpyAsync(st_outer, ho.data(), sizeof(SysState) * GSm, cudaMemcpyHostToDevice, s), "copy"));
        }
        STRY(check_cuda(cudaMemcpyAsync(ho.data(), st_outer, sizeof(SysState) * GSm, cudaMemcpyDeviceToHost, s), "copy"));
        STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        for (size_t q = 0; q < GSm; q++) if (ho[q].active) { ho[q].active = 0; ho[q].status = 1; }
        STRY(check_cuda(cudaMemcpyAsync(st, ho.data(), sizeof(SysState) * GSm, cudaMemcpyHostToDevice, s), "copy"));
    }
    {
        // final FP64 true residual and solution copy-out
        const size_t GS = (size_t)G * S;
        std::vector<SysState> hs(GS);
        STRY(check_cuda(cudaMemcpyAsync(hs.data(), st, sizeof(SysState) * GS, cudaMemcpyDeviceToHost, s), "copy"));
        spmv_kernel<double><<<gv, VB, 0, s>>>(op64, x64, Ax, nullptr, DOT_NONE, nullptr);
        residual_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial);
        reduce_update_kernel<<<G * S, VB, 0, s>>>(partial, (int)gv, S, 2, st_outer, UPD_INIT, maxit, tol, S, G, gblk, 1, nbh);
        unpad_copy_kernel<<<grid_for(n * (long long)nsys, VB), VB, 0, s>>>(n, nsys, S, x64, (double2*)x);
        STRY(check_cuda(cudaGetLastError(), "final residual"));
        std::vector<SysState> hf(GS);
        STRY(check_cuda(cudaMemcpyAsync(hf.data(), st_outer, sizeof(SysState) * GS, cudaMemcpyDeviceToHost, s), "copy"));
        STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        bool all_ok = true;
        for (int g = 0; g < G; g++)
            for (int q = 0; q < nsys; q++) {
                const SysState &e = hs[g * S + q], &f = hf[g * S + q];
                double rel = f.bn2 > 0 ? std::sqrt(f.rn2 / f.bn2) : 0.0;
                int stat = e.active ? 1 : e.status;
                if (stat == 0 && rel > tol) stat = 1;  // the recurrence drifted from the true residual
                if (status) status[g * nsys + q] = stat;
                if (iters) iters[g * nsys + q] = e.iters;
                if (relres) relres[g * nsys + q] = rel;
                all_ok &= stat == 0;
            }
        if (!all_ok) {
            set_error("emfem_krylov_solve: not every system reached the tolerance");
            rc = EMFEM_ERR_NOT_CONVERGED;
        }
    }
done:
    cudaEventRecord(ev, s);
    cudaStreamWaitEvent(h->stream, ev, 0);
    cudaStreamSynchronize(s);
    cudaEventDestroy(ev);
    cudaStreamDestroy(s);
    return rc;
#undef STRY
}

extern "C" {

int emfem_krylov_solve(emfem_handle hd, int method, int64_t n, int64_t nnz, const int32_t* indptr, const int32_t* indices,
                       const void* E_vals, const void* B_vals, int nsys, const double* k0sq,
                       int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                       const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                       int n_ports, const double* gamma, const uint8_t* free_mask, const void* rhs, void* x,
                       double tol, int maxit, int precond, int precision, void* workspace, size_t workspace_bytes,
                       int* status, int* iters, double* relres, emfem_aux aux) {
    return krylov_impl(hd, method, n, nnz, indptr, indices, E_vals, B_vals, nsys, k0sq, n_patch_rows, patch_rows,
                       patch_rowptr, patch_cols, patch_vals, patch_port, n_ports, gamma, free_mask, rhs, x, tol, maxit,
                       precond, precision, workspace, workspace_bytes, status, iters, relres, aux, 1, nullptr);
}

int emfem_krylov_solve_lu(emfem_handle hd, int64_t n, int64_t nnz, const int32_t* indptr, const int32_t* indices,
                          const void* E_vals, const void* B_vals, int nsys, const double* k0sq, int64_t n_patch_rows,
                          const int32_t* patch_rows, const int32_t* patch_rowptr, const int32_t* patch_cols,
                          const void* patch_vals, const int32_t* patch_port, int n_ports, const double* gamma,
                          const uint8_t* free_mask, const void* rhs, void* x, double tol, int maxit, emfem_mf lu,
                          void* workspace, size_t workspace_bytes, int* status, int* iters, double* relres) {
    EMFEM_REQUIRE(lu, "emfem_krylov_solve_lu: no factorization");
    return krylov_impl(hd, 1, n, nnz, indptr, indices, E_vals, B_vals, nsys, k0sq, n_patch_rows, patch_rows,
                       patch_rowptr, patch_cols, patch_vals, patch_port, n_ports, gamma, free_mask, rhs, x, tol, maxit,
                       5, 0, workspace, workspace_bytes, status, iters, relres, nullptr, 1, nullptr, lu);
}

int emfem_krylov_workspace_size_grouped(int64_t n, int64_t nnz, int nsys, int ngroups, int precision, size_t* bytes) {
    EMFEM_REQUIRE(bytes && n > 0 && nsys > 0 && nsys <= 64 && nnz >= 0 && ngroups >= 1 && (precision == 0 || precision == 1),
                  "emfem_krylov_workspace_size_grouped: bad argument");
    *bytes = make_layout(n, nnz, nnz, pow2_at_least(nsys), 8, precision, ngroups).total;
    return EMFEM_OK;
}

int emfem_krylov_solve_grouped(emfem_handle hd, int method, int64_t n, int64_t nnz, const int32_t* indptr,
                               const int32_t* indices, const void* E_vals, const void* B_vals, int ngroups,
                               const int32_t* pair_group, int nsys, const double* k0sq, int64_t n_patch_rows,
                               const int32_t* patch_rows, const int32_t* patch_rowptr, const int32_t* patch_cols,
                               const void* patch_vals, const int32_t* patch_port, int n_ports, const double* gamma,
                               const uint8_t* free_mask, const void* rhs, void* x, double tol, int maxit, int precond,
                               int precision, void* workspace, size_t workspace_bytes, int* status, int* iters,
                               double* relres, emfem_aux aux) {
    EMFEM_REQUIRE(ngroups >= 1 && ngroups <= 4096, "emfem_krylov_solve_grouped: 1 <= ngroups <= 4096");
    return krylov_impl(hd, method, n, nnz, indptr, indices, E_vals, B_vals, nsys, k0sq, n_patch_rows, patch_rows,
                       patch_rowptr, patch_cols, patch_vals, patch_port, n_ports, gamma, free_mask, rhs, x, tol, maxit,
                       precond, precision, workspace, workspace_bytes, status, iters, relres, aux, ngroups, pair_group);
}

}  // extern "C"

// ---- allocation-free variant of emfem_sweep_spmv ------------------------------------------------
// Some callers cannot call cudaMalloc: applications that hand all device memory to their own pool
// allocator up front (a raw cudaMalloc fails or fragments it), and latency-critical loops in which an
// allocation's implicit device synchronisation is not acceptable.  This entry point computes exactly
// what emfem_sweep_spmv computes, but keeps its only scratch — the row -> Robin-patch-row map, one int
// per row — in the fixed array below instead of a stream-ordered allocation.  The array is part of
// this library's device image: every GPU that loads the library holds its 16 MiB until the process
// exits.  All calls share it and it keeps the last call's contents, so every call resets the rows it
// uses before filling them, and calls that overlap on the GPU (different streams or threads) race.
#include <mutex>

namespace emfem {
static __device__ __align__(256) int g_noalloc_patch_map[EMFEM_NOALLOC_MAX_ROWS];

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocSlot {
    int* addr = nullptr;
    unsigned long long ctx_id = 0;     // the context the address was resolved in (0 = unknown)
};
static NoallocSlot g_noalloc[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mutex;

// The current context's unique id through the driver's cuCtxGetCurrent / cuCtxGetId, looked up at run
// time (the library links only the CUDA runtime).  0 when no context is current or the lookup failed.
static unsigned long long current_ctx_id() {
    typedef int (*GetCurrentFn)(void** ctx);
    typedef int (*GetIdFn)(void* ctx, unsigned long long* id);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&get_current, 12000, cudaEnableDefault, &q1) !=
                cudaSuccess || q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&get_id, 12000, cudaEnableDefault, &q2) !=
                cudaSuccess || q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    }
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the static map on `device` (which must be current).  Resolved with
// cudaGetSymbolAddress once per device and context: host code only holds a host-side stand-in for the
// symbol, which must never be passed to a kernel.  A new context on the device (after cudaDeviceReset,
// the module is loaded again and the array may move) is seen by its id and resolves the address anew.
static int noalloc_scratch(int device, int** out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        set_error("emfem_sweep_spmv_noalloc: device %d beyond the supported %d", device, NOALLOC_MAX_DEVICES);
        return EMFEM_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocSlot& slot = g_noalloc[device];
    unsigned long long ctx = current_ctx_id();
    if (slot.addr == nullptr || ctx == 0 || ctx != slot.ctx_id) {
        int* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_patch_map);
        if (e != cudaSuccess) {
            set_error("emfem_sweep_spmv_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return EMFEM_ERR_CUDA;
        }
        slot.addr = p;
        slot.ctx_id = current_ctx_id();     // the lookup above made the device's context current
    }
    *out = slot.addr;
    return EMFEM_OK;
}
}  // namespace emfem

extern "C" int emfem_sweep_spmv_noalloc(emfem_handle h, int64_t n, const int32_t* indptr, const int32_t* indices,
                                        const void* E_vals, const void* B_vals, int nsys, const double* k0sq_dev,
                                        int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                                        const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                                        int n_ports, const double* gamma_dev, const uint8_t* free_mask,
                                        const void* x, void* y) {
    EMFEM_REQUIRE(h && indptr && indices && E_vals && k0sq_dev && free_mask && x && y && n > 0,
                  "emfem_sweep_spmv_noalloc: bad argument");
    EMFEM_REQUIRE(n <= EMFEM_NOALLOC_MAX_ROWS,
                  "emfem_sweep_spmv_noalloc: %lld rows exceed the fixed scratch of %d rows; use emfem_sweep_spmv",
                  (long long)n, EMFEM_NOALLOC_MAX_ROWS);
    EMFEM_REQUIRE(nsys >= 1 && nsys <= 256 && (nsys & (nsys - 1)) == 0,
                  "emfem_sweep_spmv_noalloc: nsys must be a power of two <= 256");
    EMFEM_REQUIRE(n_patch_rows == 0 || (patch_rows && patch_rowptr && patch_cols && patch_vals && patch_port && gamma_dev),
                  "emfem_sweep_spmv_noalloc: patch arrays missing");
    int prev = 0;
    EMFEM_CUDA(cudaGetDevice(&prev));
    if (prev != h->h.device) EMFEM_CUDA(cudaSetDevice(h->h.device));
    int* pmap = nullptr;
    int rc = EMFEM_OK;
    if (n_patch_rows > 0) {
        rc = noalloc_scratch(h->h.device, &pmap);
        if (rc == EMFEM_OK) rc = check_cuda(cudaMemsetAsync(pmap, 0xff, sizeof(int) * n, h->h.stream), "cudaMemsetAsync");
        if (rc == EMFEM_OK) {
            patch_map_kernel<<<grid_for(n_patch_rows, VB), VB, 0, h->h.stream>>>(n_patch_rows, patch_rows, pmap);
            rc = check_cuda(cudaGetLastError(), "patch_map_kernel");
        }
    }
    if (rc == EMFEM_OK) {
        OpArgs a;
        build_op(a, n, nsys, indptr, indices, E_vals, B_vals, k0sq_dev, pmap, patch_rowptr, patch_cols, patch_vals,
                 patch_port, n_ports, gamma_dev, free_mask);
        spmv_kernel<double><<<grid_for(n * nsys, VB), VB, 0, h->h.stream>>>(a, (const double2*)x, (double2*)y, nullptr,
                                                                              DOT_NONE, nullptr);
        rc = check_cuda(cudaGetLastError(), "spmv_kernel");
    }
    if (prev != h->h.device) cudaSetDevice(prev);
    return rc;
}
