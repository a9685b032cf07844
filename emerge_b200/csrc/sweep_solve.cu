// Frequency-sweep operator and batched COCG solver.
//
// Replaces the per-frequency direct solve (SolverSuperLU, src/emerge/_emerge/solver.py:535-572,
// through SolveRoutine.solve :1241-1326) for the systems K_f = E - k0_f^2 B + sum_p gamma_{f,p} R_p
// that Assembler.assemble_freq_matrix builds (ASM/assembler.py:255, :314-350).  All systems of a
// batch share one CSR pattern; vectors are DOF-major (n, S) so one pass over the pattern's column
// indices and E/B values serves every system, and the S entries of a gathered column are
// contiguous.  PEC elimination (SolveRoutine's A[ids, ids], solver.py:1266-1269) is a free-DOF
// mask: eliminated rows produce 0 and eliminated entries of every Krylov vector stay 0.
//
// COCG (conjugate orthogonal CG; van der Vorst & Melissen 1990) for complex-symmetric A uses the
// unconjugated bilinear form x^T y.  Every reduction is a fixed-order tree, so runs are
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
};

// y = A x for all systems; optional: partial[block][s] = sum over the block's rows of x_i * y_i
// (unconjugated) when partial != null.  One thread per (row, system).
template <typename R>
__global__ void __launch_bounds__(VB) spmv_kernel(OpArgs a, const typename V2<R>::T* __restrict__ x,
                                                   typename V2<R>::T* __restrict__ y, double2* __restrict__ partial) {
    typedef typename V2<R>::T T;
    __shared__ double2 red[VB];
    const int S = a.S;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 contrib = make_double2(0.0, 0.0);
    if (i < a.n) {
        T out = mk2<R>(0, 0);
        if (a.mask[i]) {
            const T* Ev = (const T*)a.E;
            const T* Bv = (const T*)a.B;
            R er = 0, ei = 0, br = 0, bi = 0;
            int jb = a.indptr[i], je = a.indptr[i + 1];
            for (int j = jb; j < je; j++) {
                int c = a.indices[j];
                T xv = x[(long long)c * S + s];
                T e = Ev[j];
                er += e.x * xv.x - e.y * xv.y;
                ei += e.x * xv.y + e.y * xv.x;
                if (Bv) {
                    T b = Bv[j];
                    br += b.x * xv.x - b.y * xv.y;
                    bi += b.x * xv.y + b.y * xv.x;
                }
            }
            R k2 = (R)a.k0sq[s];
            R yr = er - k2 * br, yi = ei - k2 * bi;
            int pr = a.patch_of_row ? a.patch_of_row[i] : -1;
            if (pr >= 0) {
                const T* Pv = (const T*)a.patch_vals;
                for (int q = 0; q < a.n_ports; q++) {
                    R pr_ = 0, pi_ = 0;
                    for (int j = a.patch_rowptr[pr]; j < a.patch_rowptr[pr + 1]; j++) {
                        if (a.patch_port[j] != q) continue;
                        T xv = x[(long long)a.patch_cols[j] * S + s];
                        T v = Pv[j];
                        pr_ += v.x * xv.x - v.y * xv.y;
                        pi_ += v.x * xv.y + v.y * xv.x;
                    }
                    R gr = (R)a.gamma[2 * (s * a.n_ports + q)], gi = (R)a.gamma[2 * (s * a.n_ports + q) + 1];
                    yr += gr * pr_ - gi * pi_;
                    yi += gr * pi_ + gi * pr_;
                }
            }
            out = mk2<R>(yr, yi);
            if (partial) {
                T xi = x[i * S + s];
                contrib = make_double2((double)xi.x * yr - (double)xi.y * yi, (double)xi.x * yi + (double)xi.y * yr);
            }
        }
        y[i * S + s] = out;
    }
    if (partial) {
        red[threadIdx.x] = contrib;
        __syncthreads();
        for (int off = VB / 2; off >= S; off >>= 1) {
            if (threadIdx.x < off) {
                red[threadIdx.x].x += red[threadIdx.x + off].x;
                red[threadIdx.x].y += red[threadIdx.x + off].y;
            }
            __syncthreads();
        }
        if (threadIdx.x < S) partial[(long long)blockIdx.x * S + threadIdx.x] = red[threadIdx.x];
    }
}

// Solver state per system (device).
struct SysState {
    double2 rho;      // r^T z
    double2 mu;       // p^T A p
    double2 alpha;
    double2 beta;
    double rn2;       // ||r||^2 (conjugated)
    double bn2;       // ||b||^2
    double tol2;      // tol^2 * bn2
    int active;
    int iters;
    int status;       // 0 running/converged, 1 cap, 2 breakdown
    int pad;
};

// sum partial[b][s] over blocks in fixed order, one block per system; results to out[s]
__global__ void reduce_partials_kernel(const double2* __restrict__ partial, int nblocks, int S, double2* out,
                                       int ncomp) {
    __shared__ double2 red[VB];
    int s = blockIdx.x;
    for (int comp = 0; comp < ncomp; comp++) {
        double2 acc = make_double2(0, 0);
        for (int b = threadIdx.x; b < nblocks; b += VB) {
            double2 v = partial[((long long)comp * nblocks + b) * S + s];
            acc.x += v.x; acc.y += v.y;
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int off = VB / 2; off > 0; off >>= 1) {
            if (threadIdx.x < off) { red[threadIdx.x].x += red[threadIdx.x + off].x; red[threadIdx.x].y += red[threadIdx.x + off].y; }
            __syncthreads();
        }
        if (threadIdx.x == 0) out[comp * S + s] = red[0];
        __syncthreads();
    }
}

__device__ __forceinline__ double2 cdiv2(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

// alpha = rho / mu for active systems; breakdown check
__global__ void alpha_kernel(SysState* st, const double2* mu, int S) {
    int s = threadIdx.x;
    if (s >= S) return;
    SysState& q = st[s];
    q.mu = mu[s];
    if (!q.active) { q.alpha = make_double2(0, 0); return; }
    double m = fabs(q.mu.x) + fabs(q.mu.y);
    if (!(m > 0) || !isfinite(m)) { q.active = 0; q.status = 2; q.alpha = make_double2(0, 0); return; }
    q.alpha = cdiv2(q.rho, q.mu);
}

// Preconditioner application: z = M^-1 r on DOF pairs (i, i + h)
template <typename R>
__device__ __forceinline__ void apply_block(int precond, const typename V2<R>::T* __restrict__ minv, long long h, int S,
                                            long long i, int s, const typename V2<R>::T* r, typename V2<R>::T& z_lo,
                                            typename V2<R>::T& z_hi) {
    typedef typename V2<R>::T T;
    T a = r[i * S + s], b = r[(i + h) * S + s];
    if (precond == 0) { z_lo = a; z_hi = b; return; }
    const T* m = minv + (i * S + s) * 4;
    T m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
    z_lo = mk2<R>(m00.x * a.x - m00.y * a.y + m01.x * b.x - m01.y * b.y, m00.x * a.y + m00.y * a.x + m01.x * b.y + m01.y * b.x);
    z_hi = mk2<R>(m10.x * a.x - m10.y * a.y + m11.x * b.x - m11.y * b.y, m10.x * a.y + m10.y * a.x + m11.x * b.y + m11.y * b.x);
}

// x += alpha p; r -= alpha q; z = M^-1 r; partial rho' = r^T z and ||r||^2.  Thread per (pair i, s).
template <typename R>
__global__ void __launch_bounds__(VB) update_kernel(long long h, int S, int precond, const SysState* __restrict__ st,
                                                    typename V2<R>::T* __restrict__ x, typename V2<R>::T* __restrict__ r,
                                                    typename V2<R>::T* __restrict__ z, const typename V2<R>::T* __restrict__ p,
                                                    const typename V2<R>::T* __restrict__ q, const typename V2<R>::T* __restrict__ minv,
                                                    double2* __restrict__ partial, long long nblocks) {
    typedef typename V2<R>::T T;
    __shared__ double2 red[VB];
    __shared__ double red2[VB];
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 rz = make_double2(0, 0);
    double rr = 0;
    if (i < h) {
        double2 al = st[s].alpha;
        R ar = (R)al.x, ai = (R)al.y;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            long long k = (i + half * h) * S + s;
            T pv = p[k], qv = q[k], xv = x[k], rv = r[k];
            xv.x += ar * pv.x - ai * pv.y; xv.y += ar * pv.y + ai * pv.x;
            rv.x -= ar * qv.x - ai * qv.y; rv.y -= ar * qv.y + ai * qv.x;
            x[k] = xv; r[k] = rv;
        }
        T zl, zh;
        apply_block<R>(precond, minv, h, S, i, s, r, zl, zh);
        z[i * S + s] = zl;
        z[(i + h) * S + s] = zh;
        T rl = r[i * S + s], rh = r[(i + h) * S + s];
        rz.x = (double)rl.x * zl.x - (double)rl.y * zl.y + (double)rh.x * zh.x - (double)rh.y * zh.y;
        rz.y = (double)rl.x * zl.y + (double)rl.y * zl.x + (double)rh.x * zh.y + (double)rh.y * zh.x;
        rr = (double)rl.x * rl.x + (double)rl.y * rl.y + (double)rh.x * rh.x + (double)rh.y * rh.y;
    }
    red[threadIdx.x] = rz;
    red2[threadIdx.x] = rr;
    __syncthreads();
    for (int off = VB / 2; off >= S; off >>= 1) {
        if (threadIdx.x < off) {
            red[threadIdx.x].x += red[threadIdx.x + off].x;
            red[threadIdx.x].y += red[threadIdx.x + off].y;
            red2[threadIdx.x] += red2[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x < S) {
        partial[(long long)blockIdx.x * S + threadIdx.x] = red[threadIdx.x];
        partial[(nblocks + blockIdx.x) * S + threadIdx.x] = make_double2(red2[threadIdx.x], 0.0);
    }
}

// beta = rho'/rho, convergence / breakdown / iteration bookkeeping
__global__ void beta_kernel(SysState* st, const double2* red, int S, int maxit) {
    int s = threadIdx.x;
    if (s >= S) return;
    SysState& q = st[s];
    if (!q.active) { q.beta = make_double2(0, 0); return; }
    double2 rho_new = red[s];
    q.rn2 = red[S + s].x;
    q.iters += 1;
    if (q.rn2 <= q.tol2) { q.active = 0; q.status = 0; q.beta = make_double2(0, 0); return; }
    if (!isfinite(q.rn2)) { q.active = 0; q.status = 2; q.beta = make_double2(0, 0); return; }
    if (q.iters >= maxit) { q.active = 0; q.status = 1; q.beta = make_double2(0, 0); return; }
    double m = fabs(q.rho.x) + fabs(q.rho.y);
    if (!(m > 0)) { q.active = 0; q.status = 2; q.beta = make_double2(0, 0); return; }
    q.beta = cdiv2(rho_new, q.rho);
    q.rho = rho_new;
}

// p = z + beta p (active systems only)
template <typename R>
__global__ void pupdate_kernel(long long n, int S, const SysState* __restrict__ st, const typename V2<R>::T* __restrict__ z,
                               typename V2<R>::T* __restrict__ p) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    int s = (int)(g % S);
    if (!st[s].active) return;
    double2 b = st[s].beta;
    R br = (R)b.x, bi = (R)b.y;
    typename V2<R>::T zv = z[g], pv = p[g];
    p[g] = mk2<R>(zv.x + br * pv.x - bi * pv.y, zv.y + br * pv.y + bi * pv.x);
}

// ---- setup kernels -------------------------------------------------------------------
// r = b - A x (FP64) into r64 (masked), also ||b||^2, ||r||^2 partials. x masked entries zeroed first.
__global__ void mask_vec_kernel(long long n, int S, const uint8_t* mask, double2* v) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    if (!mask[g / S]) v[g] = make_double2(0, 0);
}

__global__ void __launch_bounds__(VB) residual_kernel(long long n, int S, const uint8_t* __restrict__ mask,
                                                       const double2* __restrict__ b, const double2* __restrict__ Ax,
                                                       double2* __restrict__ r, double2* __restrict__ partial, long long nblocks) {
    __shared__ double rb[VB], rr[VB];
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    double vb = 0, vr = 0;
    if (g < n * S) {
        long long i = g / S;
        double2 res = make_double2(0, 0);
        if (mask[i]) {
            double2 bv = b[g], av = Ax[g];
            res = make_double2(bv.x - av.x, bv.y - av.y);
            vb = bv.x * bv.x + bv.y * bv.y;
            vr = res.x * res.x + res.y * res.y;
        }
        r[g] = res;
    }
    rb[threadIdx.x] = vb; rr[threadIdx.x] = vr;
    __syncthreads();
    int S_ = S;
    for (int off = VB / 2; off >= S_; off >>= 1) {
        if (threadIdx.x < off) { rb[threadIdx.x] += rb[threadIdx.x + off]; rr[threadIdx.x] += rr[threadIdx.x + off]; }
        __syncthreads();
    }
    if (threadIdx.x < S_) {
        partial[(long long)blockIdx.x * S_ + threadIdx.x] = make_double2(rb[threadIdx.x], 0);
        partial[(nblocks + blockIdx.x) * S_ + threadIdx.x] = make_double2(rr[threadIdx.x], 0);
    }
}

// Block-Jacobi / point-Jacobi inverse blocks from the operator's diagonal 2x2 pair blocks.
__device__ __forceinline__ double2 row_value(const OpArgs& a, long long row, long long col, int s) {
    const double2* Ev = (const double2*)a.E;
    const double2* Bv = (const double2*)a.B;
    int lo = a.indptr[row], hi = a.indptr[row + 1] - 1;
    double2 v = make_double2(0, 0);
    if (hi >= lo) {
        while (lo < hi) { int mid = (lo + hi) >> 1; if (a.indices[mid] < col) lo = mid + 1; else hi = mid; }
        if (a.indices[lo] == col) {
            double2 e = Ev[lo];
            double k2 = a.k0sq[s];
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
            double gr = a.gamma[2 * (s * a.n_ports + q)], gi = a.gamma[2 * (s * a.n_ports + q) + 1];
            double2 pv = Pv[j];
            v.x += gr * pv.x - gi * pv.y;
            v.y += gr * pv.y + gi * pv.x;
        }
    }
    return v;
}

template <typename R>
__global__ void precond_setup_kernel(OpArgs a, int precond, typename V2<R>::T* __restrict__ minv) {
    long long h = a.n / 2;
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    int S = a.S;
    if (g >= h * S) return;
    long long i = g / S;
    int s = (int)(g % S);
    long long j = i + h;
    double2 m00 = make_double2(0, 0), m01 = m00, m10 = m00, m11 = m00;
    bool fi = a.mask[i] != 0, fj = a.mask[j] != 0;
    double2 a00 = fi ? row_value(a, i, i, s) : make_double2(1, 0);
    double2 a11 = fj ? row_value(a, j, j, s) : make_double2(1, 0);
    double2 a01 = (fi && fj) ? row_value(a, i, j, s) : make_double2(0, 0);
    double2 a10 = (fi && fj) ? row_value(a, j, i, s) : make_double2(0, 0);
    auto inv1 = [](double2 v) {
        double m = fabs(v.x) + fabs(v.y);
        return m > 0 ? cdiv2(make_double2(1, 0), v) : make_double2(1, 0);
    };
    if (precond == 2) {
        double2 det = make_double2(a00.x * a11.x - a00.y * a11.y - (a01.x * a10.x - a01.y * a10.y),
                                   a00.x * a11.y + a00.y * a11.x - (a01.x * a10.y + a01.y * a10.x));
        double dm = fabs(det.x) + fabs(det.y);
        double sc = fabs(a00.x) + fabs(a00.y) + fabs(a11.x) + fabs(a11.y);
        if (dm > 1e-14 * sc * sc && isfinite(dm)) {
            double2 id = cdiv2(make_double2(1, 0), det);
            auto mul = [](double2 u, double2 v) { return make_double2(u.x * v.x - u.y * v.y, u.x * v.y + u.y * v.x); };
            m00 = mul(a11, id);
            m11 = mul(a00, id);
            m01 = mul(make_double2(-a01.x, -a01.y), id);
            m10 = mul(make_double2(-a10.x, -a10.y), id);
        } else {
            m00 = inv1(a00); m11 = inv1(a11);
        }
    } else {
        m00 = inv1(a00); m11 = inv1(a11);
    }
    typename V2<R>::T* m = minv + (i * S + s) * 4;
    m[0] = mk2<R>((R)m00.x, (R)m00.y); m[1] = mk2<R>((R)m01.x, (R)m01.y);
    m[2] = mk2<R>((R)m10.x, (R)m10.y); m[3] = mk2<R>((R)m11.x, (R)m11.y);
}

__global__ void init_state_kernel(SysState* st, const double2* red, int S, int nsys, double tol, int use_x0) {
    int s = threadIdx.x;
    if (s >= S) return;
    SysState q;
    q.rho = make_double2(0, 0); q.mu = q.rho; q.alpha = q.rho; q.beta = q.rho;
    q.bn2 = red[s].x;
    q.rn2 = red[S + s].x;
    q.tol2 = tol * tol * q.bn2;
    q.iters = 0; q.status = 0; q.pad = 0;
    q.active = (s < nsys) && (q.rn2 > q.tol2) && (q.bn2 > 0);
    st[s] = q;
}

// after z = M^-1 r for the initial residual: rho = r^T z, p = z
template <typename R>
__global__ void __launch_bounds__(VB) init_z_kernel(long long h, int S, int precond, const typename V2<R>::T* __restrict__ r,
                                                    typename V2<R>::T* __restrict__ z, typename V2<R>::T* __restrict__ p,
                                                    const typename V2<R>::T* __restrict__ minv, double2* __restrict__ partial) {
    typedef typename V2<R>::T T;
    __shared__ double2 red[VB];
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    long long i = g / S;
    int s = (int)(g % S);
    double2 rz = make_double2(0, 0);
    if (i < h) {
        T zl, zh;
        apply_block<R>(precond, minv, h, S, i, s, r, zl, zh);
        z[i * S + s] = zl; z[(i + h) * S + s] = zh;
        p[i * S + s] = zl; p[(i + h) * S + s] = zh;
        T rl = r[i * S + s], rh = r[(i + h) * S + s];
        rz.x = (double)rl.x * zl.x - (double)rl.y * zl.y + (double)rh.x * zh.x - (double)rh.y * zh.y;
        rz.y = (double)rl.x * zl.y + (double)rl.y * zl.x + (double)rh.x * zh.y + (double)rh.y * zh.x;
    }
    red[threadIdx.x] = rz;
    __syncthreads();
    for (int off = VB / 2; off >= S; off >>= 1) {
        if (threadIdx.x < off) { red[threadIdx.x].x += red[threadIdx.x + off].x; red[threadIdx.x].y += red[threadIdx.x + off].y; }
        __syncthreads();
    }
    if (threadIdx.x < S) partial[(long long)blockIdx.x * S + threadIdx.x] = red[threadIdx.x];
}

__global__ void set_rho_kernel(SysState* st, const double2* red, int S) {
    int s = threadIdx.x;
    if (s < S) st[s].rho = red[s];
}

// conversions / scaled copies for the mixed-precision refinement
__global__ void to_f32_scaled_kernel(long long n, int S, const double2* __restrict__ src, const SysState* st64,
                                     float2* __restrict__ dst, double* __restrict__ scale) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    int s = (int)(g % S);
    double rn = sqrt(st64[s].rn2);
    double sc = rn > 0 ? 1.0 / rn : 0.0;
    double2 v = src[g];
    dst[g] = make_float2((float)(v.x * sc), (float)(v.y * sc));
    if (g < S) scale[g] = rn;
}

__global__ void add_scaled_f32_kernel(long long n, int S, const float2* __restrict__ d, const double* __restrict__ scale,
                                      const int* __restrict__ outer_active, double2* __restrict__ x) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g >= n * S) return;
    int s = (int)(g % S);
    if (!outer_active[s]) return;
    double sc = scale[s];
    float2 v = d[g];
    x[g].x += sc * (double)v.x;
    x[g].y += sc * (double)v.y;
}

__global__ void cast_values_kernel(long long nnz, const double2* __restrict__ src, float2* __restrict__ dst) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g < nnz) dst[g] = make_float2((float)src[g].x, (float)src[g].y);
}

__global__ void patch_map_kernel(long long np, const int* rows, int* patch_of_row) {
    long long g = (long long)blockIdx.x * VB + threadIdx.x;
    if (g < np) patch_of_row[rows[g]] = (int)g;
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
    // (E - (k0^2 B)) with the product rounded first, as the reference's E - B*k0**2
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
    size_t off_state, off_gamma, off_k0, off_partial, off_red, off_patchmap, off_scale, off_oactive;
    size_t off_x, off_b, off_r64, off_Ax;                  // FP64 vectors (n, S)
    size_t off_r, off_z, off_p, off_q, off_minv;           // Krylov vectors of the inner precision
    size_t off_E32, off_B32, off_P32;                      // FP32 matrix copies (mixed)
    size_t total;
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static Layout make_layout(long long n, long long nnz, long long npatch, int S, int nports, int precision) {
    Layout L;
    size_t o = 0;
    long long nb = (n * S + VB - 1) / VB + 1;
    size_t vec64 = (size_t)n * S * sizeof(double2);
    size_t vecw = (size_t)n * S * (precision ? sizeof(float2) : sizeof(double2));
    L.off_state = o; o = align256(o + sizeof(SysState) * 2 * S);
    L.off_gamma = o; o = align256(o + sizeof(double) * 2 * S * (nports > 0 ? nports : 1));
    L.off_k0 = o; o = align256(o + sizeof(double) * S);
    L.off_partial = o; o = align256(o + sizeof(double2) * 2 * nb * S);
    L.off_red = o; o = align256(o + sizeof(double2) * 2 * S);
    L.off_patchmap = o; o = align256(o + sizeof(int) * n);
    L.off_scale = o; o = align256(o + sizeof(double) * S);
    L.off_oactive = o; o = align256(o + sizeof(int) * S);
    L.off_x = o; o = align256(o + vec64);
    L.off_b = o; o = align256(o + vec64);
    L.off_r64 = o; o = align256(o + vec64);
    L.off_Ax = o; o = align256(o + vec64);
    L.off_r = o; o = align256(o + vecw);
    L.off_z = o; o = align256(o + vecw);
    L.off_p = o; o = align256(o + vecw);
    L.off_q = o; o = align256(o + vecw);
    L.off_minv = o; o = align256(o + vecw * 2);  // (n/2) * S * 4 entries
    if (precision) {
        L.off_E32 = o; o = align256(o + sizeof(float2) * nnz);
        L.off_B32 = o; o = align256(o + sizeof(float2) * nnz);
        L.off_P32 = o; o = align256(o + sizeof(float2) * (npatch > 0 ? npatch : 1));
    } else {
        L.off_E32 = L.off_B32 = L.off_P32 = 0;
    }
    L.total = o;
    return L;
}

// One Krylov solve (inner precision R) on the operator `op` for rhs already in r (= b - A x0 form
// is handled by the caller): runs COCG iterations from x = 0 with initial residual r.
template <typename R>
struct Cocg {
    typedef typename V2<R>::T T;
    OpArgs op;
    long long n, h;
    int S, precond, maxit;
    T *x, *r, *z, *p, *q, *minv;
    double2 *partial, *red;
    SysState* st;
    long long nb_rows, nb_pairs;
    cudaStream_t s;

    int launch_iteration() {
        spmv_kernel<R><<<(unsigned)nb_rows, VB, 0, s>>>(op, p, q, partial);
        reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_rows, S, red, 1);
        alpha_kernel<<<1, 64, 0, s>>>(st, red, S);
        update_kernel<R><<<(unsigned)nb_pairs, VB, 0, s>>>(h, S, precond, st, x, r, z, p, q, minv, partial, nb_pairs);
        reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_pairs, S, red, 2);
        beta_kernel<<<1, 64, 0, s>>>(st, red, S, maxit);
        pupdate_kernel<R><<<grid_for(n * S, VB), VB, 0, s>>>(n, S, st, z, p);
        return check_cuda(cudaGetLastError(), "cocg iteration");
    }

    // start: r holds the initial residual (masked), x holds 0; st[].bn2/tol2/active set.
    int start() {
        init_z_kernel<R><<<(unsigned)nb_pairs, VB, 0, s>>>(h, S, precond, r, z, p, minv, partial);
        reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_pairs, S, red, 1);
        set_rho_kernel<<<1, 64, 0, s>>>(st, red, S);
        return check_cuda(cudaGetLastError(), "cocg start");
    }

    int run(int chunk) {
        // capture `chunk` iterations once, replay until no system is active
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        EMFEM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st_cap = EMFEM_OK;
        for (int k = 0; k < chunk && st_cap == EMFEM_OK; k++) st_cap = launch_iteration();
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st_cap != EMFEM_OK) { if (graph) cudaGraphDestroy(graph); return st_cap; }
        EMFEM_CUDA(e);
        EMFEM_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        std::vector<SysState> host(S);
        int rounds = (maxit + chunk - 1) / chunk + 1;
        int rc = EMFEM_OK;
        for (int it = 0; it < rounds; it++) {
            if ((rc = check_cuda(cudaGraphLaunch(exec, s), "cudaGraphLaunch")) != EMFEM_OK) break;
            if ((rc = check_cuda(cudaMemcpyAsync(host.data(), st, sizeof(SysState) * S, cudaMemcpyDeviceToHost, s), "copy state")) != EMFEM_OK) break;
            if ((rc = check_cuda(cudaStreamSynchronize(s), "sync")) != EMFEM_OK) break;
            bool any = false;
            for (int k = 0; k < S; k++) any |= host[k].active != 0;
            if (!any) break;
        }
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return rc;
    }
};

}  // namespace emfem

using namespace emfem;

extern "C" {

int emfem_cocg_workspace_size(int64_t n, int64_t nnz, int nsys, int precision, size_t* bytes) {
    EMFEM_REQUIRE(bytes && n > 0 && nsys > 0 && nsys <= 64, "emfem_cocg_workspace_size: bad argument");
    int S = pow2_at_least(nsys);
    // patch size bound: callers pass npatch <= nnz; reserve for nnz/8 (ports touch few rows)
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

static int build_op(OpArgs& a, int64_t n, int S, const int32_t* indptr, const int32_t* indices, const void* E,
                    const void* B, const double* k0dev, const int* pmap, const int32_t* prowptr, const int32_t* pcols,
                    const void* pvals, const int32_t* pport, int nports, const double* gdev, const uint8_t* mask) {
    a.n = n; a.S = S; a.indptr = indptr; a.indices = indices; a.E = E; a.B = B; a.k0sq = k0dev;
    a.patch_of_row = pmap; a.patch_rowptr = prowptr; a.patch_cols = pcols; a.patch_vals = pvals; a.patch_port = pport;
    a.n_ports = nports; a.gamma = gdev; a.mask = mask;
    return EMFEM_OK;
}

int emfem_sweep_spmv(emfem_handle h, int64_t n, const int32_t* indptr, const int32_t* indices,
                     const void* E_vals, const void* B_vals, int nsys, const double* k0sq_dev,
                     int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                     const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                     int n_ports, const double* gamma_dev, const uint8_t* free_mask, const void* x, void* y) {
    EMFEM_REQUIRE(h && indptr && indices && E_vals && k0sq_dev && free_mask && x && y && n > 0,
                  "emfem_sweep_spmv: bad argument");
    EMFEM_REQUIRE(nsys >= 1 && nsys <= 256 && (VB % nsys) == 0 && (nsys & (nsys - 1)) == 0,
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
    spmv_kernel<double><<<grid_for(n * nsys, VB), VB, 0, h->h.stream>>>(a, (const double2*)x, (double2*)y, nullptr);
    EMFEM_LAUNCH("spmv_kernel");
    if (pmap) EMFEM_CUDA(cudaFreeAsync(pmap, h->h.stream));
    return EMFEM_OK;
}

int emfem_cocg_solve(emfem_handle hd, int64_t n, int64_t nnz, const int32_t* indptr, const int32_t* indices,
                     const void* E_vals, const void* B_vals, int nsys, const double* k0sq,
                     int64_t n_patch_rows, const int32_t* patch_rows, const int32_t* patch_rowptr,
                     const int32_t* patch_cols, const void* patch_vals, const int32_t* patch_port,
                     int n_ports, const double* gamma, const uint8_t* free_mask, const void* rhs, void* x,
                     double tol, int maxit, int precond, int precision, void* workspace, size_t workspace_bytes,
                     int* status, int* iters, double* relres) {
    EMFEM_REQUIRE(hd && indptr && indices && E_vals && k0sq && free_mask && rhs && x && workspace,
                  "emfem_cocg_solve: null argument");
    EMFEM_REQUIRE(n > 0 && (n % 2) == 0, "emfem_cocg_solve: n must be even (DOF pairs i, i + n/2)");
    EMFEM_REQUIRE(nsys >= 1 && nsys <= 64, "emfem_cocg_solve: 1 <= nsys <= 64");
    EMFEM_REQUIRE(precond >= 0 && precond <= 2 && (precision == 0 || precision == 1), "emfem_cocg_solve: bad option");
    EMFEM_REQUIRE(n_ports >= 0 && n_ports <= 8, "emfem_cocg_solve: at most 8 ports");
    EMFEM_REQUIRE(n_patch_rows == 0 || (patch_rows && patch_rowptr && patch_cols && patch_vals && patch_port && gamma),
                  "emfem_cocg_solve: patch arrays missing");
    EMFEM_REQUIRE(tol > 0 && maxit > 0, "emfem_cocg_solve: tol and maxit must be positive");
    Handle* h = &hd->h;
    int S = pow2_at_least(nsys);
    int64_t npatch = 0;
    if (n_patch_rows > 0) {
        int32_t last = 0;
        EMFEM_CUDA(cudaMemcpy(&last, patch_rowptr + n_patch_rows, sizeof(int32_t), cudaMemcpyDeviceToHost));
        npatch = last;
    }
    Layout L = make_layout(n, nnz, npatch, S, n_ports, precision);
    if (workspace_bytes < L.total) {
        set_error("emfem_cocg_solve: workspace of %zu bytes, %zu needed", workspace_bytes, L.total);
        return EMFEM_ERR_WORKSPACE;
    }
    char* ws = (char*)workspace;
    cudaStream_t s = nullptr;
    EMFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t ev;
    EMFEM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    EMFEM_CUDA(cudaEventRecord(ev, h->stream));
    EMFEM_CUDA(cudaStreamWaitEvent(s, ev, 0));

    SysState* st = (SysState*)(ws + L.off_state);
    SysState* st_outer = st + S;
    double* gdev = (double*)(ws + L.off_gamma);
    double* k0dev = (double*)(ws + L.off_k0);
    double2* partial = (double2*)(ws + L.off_partial);
    double2* red = (double2*)(ws + L.off_red);
    int* pmap = (int*)(ws + L.off_patchmap);
    double* scale = (double*)(ws + L.off_scale);
    int* oactive = (int*)(ws + L.off_oactive);
    double2* x64 = (double2*)(ws + L.off_x);
    double2* b64 = (double2*)(ws + L.off_b);
    double2* r64 = (double2*)(ws + L.off_r64);
    double2* Ax = (double2*)(ws + L.off_Ax);

    std::vector<double> hk0(S, 0.0), hg(2 * S * (n_ports > 0 ? n_ports : 1), 0.0);
    for (int k = 0; k < nsys; k++) hk0[k] = k0sq[k];
    for (int k = 0; k < nsys; k++)
        for (int q = 0; q < n_ports; q++) { hg[2 * (k * n_ports + q)] = gamma[2 * (k * n_ports + q)]; hg[2 * (k * n_ports + q) + 1] = gamma[2 * (k * n_ports + q) + 1]; }
    int rc = EMFEM_OK;
#define STRY(x) do { rc = (x); if (rc != EMFEM_OK) goto done; } while (0)
    STRY(check_cuda(cudaMemcpyAsync(k0dev, hk0.data(), sizeof(double) * S, cudaMemcpyHostToDevice, s), "copy k0"));
    STRY(check_cuda(cudaMemcpyAsync(gdev, hg.data(), sizeof(double) * hg.size(), cudaMemcpyHostToDevice, s), "copy gamma"));
    STRY(check_cuda(cudaMemsetAsync(pmap, 0xff, sizeof(int) * n, s), "memset"));
    if (n_patch_rows > 0) {
        patch_map_kernel<<<grid_for(n_patch_rows, VB), VB, 0, s>>>(n_patch_rows, patch_rows, pmap);
        STRY(check_cuda(cudaGetLastError(), "patch_map_kernel"));
    }
    {
        long long nS = n * (long long)S;
        unsigned gv = grid_for(nS, VB);
        pad_copy_kernel<<<gv, VB, 0, s>>>(n, nsys, S, (const double2*)rhs, b64);
        pad_copy_kernel<<<gv, VB, 0, s>>>(n, nsys, S, (const double2*)x, x64);
        mask_vec_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, b64);
        mask_vec_kernel<<<gv, VB, 0, s>>>(n, S, free_mask, x64);
        STRY(check_cuda(cudaGetLastError(), "setup copies"));

        OpArgs op64;
        build_op(op64, n, S, indptr, indices, E_vals, B_vals, k0dev, n_patch_rows ? pmap : nullptr, patch_rowptr,
                 patch_cols, patch_vals, patch_port, n_ports, gdev, free_mask);
        long long nb_rows = grid_for(nS, VB);
        long long nb_pairs = grid_for((n / 2) * (long long)S, VB);
        // initial residual r64 = b - A x0, norms
        spmv_kernel<double><<<(unsigned)nb_rows, VB, 0, s>>>(op64, x64, Ax, nullptr);
        residual_kernel<<<(unsigned)nb_rows, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial, nb_rows);
        reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_rows, S, red, 2);
        init_state_kernel<<<1, 64, 0, s>>>(st_outer, red, S, nsys, tol, 1);
        STRY(check_cuda(cudaGetLastError(), "initial residual"));

        if (precision == 0) {
            Cocg<double> c;
            c.op = op64; c.n = n; c.h = n / 2; c.S = S; c.precond = precond; c.maxit = maxit;
            c.x = x64; c.r = (double2*)(ws + L.off_r); c.z = (double2*)(ws + L.off_z); c.p = (double2*)(ws + L.off_p);
            c.q = (double2*)(ws + L.off_q); c.minv = (double2*)(ws + L.off_minv);
            c.partial = partial; c.red = red; c.st = st; c.nb_rows = nb_rows; c.nb_pairs = nb_pairs; c.s = s;
            if (precond) {
                precond_setup_kernel<double><<<grid_for((n / 2) * (long long)S, VB), VB, 0, s>>>(op64, precond, c.minv);
                STRY(check_cuda(cudaGetLastError(), "precond_setup"));
            }
            STRY(check_cuda(cudaMemcpyAsync(c.r, r64, sizeof(double2) * nS, cudaMemcpyDeviceToDevice, s), "copy r"));
            STRY(check_cuda(cudaMemcpyAsync(st, st_outer, sizeof(SysState) * S, cudaMemcpyDeviceToDevice, s), "copy st"));
            STRY(c.start());
            STRY(c.run(16));
        } else {
            // FP32 operator copies
            float2* E32 = (float2*)(ws + L.off_E32);
            float2* B32 = (float2*)(ws + L.off_B32);
            float2* P32 = (float2*)(ws + L.off_P32);
            cast_values_kernel<<<grid_for(nnz, VB), VB, 0, s>>>(nnz, (const double2*)E_vals, E32);
            if (B_vals) cast_values_kernel<<<grid_for(nnz, VB), VB, 0, s>>>(nnz, (const double2*)B_vals, B32);
            if (npatch > 0) cast_values_kernel<<<grid_for(npatch, VB), VB, 0, s>>>(npatch, (const double2*)patch_vals, P32);
            STRY(check_cuda(cudaGetLastError(), "cast values"));
            OpArgs op32 = op64;
            op32.E = E32; op32.B = B_vals ? B32 : nullptr; op32.patch_vals = P32;
            Cocg<float> c;
            c.op = op32; c.n = n; c.h = n / 2; c.S = S; c.precond = precond;
            c.r = (float2*)(ws + L.off_r); c.z = (float2*)(ws + L.off_z); c.p = (float2*)(ws + L.off_p);
            c.q = (float2*)(ws + L.off_q); c.minv = (float2*)(ws + L.off_minv);
            c.x = (float2*)(ws + L.off_Ax);  // reuse: d (FP32) lives in the Ax buffer's first half
            c.partial = partial; c.red = red; c.st = st; c.nb_rows = nb_rows; c.nb_pairs = nb_pairs; c.s = s;
            if (precond) {
                precond_setup_kernel<float><<<grid_for((n / 2) * (long long)S, VB), VB, 0, s>>>(op64, precond, c.minv);
                STRY(check_cuda(cudaGetLastError(), "precond_setup"));
            }
            float2* d32 = (float2*)(ws + L.off_Ax);
            std::vector<SysState> ho(S);
            int total_inner = 0;
            std::vector<int> inner_iters(S, 0);
            const int max_outer = 40;
            for (int outer = 0; outer < max_outer; outer++) {
                STRY(check_cuda(cudaMemcpyAsync(ho.data(), st_outer, sizeof(SysState) * S, cudaMemcpyDeviceToHost, s), "copy"));
                STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
                std::vector<int> act(S, 0);
                bool any = false;
                for (int k = 0; k < S; k++) { act[k] = ho[k].active; any |= act[k] != 0; }
                if (!any || total_inner >= maxit) break;
                STRY(check_cuda(cudaMemcpyAsync(oactive, act.data(), sizeof(int) * S, cudaMemcpyHostToDevice, s), "copy"));
                // inner: A d = r64 / ||r64|| in FP32 to a relative 1e-4 (bounded by remaining budget)
                to_f32_scaled_kernel<<<gv, VB, 0, s>>>(n, S, r64, st_outer, c.r, scale);
                STRY(check_cuda(cudaMemsetAsync(d32, 0, sizeof(float2) * nS, s), "memset d"));
                std::vector<SysState> hin(S);
                for (int k = 0; k < S; k++) {
                    SysState q;
                    memset(&q, 0, sizeof(q));
                    q.bn2 = act[k] ? 1.0 : 0.0;
                    q.rn2 = q.bn2;
                    q.tol2 = 1e-8;  // inner relative tolerance 1e-4
                    q.active = act[k];
                    hin[k] = q;
                }
                STRY(check_cuda(cudaMemcpyAsync(st, hin.data(), sizeof(SysState) * S, cudaMemcpyHostToDevice, s), "copy"));
                c.maxit = std::max(1, maxit - total_inner);
                STRY(c.start());
                STRY(c.run(16));
                STRY(check_cuda(cudaMemcpyAsync(hin.data(), st, sizeof(SysState) * S, cudaMemcpyDeviceToHost, s), "copy"));
                STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
                int mx = 0;
                for (int k = 0; k < S; k++) { inner_iters[k] += act[k] ? hin[k].iters : 0; mx = std::max(mx, act[k] ? hin[k].iters : 0); }
                total_inner += std::max(mx, 1);
                add_scaled_f32_kernel<<<gv, VB, 0, s>>>(n, S, d32, scale, oactive, x64);
                // new FP64 residual
                spmv_kernel<double><<<(unsigned)nb_rows, VB, 0, s>>>(op64, x64, Ax, nullptr);
                residual_kernel<<<(unsigned)nb_rows, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial, nb_rows);
                reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_rows, S, red, 2);
                // refresh outer state: keep bn2/tol2, update rn2 and active
                STRY(check_cuda(cudaGetLastError(), "refinement"));
                std::vector<double2> hred(2 * S);
                STRY(check_cuda(cudaMemcpyAsync(hred.data(), red, sizeof(double2) * 2 * S, cudaMemcpyDeviceToHost, s), "copy"));
                STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
                for (int k = 0; k < S; k++) {
                    ho[k].rn2 = hred[S + k].x;
                    ho[k].iters = inner_iters[k];
                    if (ho[k].active) {
                        if (ho[k].rn2 <= ho[k].tol2) { ho[k].active = 0; ho[k].status = 0; }
                        else if (!std::isfinite(ho[k].rn2) || hin[k].status == 2) { ho[k].active = 0; ho[k].status = 2; }
                    }
                }
                STRY(check_cuda(cudaMemcpyAsync(st_outer, ho.data(), sizeof(SysState) * S, cudaMemcpyHostToDevice, s), "copy"));
            }
            STRY(check_cuda(cudaMemcpyAsync(ho.data(), st_outer, sizeof(SysState) * S, cudaMemcpyDeviceToHost, s), "copy"));
            STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
            for (int k = 0; k < S; k++) {
                if (ho[k].active) { ho[k].active = 0; ho[k].status = 1; }
                ho[k].iters = inner_iters[k];
            }
            STRY(check_cuda(cudaMemcpyAsync(st, ho.data(), sizeof(SysState) * S, cudaMemcpyHostToDevice, s), "copy"));
        }
        // final FP64 true residual
        spmv_kernel<double><<<(unsigned)nb_rows, VB, 0, s>>>(op64, x64, Ax, nullptr);
        residual_kernel<<<(unsigned)nb_rows, VB, 0, s>>>(n, S, free_mask, b64, Ax, r64, partial, nb_rows);
        reduce_partials_kernel<<<S, VB, 0, s>>>(partial, (int)nb_rows, S, red, 2);
        unpad_copy_kernel<<<grid_for(n * (long long)nsys, VB), VB, 0, s>>>(n, nsys, S, x64, (double2*)x);
        STRY(check_cuda(cudaGetLastError(), "final residual"));
        std::vector<SysState> hs(S);
        std::vector<double2> hred(2 * S);
        STRY(check_cuda(cudaMemcpyAsync(hs.data(), st, sizeof(SysState) * S, cudaMemcpyDeviceToHost, s), "copy"));
        STRY(check_cuda(cudaMemcpyAsync(hred.data(), red, sizeof(double2) * 2 * S, cudaMemcpyDeviceToHost, s), "copy"));
        STRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        bool all_ok = true;
        for (int k = 0; k < nsys; k++) {
            double bn = hred[k].x, rn = hred[S + k].x;
            double rel = bn > 0 ? std::sqrt(rn / bn) : 0.0;
            int stat = hs[k].status;
            if (hs[k].active) stat = 1;
            if (stat == 0 && rel > tol * 10) stat = 1;  // recurrence drifted from the true residual
            if (status) status[k] = stat;
            if (iters) iters[k] = hs[k].iters;
            if (relres) relres[k] = rel;
            all_ok &= stat == 0;
        }
        if (!all_ok) {
            set_error("emfem_cocg_solve: not every system reached the tolerance");
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

}  // extern "C"
