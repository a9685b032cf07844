// Multifrontal sparse LU of the sweep system on the device, the direct solve that replaces the
// reference's SolverSuperLU (src/emerge/_emerge/solver.py:535-572).  It factors the equilibrated
// D^-1/2 K D^-1/2 (D = |diag K|) with complex64 fronts, or complex128 fronts after
// emfem_mf_set_precision(lu, 128); the factor store is complex64 either way.
//
// The symbolic structure (nested-dissection tree, front DOF lists, extend-add maps, assembly lists) is
// built on the host (emerge_b200/direct.py) and uploaded once per mesh.  The numeric factorization runs
// level by level over the tree (all fronts of one height at once):
//   1. every front of the level is zeroed and gets its own entries of the scaled K (FP64 -> front
//      precision) and the Schur complements of its children (extend-add, one child slot after the other:
//      no atomics);
//   2. the first e columns of every front are eliminated in steps of 32: LU with partial pivoting inside
//      the 32 x 32 diagonal block (diag_kernel, one warp per front, also forming the explicit inverses
//      of its L and U), the block row (row swaps + L^-1) and block column (U^-1) of the panel
//      (panel_kernel), and the rank-32 update of the trailing matrix (trail_kernel: 64 x 64 tiles,
//      4 x 4 complex register tiles per thread), every kernel batched over the level's fronts;
//   3. the factor columns, the U block row and the Schur complement are copied out of the level
//      workspace (compact_kernel): factors to the factor store (rounded to complex64), the Schur
//      complement to the update store (front precision) until the parent's level consumes it.
// Pivoting stays inside each 32-row diagonal block (rows are never exchanged across blocks), so row swaps
// touch only the block row; the solves apply them step by step.  A pivot smaller than 1e-6 of its block's
// largest entry is raised to that floor and counted: the factorization is a preconditioner under an FP64
// Krylov iteration, which removes such perturbations.
//
// Solves (M^-1 r for S right-hand sides, FP64 in and out, FP32 inside, scaled by D^-1/2 on the way in
// and out) run the same tree: forward in level order (gather, children's update vectors, blocked L solve
// with 256-row blocks, update vector for the parent), backward in reverse (gather of the solved boundary,
// U12 product, blocked U solve).
#include "emfem_internal.cuh"

#include <algorithm>
#include <map>
#include <vector>

namespace emfem {

constexpr int MF_NB = 32;          // pivot block / elimination step
constexpr int MF_SB = 256;         // solve block
constexpr int MF_TILE = 64;        // trailing-update tile
constexpr long long MF_CHUNK = 4096;
constexpr int MF_MAX_FRONT = 46340; // n^2 must fit an int32 local offset

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cfma(float2& c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x));
    c.y = fmaf(a.x, b.y, fmaf(a.y, b.x, c.y));
}
__device__ __forceinline__ void cfms(float2& c, float2 a, float2 b) {   // c -= a b
    c.x = fmaf(-a.x, b.x, fmaf(a.y, b.y, c.x));
    c.y = fmaf(-a.x, b.y, fmaf(-a.y, b.x, c.y));
}
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// 8-byte asynchronous global -> shared copies: a thread issues all of its copies before waiting once,
// so a staging loop costs one memory round trip instead of one per element
__device__ __forceinline__ void cp_async8(void* dst_smem, const void* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most one committed group is still in flight
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ float2 cinv(float2 a) {
    float d = 1.0f / cabs2(a);
    return make_float2(a.x * d, -a.y * d);
}

// The same operations in double precision (factorizations computed in complex128)
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cfma(double2& c, double2 a, double2 b) {
    c.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
    c.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
}
__device__ __forceinline__ void cfms(double2& c, double2 a, double2 b) {
    c.x = fma(-a.x, b.x, fma(a.y, b.y, c.x));
    c.y = fma(-a.x, b.y, fma(-a.y, b.x, c.y));
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double2 cinv(double2 a) {
    double d = 1.0 / cabs2(a);
    return make_double2(a.x * d, -a.y * d);
}

// complex64 / complex128 element helpers for the templated factorization kernels
template <typename T> struct CxT;
template <> struct CxT<float2> {
    typedef float R;
    __device__ static float2 make(double x, double y) { return make_float2((float)x, (float)y); }
};
template <> struct CxT<double2> {
    typedef double R;
    __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
__device__ __forceinline__ float2 to_c64(float2 v) { return v; }
__device__ __forceinline__ float2 to_c64(double2 v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_c(float2* dst_smem, const float2* src) { cp_async8(dst_smem, src); }
__device__ __forceinline__ void cp_async_c(double2* dst_smem, const double2* src) { cp_async16(dst_smem, src); }

struct FrontMeta {        // per front, device
    int e, b, n, parent;
    int child[2];
    long long fdof, ea, asm0, asm1;   // offsets into fdof / ea / asm arrays
    long long fact, inv, piv;         // factor store offsets (float2 / float2 / int)
    long long ws, upd;                // level workspace (float2) / update store (float2) offsets
    long long wv, uv, y;              // solve buffers: level w (rows), update vectors (rows), own solution (rows)
};

// ---------------------------------------------------------------- factorization kernels
// Symmetric diagonal equilibration: the factorization runs on D^-1/2 K D^-1/2 with D = |diag K|, so every
// pivot candidate is measured against unit diagonals.  Without it the gradient-type DOFs of the
// second-order basis (curl-curl column exactly zero, diagonal -k0^2 B_jj only) carry legitimate pivots
// far below the curl-curl scale at low frequency, and the 32-row pivot floor would perturb them.
// The scale of a DOF is set by the front that eliminates it, from its diagonal assembly entry.
__global__ void mf_scale_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                const double2* __restrict__ K, const int* __restrict__ slot, const int* __restrict__ off,
                                const int* __restrict__ fdof, double* __restrict__ scale) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long k0 = f.asm0 + (long long)blockIdx.x * MF_CHUNK;
    long long k1 = min(k0 + MF_CHUNK, f.asm1);
    const int n = f.n;
    for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const int o = off[k], li = o % n;
        if (li != o / n || li >= f.e) continue;
        double2 v = K[slot[k]];
        double a = fabs(v.x) + fabs(v.y);          // |.|_1 of the diagonal: scale only, no accuracy rides on it
        scale[fdof[f.fdof + li]] = a > 0.0 ? rsqrt(a) : 1.0;
    }
}

// Factorization kernels are templated on the workspace element T: float2 (complex64 fronts) or double2
// (complex128 fronts).  The factor store that the solves read is complex64 in both cases; a complex128
// factorization rounds its factors once, at compaction, so the rounding error does not compound through
// the Schur-complement chain.
template <typename T>
__global__ void mf_asm_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                              const double2* __restrict__ K, const int* __restrict__ slot, const int* __restrict__ off,
                              const int* __restrict__ fdof, const double* __restrict__ scale, T* __restrict__ ws) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long k0 = f.asm0 + (long long)blockIdx.x * MF_CHUNK;
    long long k1 = min(k0 + MF_CHUNK, f.asm1);
    T* W = ws + f.ws;
    const int n = f.n;
    const int* D = fdof + f.fdof;
    for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const int o = off[k];
        double2 v = K[slot[k]];
        double sc = scale[D[o % n]] * scale[D[o / n]];
        W[o] = CxT<T>::make(v.x * sc, v.y * sc);
    }
}

template <typename T>
__global__ void mf_ea_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int cslot,
                             const int* __restrict__ ea, const T* __restrict__ upd, T* __restrict__ ws) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    int c = f.child[cslot];
    if (c < 0) return;
    const FrontMeta& g = fm[c];
    long long nb = g.b;
    long long tot = nb * nb;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    const int* map = ea + g.ea;
    const T* U = upd + g.upd;
    T* W = ws + f.ws;
    long long ld = f.n;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx % nb, j = idx / nb;
        T u = U[idx];
        T* dst = W + map[i] + (long long)map[j] * ld;
        dst->x += u.x;
        dst->y += u.y;
    }
}

// LU with partial pivoting of the 32 x 32 diagonal block at step k, plus the explicit inverses of its
// unit-lower L and upper U.  One warp per front; lane = column (or row in the pivot search).  The
// inverses go to inv (complex64, read by the solves) and, for a complex128 factorization, also to invc
// (complex128, read by the panel kernel); for complex64 invc is inv.
template <typename T>
__global__ void __launch_bounds__(32) mf_diag_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int k,
                                                     T* __restrict__ ws, float2* __restrict__ inv, T* __restrict__ invc,
                                                     int* __restrict__ piv, int* __restrict__ nperturbed) {
    typedef typename CxT<T>::R R;
    __shared__ T D[MF_NB][MF_NB + 1];
    __shared__ T X[MF_NB][MF_NB + 1];
    const FrontMeta& f = fm[lst[blockIdx.x]];
    if (k >= f.e) return;
    const int kb = min(MF_NB, f.e - k);
    const int lane = threadIdx.x;
    const long long ld = f.n;
    T* W = ws + f.ws + k + (long long)k * ld;
    const T zero = CxT<T>::make(0.0, 0.0);
    R bmax = 0;
    for (int c = 0; c < kb; c++) {
        T v = lane < kb ? W[lane + (long long)c * ld] : zero;
        D[lane][c] = v;
        bmax = max(bmax, cabs2(v));
    }
    for (int o = 16; o > 0; o >>= 1) bmax = max(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    const R floor2 = max(bmax, (R)1e-30) * (R)1e-12;      // (1e-6 of the block's largest entry)^2
    __syncwarp();
    int* P = piv + f.piv + k;
    int pert = 0;
    for (int j = 0; j < kb; j++) {
        // pivot: largest |D[r][j]| for r >= j (ties: smallest r)
        R best = (lane >= j && lane < kb) ? cabs2(D[lane][j]) : (R)-1;
        int br = lane;
        for (int o = 16; o > 0; o >>= 1) {
            R ob = __shfl_xor_sync(0xffffffffu, best, o);
            int orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
        }
        if (lane == 0) P[j] = br;
        if (br != j && lane < kb) {
            T t = D[j][lane];
            D[j][lane] = D[br][lane];
            D[br][lane] = t;
        }
        __syncwarp();
        if (lane == 0 && cabs2(D[j][j]) < floor2) {
            T d = D[j][j];
            R a = sqrt(cabs2(d));
            R fl = sqrt(floor2);
            D[j][j] = a > 0 ? CxT<T>::make(d.x / a * fl, d.y / a * fl) : CxT<T>::make(fl, 0.0);
            pert++;
        }
        __syncwarp();
        T pinv = cinv(D[j][j]);
        if (lane > j && lane < kb) D[lane][j] = cmul(D[lane][j], pinv);
        __syncwarp();
        if (lane > j && lane < kb) {
            T u = D[j][lane];
            for (int r = j + 1; r < kb; r++) cfms(D[r][lane], D[r][j], u);
        }
        __syncwarp();
    }
    if (lane == 0 && pert) atomicAdd(nperturbed, pert);
    // write L\U back
    for (int c = 0; c < kb; c++)
        if (lane < kb) W[lane + (long long)c * ld] = D[lane][c];
    const long long ib = f.inv + (long long)(k / MF_NB) * 2 * MF_NB * MF_NB;   // Linv then Uinv, column-major 32x32
    float2* Li = inv + ib;
    float2* Ui = Li + MF_NB * MF_NB;
    T* Lc = invc + ib;
    T* Uc = Lc + MF_NB * MF_NB;
    constexpr bool wide = sizeof(T) != sizeof(float2);
    // Uinv: lane = column c of X = U^-1 (back substitution, own column only)
    {
        int c = lane;
        for (int i = 0; i < MF_NB; i++) X[i][c] = zero;
        if (c < kb) {
            X[c][c] = cinv(D[c][c]);
            for (int i = c - 1; i >= 0; i--) {
                T s = zero;
                for (int t = i + 1; t <= c; t++) cfma(s, D[i][t], X[t][c]);
                T q = cmul(s, cinv(D[i][i]));
                X[i][c] = CxT<T>::make(-q.x, -q.y);
            }
        }
    }
    __syncwarp();
    for (int c = 0; c < MF_NB; c++) {
        Ui[lane + c * MF_NB] = to_c64(X[lane][c]);
        if (wide) Uc[lane + c * MF_NB] = X[lane][c];
    }
    __syncwarp();
    // Linv: lane = column c of Y = L^-1 (unit lower, forward substitution)
    {
        int c = lane;
        for (int i = 0; i < MF_NB; i++) X[i][c] = zero;
        if (c < kb) {
            X[c][c] = CxT<T>::make(1.0, 0.0);
            for (int i = c + 1; i < kb; i++) {
                T s = zero;
                for (int t = c; t < i; t++) cfma(s, D[i][t], X[t][c]);
                X[i][c] = CxT<T>::make(-s.x, -s.y);
            }
        }
    }
    __syncwarp();
    // the block's row swaps folded into the inverse: w' = P w (swaps j = 0..kb-1 in order) has
    // w'[i] = w[q[i]], so y = Linv w' = (Linv P) w with column q[i] of Linv P = column i of Linv
    int q[MF_NB];
#pragma unroll
    for (int i = 0; i < MF_NB; i++) q[i] = i;
    for (int j = 0; j < kb; j++) {
        int r = P[j];
        int a = 0, b2 = 0;
#pragma unroll
        for (int i = 0; i < MF_NB; i++) { if (i == j) a = q[i]; if (i == r) b2 = q[i]; }
#pragma unroll
        for (int i = 0; i < MF_NB; i++) { if (i == j) q[i] = b2; if (i == r) q[i] = a; }
    }
#pragma unroll
    for (int i = 0; i < MF_NB; i++) {
        Li[lane + q[i] * MF_NB] = to_c64(X[lane][i]);
        if (wide) Lc[lane + q[i] * MF_NB] = X[lane][i];
    }
}

// Block row (columns >= k + kb): row swaps, then L^-1; block column (rows >= k + kb): times U^-1.
// Items 0 .. m-1 are columns, m .. 2m-1 rows (m = n - k - kb).
template <typename T>
__global__ void __launch_bounds__(256) mf_panel_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int k,
                                                       T* __restrict__ ws, const T* __restrict__ invc,
                                                       const int* __restrict__ piv) {
    __shared__ T Li[MF_NB * MF_NB];
    __shared__ T Ui[MF_NB * MF_NB];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (k >= f.e) return;
    const int kb = min(MF_NB, f.e - k);
    const long long m = f.n - k - kb;
    long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if ((long long)blockIdx.x * blockDim.x >= 2 * m) return;
    const T* L = invc + f.inv + (long long)(k / MF_NB) * 2 * MF_NB * MF_NB;
    for (int t = threadIdx.x; t < MF_NB * MF_NB; t += blockDim.x) { Li[t] = L[t]; Ui[t] = L[MF_NB * MF_NB + t]; }
    __syncthreads();
    if (item >= 2 * m) return;
    const long long ld = f.n;
    T* W = ws + f.ws;
    const T zero = CxT<T>::make(0.0, 0.0);
    T v[MF_NB];
    if (item < m) {
        long long c = k + kb + item;
        T* col = W + k + c * ld;
#pragma unroll
        for (int i = 0; i < MF_NB; i++) v[i] = i < kb ? col[i] : zero;
#pragma unroll
        for (int i = 0; i < MF_NB; i++) {
            if (i < kb) {
                T s = zero;
#pragma unroll
                for (int t = 0; t < MF_NB; t++) cfma(s, Li[i + t * MF_NB], v[t]);   // (Linv P) times the column
                col[i] = s;
            }
        }
    } else {
        long long r = k + kb + (item - m);
        T* row = W + r + (long long)k * ld;
#pragma unroll
        for (int i = 0; i < MF_NB; i++) v[i] = i < kb ? row[(long long)i * ld] : zero;
#pragma unroll
        for (int c = 0; c < MF_NB; c++) {
            if (c < kb) {
                T s = zero;
#pragma unroll
                for (int t = 0; t < MF_NB; t++) cfma(s, v[t], Ui[t + c * MF_NB]);
                row[(long long)c * ld] = s;
            }
        }
    }
}

// Trailing update C -= A B on 64 x 64 tiles: A = W[k+kb.., k..k+kb), B = W[k..k+kb, k+kb..).  The k
// extent runs in stages of KH columns (32 for complex64: one stage; 16 for complex128, whose tiles
// would otherwise exceed the static shared-memory limit).
template <typename T>
__global__ void __launch_bounds__(256) mf_trail_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int k,
                                                       T* __restrict__ ws) {
    constexpr int KH = sizeof(T) == sizeof(float2) ? MF_NB : MF_NB / 2;
    __shared__ T As[KH][MF_TILE + 1];
    __shared__ T Bs[KH][MF_TILE + 1];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (k >= f.e) return;
    const int kb = min(MF_NB, f.e - k);
    const long long m = f.n - k - kb;
    const long long nt = (m + MF_TILE - 1) / MF_TILE;
    if ((long long)blockIdx.x >= nt * nt) return;
    const long long ti = blockIdx.x % nt, tj = blockIdx.x / nt;
    const long long r0 = k + kb + ti * MF_TILE, c0 = k + kb + tj * MF_TILE;
    const long long ld = f.n;
    T* W = ws + f.ws;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const T zero = CxT<T>::make(0.0, 0.0);
    T acc[4][4];
    for (int k2 = 0; k2 < kb; k2 += KH) {
        if (k2) __syncthreads();                  // the previous stage's tiles are consumed
        // A tile (64 rows x KH) and B tile (KH x 64 cols) by asynchronous copies; out-of-range parts zeroed
        for (int t = tid; t < KH * MF_TILE; t += 256) {
            int rr = t % MF_TILE, kk = t / MF_TILE;
            long long r = r0 + rr;
            if (k2 + kk < kb && r < f.n) cp_async_c(&As[kk][rr], &W[r + (long long)(k + k2 + kk) * ld]);
            else As[kk][rr] = zero;
            int kk2 = t % KH, cc = t / KH;
            long long c = c0 + cc;
            if (k2 + kk2 < kb && c < f.n) cp_async_c(&Bs[kk2][cc], &W[(k + k2 + kk2) + c * ld]);
            else Bs[kk2][cc] = zero;
        }
        if (k2 == 0) {
            // the thread's 16 C entries go straight into its accumulators while the tiles are in flight
#pragma unroll
            for (int j = 0; j < 4; j++) {
                long long c = c0 + ty + 16 * j;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    long long r = r0 + tx + 16 * i;
                    acc[i][j] = (r < f.n && c < f.n) ? W[r + c * ld] : zero;
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        const int kn = min(KH, kb - k2);
        for (int kk = 0; kk < kn; kk++) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) cfms(acc[i][j], a[i], b[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        long long c = c0 + ty + 16 * j;
        if (c >= f.n) continue;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            long long r = r0 + tx + 16 * i;
            if (r < f.n) W[r + c * ld] = acc[i][j];
        }
    }
}

// Factor columns (n x e) and U block row (e x b), rounded to complex64, and the Schur complement (b x b,
// workspace precision) out of the workspace.
template <typename T>
__global__ void mf_compact_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                  const T* __restrict__ ws, float2* __restrict__ fact, T* __restrict__ upd) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    const long long n = f.n, e = f.e, b = f.b;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= n * n) return;
    long long i1 = min(i0 + MF_CHUNK, n * n);
    const T* W = ws + f.ws;
    float2* F = fact + f.fact;
    T* U = upd + f.upd;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx % n, j = idx / n;
        T v = W[idx];
        if (j < e) F[idx] = to_c64(v);
        else if (i < e) F[n * e + i + (j - e) * e] = to_c64(v);
        else U[(i - e) + (j - e) * b] = v;
    }
}

// ---------------------------------------------------------------- assembly lists on the device
// Every CSR entry (r, c) of the free rows and columns belongs to the front that eliminates the earlier of
// r and c; its local row/column is the DOF's own index there, or e + its index among the front's boundary
// DOFs (sorted by elimination position: binary search).
__device__ __forceinline__ int mf_local(const FrontMeta& f, int v, int d, int p, const int* __restrict__ fpos,
                                        const long long* __restrict__ own0, const int* __restrict__ fdof,
                                        const int* __restrict__ pos) {
    if (fpos[p] == v) return (int)(p - own0[v]);
    int lo = f.e, hi = f.n - 1;
    const int* D = fdof + f.fdof;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (pos[D[mid]] < p) lo = mid + 1; else hi = mid;
    }
    return (lo < f.n && D[lo] == d) ? lo : -1;
}

__global__ void mf_list_count_kernel(long long n, const int* __restrict__ indptr, const int* __restrict__ indices,
                                     const int* __restrict__ pos, const int* __restrict__ fpos, int* __restrict__ cnt) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int pr = pos[r];
    if (pr < 0) return;
    for (int k = indptr[r]; k < indptr[r + 1]; k++) {
        const int pc = pos[indices[k]];
        if (pc < 0) continue;
        atomicAdd(&cnt[fpos[min(pr, pc)]], 1);
    }
}

__global__ void mf_list_fill_kernel(long long n, const int* __restrict__ indptr, const int* __restrict__ indices,
                                    const int* __restrict__ pos, const int* __restrict__ fpos,
                                    const long long* __restrict__ own0, const FrontMeta* __restrict__ fm,
                                    const int* __restrict__ fdof, const int* __restrict__ base, int* __restrict__ cur,
                                    int* __restrict__ slot, int* __restrict__ off, int* __restrict__ status) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int pr = pos[r];
    if (pr < 0) return;
    for (int k = indptr[r]; k < indptr[r + 1]; k++) {
        const int c = indices[k];
        const int pc = pos[c];
        if (pc < 0) continue;
        const int v = fpos[min(pr, pc)];
        const FrontMeta& f = fm[v];
        const int li = mf_local(f, v, (int)r, pr, fpos, own0, fdof, pos);
        const int lj = mf_local(f, v, c, pc, fpos, own0, fdof, pos);
        const int q = base[v] + atomicAdd(&cur[v], 1);
        if (li < 0 || lj < 0) {
            flag(status, DEV_BAD_INDEX);
            slot[q] = k;
            off[q] = 0;
            continue;
        }
        slot[q] = k;
        off[q] = li + lj * f.n;
    }
}

// ---------------------------------------------------------------- solve kernels
// w (rows of the level's fronts, S per row): own rows from the right-hand side, boundary rows zero
__global__ void mf_fwd_gather_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S,
                                     const int* __restrict__ fdof, const double* __restrict__ scale,
                                     const double2* __restrict__ rhs, float2* __restrict__ w) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long tot = (long long)f.n * S;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    float2* W = w + f.wv * S;
    const int* d = fdof + f.fdof;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx / S;
        int s = (int)(idx % S);
        float2 v = make_float2(0.f, 0.f);
        if (i < f.e) {
            double2 r = rhs[(long long)d[i] * S + s];
            double sc = scale[d[i]];
            v = make_float2((float)(r.x * sc), (float)(r.y * sc));
        }
        W[idx] = v;
    }
}

__global__ void mf_fwd_ea_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S, int cslot,
                                 const int* __restrict__ ea, const float2* __restrict__ uvec, float2* __restrict__ w) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    int c = f.child[cslot];
    if (c < 0) return;
    const FrontMeta& g = fm[c];
    long long tot = (long long)g.b * S;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    const int* map = ea + g.ea;
    const float2* U = uvec + g.uv * S;
    float2* W = w + f.wv * S;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx / S;
        int s = (int)(idx % S);
        float2 u = U[idx];
        float2* p = W + (long long)map[i] * S + s;
        p->x += u.x;
        p->y += u.y;
    }
}

// Forward solve inside the 256-row block [k0, k1) of the own rows, held in shared memory: for each
// 32-step y = (Linv P) w_step, then the block's remaining rows.  One CTA per front, 16 right-hand sides
// at a time.  Each step's inverse block and L panel (the block's rows below the step, 32 columns) are
// first staged in shared memory with coalesced loads, so a step costs one global round trip.
constexpr int MF_SC = 16;
constexpr int MF_PAN = MF_SB - MF_NB;     // panel rows below a step inside the block
template <int NBUF>
struct MfBlockSmem {
    float2 wb[MF_SB][MF_SC];
    float2 y[MF_NB][MF_SC];
    float2 li[NBUF][MF_NB * MF_NB];
    float2 pan[NBUF][MF_PAN][MF_NB + 1];
};
constexpr size_t MF_BLOCK_SMEM = sizeof(MfBlockSmem<1>);
constexpr size_t MF_BLOCK_SMEM2 = sizeof(MfBlockSmem<2>);

// Stage step st's inverse block and panel (forward: rows below the step inside the block; backward: rows
// above it) into buffer slot, as one committed group of asynchronous copies.
__device__ __forceinline__ void mf_stage_step(float2* li, float2 (*pan)[MF_NB + 1], const float2* Ib,
                                              const float2* F, long long n, int rbase, int pr, int kcol, int kb) {
    for (int t = threadIdx.x; t < MF_NB * MF_NB; t += blockDim.x) cp_async8(&li[t], &Ib[t]);
    for (int t = threadIdx.x; t < pr * kb; t += blockDim.x) {
        int c = t / pr, r = t - c * pr;          // consecutive threads: consecutive rows of one column
        cp_async8(&pan[r][c], &F[(rbase + r) + (long long)(kcol + c) * n]);
    }
    cp_async_commit();
}

// NT threads: 256 on levels of many fronts (several CTAs per SM), 1024 on levels of few fronts, where the
// block chain of one front is serial and a step's items (rows x right-hand sides) spread over more threads.
constexpr int MF_BLOCK_NT_FEW = 1024;
template <int NBUF, int NT>
__global__ void __launch_bounds__(NT) mf_fwd_block_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                           int S, int k0, const float2* __restrict__ fact,
                                                           const float2* __restrict__ inv, float2* __restrict__ w) {
    extern __shared__ __align__(16) unsigned char mf_smem[];
    MfBlockSmem<NBUF>& sm = *reinterpret_cast<MfBlockSmem<NBUF>*>(mf_smem);
    const FrontMeta& f = fm[lst[blockIdx.x]];
    if (k0 >= f.e) return;
    const int k1 = min(k0 + MF_SB, f.e);
    const int rows = k1 - k0;
    const int nsteps = (rows + MF_NB - 1) / MF_NB;
    const long long n = f.n;
    float2* W = w + f.wv * S;
    const float2* F = fact + f.fact;
    const int tid = threadIdx.x;
    auto stage = [&](int st) {
        const int k = k0 + st * MF_NB, kb = min(MF_NB, f.e - k);
        mf_stage_step(sm.li[st % NBUF], sm.pan[st % NBUF], inv + f.inv + (long long)(k / MF_NB) * 2 * MF_NB * MF_NB,
                      F, n, k + kb, k1 - k - kb, k, kb);
    };
    for (int sc = 0; sc < S; sc += MF_SC) {
        const int ns = min(MF_SC, S - sc);
        for (int t = tid; t < rows * ns; t += blockDim.x)
            cp_async8(&sm.wb[t / ns][t % ns], &W[(long long)(k0 + t / ns) * S + sc + t % ns]);
        stage(0);
        for (int st = 0; st < nsteps; st++) {
            const int k = k0 + st * MF_NB, kb = min(MF_NB, f.e - k), pr = k1 - k - kb;
            if (NBUF == 2 && st + 1 < nsteps) {
                stage(st + 1);                   // the next step's copies fly while this step computes
                cp_async_wait_1();
            } else {
                cp_async_wait_all();
            }
            __syncthreads();
            const float2* li = sm.li[st % NBUF];
            for (int t = tid; t < kb * ns; t += blockDim.x) {
                int i = t / ns, sj = t % ns;
                float2 acc = make_float2(0.f, 0.f);
                for (int c = 0; c < kb; c++) cfma(acc, li[i + c * MF_NB], sm.wb[k - k0 + c][sj]);
                sm.y[i][sj] = acc;
            }
            __syncthreads();
            for (int t = tid; t < kb * ns; t += blockDim.x) sm.wb[k - k0 + t / ns][t % ns] = sm.y[t / ns][t % ns];
            for (int t = tid; t < pr * ns; t += blockDim.x) {
                int r = t / ns, sj = t % ns;
                float2 acc = sm.wb[k + kb - k0 + r][sj];
                for (int c = 0; c < kb; c++) cfms(acc, sm.pan[st % NBUF][r][c], sm.y[c][sj]);
                sm.wb[k + kb - k0 + r][sj] = acc;
            }
            __syncthreads();
            if (NBUF == 1 && st + 1 < nsteps) stage(st + 1);
        }
        for (int t = tid; t < rows * ns; t += blockDim.x) W[(long long)(k0 + t / ns) * S + sc + t % ns] = sm.wb[t / ns][t % ns];
        __syncthreads();
    }
}

// w[r] -= sum_{c in [c0, c1)} M[r, c] x[c] for the rows [r0, r1) of a front, M column-major with leading
// dimension ldm, x = rows c of w (or of xsrc).  A CTA owns 32 rows; its 8 warps take every 8th column
// and their sums meet in shared memory.  8 right-hand sides per CTA (grid.z).
// RPL row sets per lane: lane rl of warp g holds rows rb + rl + 32 i (i < RPL), so a warp streams
// 32 * RPL consecutive rows (256 * RPL contiguous bytes) of every column it visits, with RPL loads in
// flight per column.  Each row sums its columns in the same order as with one row set (bit-identical).
constexpr int MF_RPL = 2;
template <int RPL>
__device__ __forceinline__ void mf_gemv_rowsets(float2* W, int S, long long rb, int rl, int g, long long rlim,
                                                const float2* M, long long ldm, long long c0, long long c1,
                                                const float2* X, long long xrow0, int s0, int ns,
                                                float2 (*red)[32 * RPL][8]) {
    float2 acc[RPL][8];
#pragma unroll
    for (int i = 0; i < RPL; i++)
#pragma unroll
        for (int q = 0; q < 8; q++) acc[i][q] = make_float2(0.f, 0.f);
    bool live[RPL];
#pragma unroll
    for (int i = 0; i < RPL; i++) live[i] = rb + rl + 32 * i < rlim;
    if (live[0]) {
#pragma unroll 4
        for (long long c = c0 + g; c < c1; c += 8) {
            float2 mv[RPL];
#pragma unroll
            for (int i = 0; i < RPL; i++) mv[i] = live[i] ? M[rb + rl + 32 * i + c * ldm] : make_float2(0.f, 0.f);
            const float2* xc = X + (xrow0 + c - c0) * S + s0;
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < ns) {
                    const float2 xv = xc[q];
#pragma unroll
                    for (int i = 0; i < RPL; i++) cfma(acc[i][q], mv[i], xv);
                }
        }
    }
#pragma unroll
    for (int i = 0; i < RPL; i++)
#pragma unroll
        for (int q = 0; q < 8; q++) red[g][rl + 32 * i][q] = acc[i][q];
    __syncthreads();
    if (g < RPL && live[g]) {
        const long long r = rb + rl + 32 * g;
        for (int q = 0; q < ns; q++) {
            float2 t = make_float2(0.f, 0.f);
#pragma unroll
            for (int gg = 0; gg < 8; gg++) { t.x += red[gg][rl + 32 * g][q].x; t.y += red[gg][rl + 32 * g][q].y; }
            float2* p = W + r * S + s0 + q;
            p->x -= t.x;
            p->y -= t.y;
        }
    }
}

// Rows [k1, n) of every front: w[r] -= L[r, k0:k1] y[k0:k1]
__global__ void __launch_bounds__(256) mf_fwd_update_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                            int S, int k0, const float2* __restrict__ fact,
                                                            float2* __restrict__ w) {
    __shared__ float2 red[8][32 * MF_RPL][8];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (k0 >= f.e) return;
    const int k1 = min(k0 + MF_SB, f.e);
    const long long r0 = k1 + (long long)blockIdx.x * 32 * MF_RPL;
    if (r0 >= f.n) return;
    const int s0 = blockIdx.z * 8, ns = min(8, S - s0);
    const int rl = threadIdx.x % 32, g = threadIdx.x / 32;
    float2* W = w + f.wv * S;
    mf_gemv_rowsets<MF_RPL>(W, S, r0, rl, g, f.n, fact + f.fact, f.n, k0, k1, W, k0, s0, ns, red);
}

// own rows -> y store, boundary rows -> update vector for the parent
__global__ void mf_fwd_finish_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S,
                                     const float2* __restrict__ w, float2* __restrict__ ystore, float2* __restrict__ uvec) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long tot = (long long)f.n * S;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    const float2* W = w + f.wv * S;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx / S;
        if (i < f.e) ystore[f.y * S + idx] = W[idx];
        else uvec[f.uv * S + (idx - (long long)f.e * S)] = W[idx];
    }
}

// backward: own rows from y, boundary rows from the solved x (FP32, DOF order)
__global__ void mf_bwd_gather_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S,
                                     const int* __restrict__ fdof, const float2* __restrict__ ystore,
                                     const float2* __restrict__ xs, float2* __restrict__ w) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long tot = (long long)f.n * S;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    float2* W = w + f.wv * S;
    const int* d = fdof + f.fdof;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx / S;
        int s = (int)(idx % S);
        W[idx] = i < f.e ? ystore[f.y * S + idx] : xs[(long long)d[i] * S + s];
    }
}

// own rows: w[r] -= U12[r, :] x_bnd   (U12 is e x b, column-major with ld e; x_bnd = rows e.. of w)
// The same U12 product split over the boundary columns for fronts with long boundaries: CTA (row group,
// column chunk of MF_CW) writes its partial sums to part[chunk][level row][S]; mf_bwd_bnd_sum_kernel
// then subtracts the chunks in ascending order (deterministic).  A front's own rows [0, e) of its
// level rows f.wv .. f.wv + n index the partials; chunks past the front's boundary write zeros.
constexpr int MF_CW = 512;
__global__ void __launch_bounds__(256) mf_bwd_bnd_split_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                               int S, int nrg, long long wvl,
                                                               const float2* __restrict__ fact,
                                                               const float2* __restrict__ w, float2* __restrict__ part) {
    __shared__ float2 red[8][32 * MF_RPL][8];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (f.b == 0) return;
    const int rg = blockIdx.x % nrg, sp = blockIdx.x / nrg;
    const long long r0 = (long long)rg * 32 * MF_RPL;
    if (r0 >= f.e) return;
    const int s0 = blockIdx.z * 8, ns = min(8, S - s0);
    const int rl = threadIdx.x % 32, g = threadIdx.x / 32;
    const float2* W = w + f.wv * S;
    const float2* M = fact + f.fact + (long long)f.n * f.e;
    const long long c0 = min((long long)sp * MF_CW, (long long)f.b), c1 = min(c0 + MF_CW, (long long)f.b);
    float2 acc[MF_RPL][8];
    bool live[MF_RPL];
#pragma unroll
    for (int i = 0; i < MF_RPL; i++) {
        live[i] = r0 + rl + 32 * i < f.e;
#pragma unroll
        for (int q = 0; q < 8; q++) acc[i][q] = make_float2(0.f, 0.f);
    }
    if (live[0]) {
#pragma unroll 4
        for (long long c = c0 + g; c < c1; c += 8) {
            float2 mv[MF_RPL];
#pragma unroll
            for (int i = 0; i < MF_RPL; i++) mv[i] = live[i] ? M[r0 + rl + 32 * i + c * f.e] : make_float2(0.f, 0.f);
            const float2* xc = W + (f.e + c) * S + s0;
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < ns) {
                    const float2 xv = xc[q];
#pragma unroll
                    for (int i = 0; i < MF_RPL; i++) cfma(acc[i][q], mv[i], xv);
                }
        }
    }
#pragma unroll
    for (int i = 0; i < MF_RPL; i++)
#pragma unroll
        for (int q = 0; q < 8; q++) red[g][rl + 32 * i][q] = acc[i][q];
    __syncthreads();
    if (g < MF_RPL && live[g]) {
        const long long r = r0 + rl + 32 * g;
        float2* P = part + ((long long)sp * wvl + f.wv + r) * S + s0;
        for (int q = 0; q < ns; q++) {
            float2 t = make_float2(0.f, 0.f);
#pragma unroll
            for (int gg = 0; gg < 8; gg++) { t.x += red[gg][rl + 32 * g][q].x; t.y += red[gg][rl + 32 * g][q].y; }
            P[q] = t;
        }
    }
}

__global__ void mf_bwd_bnd_sum_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S, int nsplit,
                                      long long wvl, const float2* __restrict__ part, float2* __restrict__ w) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (f.b == 0) return;
    const long long tot = (long long)f.e * S;
    const long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    const long long i1 = min(i0 + MF_CHUNK, tot);
    float2* W = w + f.wv * S;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        float2 t = make_float2(0.f, 0.f);
        for (int sp = 0; sp < nsplit; sp++) {
            float2 v = part[((long long)sp * wvl + f.wv) * S + idx];
            t.x += v.x;
            t.y += v.y;
        }
        W[idx].x -= t.x;
        W[idx].y -= t.y;
    }
}

__global__ void __launch_bounds__(256) mf_bwd_bnd_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                         int S, const float2* __restrict__ fact, float2* __restrict__ w) {
    __shared__ float2 red[8][32 * MF_RPL][8];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (f.b == 0) return;
    const long long r0 = (long long)blockIdx.x * 32 * MF_RPL;
    if (r0 >= f.e) return;
    const int s0 = blockIdx.z * 8, ns = min(8, S - s0);
    const int rl = threadIdx.x % 32, g = threadIdx.x / 32;
    float2* W = w + f.wv * S;
    mf_gemv_rowsets<MF_RPL>(W, S, r0, rl, g, f.e, fact + f.fact + (long long)f.n * f.e, f.e, 0, f.b, W, f.e, s0, ns,
                            red);
}

// Backward solve inside the block [k0, k1), held in shared memory: 32-steps from the last,
// x_k = Uinv (w_k), then the block's earlier rows.  One CTA per front, 16 right-hand sides at a time;
// each step's Uinv block and U panel (the block's rows above the step) staged in shared memory first.
template <int NBUF, int NT>
__global__ void __launch_bounds__(NT) mf_bwd_block_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                           int S, int k0, const float2* __restrict__ fact,
                                                           const float2* __restrict__ inv, float2* __restrict__ w) {
    extern __shared__ __align__(16) unsigned char mf_smem[];
    MfBlockSmem<NBUF>& sm = *reinterpret_cast<MfBlockSmem<NBUF>*>(mf_smem);
    const FrontMeta& f = fm[lst[blockIdx.x]];
    if (k0 >= f.e) return;
    const int k1 = min(k0 + MF_SB, f.e);
    const int rows = k1 - k0;
    const long long n = f.n;
    float2* W = w + f.wv * S;
    const float2* F = fact + f.fact;
    const int tid = threadIdx.x;
    const int nsteps = (rows + MF_NB - 1) / MF_NB;
    // processing order j = 0.. runs the steps from the last (st = nsteps - 1 - j); buffers follow j
    auto stage = [&](int j) {
        const int k = k0 + (nsteps - 1 - j) * MF_NB, kb = min(MF_NB, f.e - k);
        mf_stage_step(sm.li[j % NBUF], sm.pan[j % NBUF],
                      inv + f.inv + (long long)(k / MF_NB) * 2 * MF_NB * MF_NB + MF_NB * MF_NB, F, n, k0, k - k0, k, kb);
    };
    for (int sc = 0; sc < S; sc += MF_SC) {
        const int ns = min(MF_SC, S - sc);
        for (int t = tid; t < rows * ns; t += blockDim.x)
            cp_async8(&sm.wb[t / ns][t % ns], &W[(long long)(k0 + t / ns) * S + sc + t % ns]);
        stage(0);
        for (int j = 0; j < nsteps; j++) {
            const int k = k0 + (nsteps - 1 - j) * MF_NB, kb = min(MF_NB, f.e - k), pr = k - k0;
            if (NBUF == 2 && j + 1 < nsteps) {
                stage(j + 1);
                cp_async_wait_1();
            } else {
                cp_async_wait_all();
            }
            __syncthreads();
            const float2* ui = sm.li[j % NBUF];
            for (int t = tid; t < kb * ns; t += blockDim.x) {
                int i = t / ns, sj = t % ns;
                float2 acc = make_float2(0.f, 0.f);
                for (int c = i; c < kb; c++) cfma(acc, ui[i + c * MF_NB], sm.wb[k - k0 + c][sj]);
                sm.y[i][sj] = acc;
            }
            __syncthreads();
            for (int t = tid; t < kb * ns; t += blockDim.x) sm.wb[k - k0 + t / ns][t % ns] = sm.y[t / ns][t % ns];
            for (int t = tid; t < pr * ns; t += blockDim.x) {
                int r = t / ns, sj = t % ns;
                float2 acc = sm.wb[r][sj];
                for (int c = 0; c < kb; c++) cfms(acc, sm.pan[j % NBUF][r][c], sm.y[c][sj]);
                sm.wb[r][sj] = acc;
            }
            __syncthreads();
            if (NBUF == 1 && j + 1 < nsteps) stage(j + 1);
        }
        for (int t = tid; t < rows * ns; t += blockDim.x) W[(long long)(k0 + t / ns) * S + sc + t % ns] = sm.wb[t / ns][t % ns];
        __syncthreads();
    }
}

// rows [0, k0): w[r] -= U[r, k0:k1] x[k0:k1]
__global__ void __launch_bounds__(256) mf_bwd_update_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm,
                                                            int S, int k0, const float2* __restrict__ fact,
                                                            float2* __restrict__ w) {
    __shared__ float2 red[8][32 * MF_RPL][8];
    const FrontMeta& f = fm[lst[blockIdx.y]];
    if (k0 >= f.e) return;
    const int k1 = min(k0 + MF_SB, f.e);
    const long long r0 = (long long)blockIdx.x * 32 * MF_RPL;
    if (r0 >= k0) return;
    const int s0 = blockIdx.z * 8, ns = min(8, S - s0);
    const int rl = threadIdx.x % 32, g = threadIdx.x / 32;
    float2* W = w + f.wv * S;
    mf_gemv_rowsets<MF_RPL>(W, S, r0, rl, g, k0, fact + f.fact, f.n, k0, k1, W, k0, s0, ns, red);
}

__global__ void mf_bwd_finish_kernel(const int* __restrict__ lst, const FrontMeta* __restrict__ fm, int S,
                                     const int* __restrict__ fdof, const float2* __restrict__ w, float2* __restrict__ xs) {
    const FrontMeta& f = fm[lst[blockIdx.y]];
    long long tot = (long long)f.e * S;
    long long i0 = (long long)blockIdx.x * MF_CHUNK;
    if (i0 >= tot) return;
    long long i1 = min(i0 + MF_CHUNK, tot);
    const float2* W = w + f.wv * S;
    const int* d = fdof + f.fdof;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        long long i = idx / S;
        int s = (int)(idx % S);
        xs[(long long)d[i] * S + s] = W[idx];
    }
}

__global__ void mf_fill_kernel(long long n, double v, double* __restrict__ x) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) x[g] = v;
}

// x = D^-1/2 (scaled solution), zero outside every front
__global__ void mf_out_kernel(long long n, int S, const uint8_t* __restrict__ freed, const double* __restrict__ scale,
                              const float2* __restrict__ xs, double2* __restrict__ x) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * S) return;
    float2 v = xs[g];
    const double sc = scale[g / S];
    x[g] = freed[g / S] ? make_double2((double)v.x * sc, (double)v.y * sc) : make_double2(0.0, 0.0);
}

}  // namespace emfem

using namespace emfem;

struct emfem_mf_s {
    Handle* h = nullptr;
    long long n = 0;
    int nf = 0;
    std::vector<FrontMeta> meta;                  // host copy
    std::vector<std::vector<int>> levels;         // fronts per level
    std::vector<long long> lvl_off;               // offsets of each level's list in d_lst
    std::vector<int> lvl_max_e, lvl_max_n;
    std::vector<long long> lvl_max_asm, lvl_max_b;
    FrontMeta* d_meta = nullptr;
    int* d_lst = nullptr;
    int* d_fdof = nullptr;
    int* d_ea = nullptr;
    int* d_slot = nullptr;
    int* d_off = nullptr;
    uint8_t* d_free = nullptr;                    // 1 where a DOF belongs to some front
    double* d_scale = nullptr;                    // equilibration D^-1/2 of the current factorization
    float2* fact = nullptr;
    float2* inv = nullptr;
    int* piv = nullptr;
    void* ws = nullptr;                           // level workspace, complex64 or (wide) complex128
    void* upd = nullptr;                          // update store, same precision as ws
    void* invc = nullptr;                         // complex128 copies of the inverse blocks (wide only)
    bool wide = false;                            // fronts factored in complex128
    int* d_npert = nullptr;
    long long fact_n = 0, inv_n = 0, piv_n = 0, ws_n = 0, upd_n = 0;
    long long wv_n = 0, uv_n = 0, y_n = 0;        // solve buffer rows
    std::vector<long long> lvl_wv, lvl_max_ob;    // per level: its fronts' rows (sum of n), largest own boundary
    long long part_n = 0;                         // split U12 partials: max over levels of chunks x level rows
    float2* spart = nullptr;                      // (part_n, S) partial sums of the split backward products
    // solve buffers for the current S
    int S = 0;
    float2 *sw = nullptr, *suv = nullptr, *sy = nullptr, *sx = nullptr;
    double flops = 0.0;
    bool factored = false;
    bool lists = false;                           // assembly lists present (given or built)
    std::vector<int> h_pos, h_fpos;               // host copies used to build the lists on the device
    std::vector<long long> h_own0;
};

static void mf_free(emfem_mf_s* m) {
    void* ps[] = {m->d_meta, m->d_lst, m->d_fdof, m->d_ea, m->d_slot, m->d_off, m->d_free, m->d_scale, m->fact, m->inv, m->piv,
                  m->ws, m->upd, m->invc, m->d_npert, m->sw, m->suv, m->sy, m->sx, m->spart};
    for (void* p : ps)
        if (p) cudaFree(p);
}

static inline unsigned nblk(long long items, long long per) {
    long long g = (items + per - 1) / per;
    return (unsigned)std::max(1LL, g);
}

static int mf_reserve(emfem_mf_s* m, int S) {
    if (m->S >= S) return EMFEM_OK;
    void* ps[] = {m->sw, m->suv, m->sy, m->sx, m->spart};
    for (void* p : ps)
        if (p) cudaFree(p);
    m->sw = m->suv = m->sy = m->sx = m->spart = nullptr;
    m->S = 0;
    if (m->part_n > 0) EMFEM_CUDA(cudaMalloc(&m->spart, sizeof(float2) * m->part_n * S));
    EMFEM_CUDA(cudaMalloc(&m->sw, sizeof(float2) * std::max(1LL, m->wv_n) * S));
    EMFEM_CUDA(cudaMalloc(&m->suv, sizeof(float2) * std::max(1LL, m->uv_n) * S));
    EMFEM_CUDA(cudaMalloc(&m->sy, sizeof(float2) * std::max(1LL, m->y_n) * S));
    EMFEM_CUDA(cudaMalloc(&m->sx, sizeof(float2) * m->n * S));
    m->S = S;
    return EMFEM_OK;
}

namespace emfem {
int mf_reserved(const emfem_mf_s* m) { return m ? m->S : 0; }

// M^-1 r for S right-hand sides (n, S) FP64 DOF-major -> x (FP64), zero on DOFs outside every front.
int mf_apply(emfem_mf_s* m, int S, const double2* r, double2* x, cudaStream_t s) {
    EMFEM_REQUIRE(m->factored, "emfem_mf: solve before a successful factorization");
    if (m->S < S) {
        set_error("emfem_mf: %d right-hand sides exceed the reserved %d (emfem_mf_reserve)", S, m->S);
        return EMFEM_ERR_INVALID_ARG;
    }
    const int nl = (int)m->levels.size();
    EMFEM_CUDA(cudaMemsetAsync(m->sx, 0, sizeof(float2) * m->n * S, s));
    for (int L = 0; L < nl; L++) {
        const int nfl = (int)m->levels[L].size();
        const int* lst = m->d_lst + m->lvl_off[L];
        long long maxn = m->lvl_max_n[L], maxb = m->lvl_max_b[L];
        for (int y0 = 0; y0 < nfl; y0 += 65535) {
            const int ny = std::min(65535, nfl - y0);
            dim3 g(nblk(maxn * S, MF_CHUNK), ny);
            mf_fwd_gather_kernel<<<g, 256, 0, s>>>(lst + y0, m->d_meta, S, m->d_fdof, m->d_scale, r, m->sw);
            dim3 ge(nblk(maxb * S, MF_CHUNK), ny);
            mf_fwd_ea_kernel<<<ge, 256, 0, s>>>(lst + y0, m->d_meta, S, 0, m->d_ea, m->suv, m->sw);
            mf_fwd_ea_kernel<<<ge, 256, 0, s>>>(lst + y0, m->d_meta, S, 1, m->d_ea, m->suv, m->sw);
            const unsigned sz = (unsigned)((S + 7) / 8);
            for (int k0 = 0; k0 < m->lvl_max_e[L]; k0 += MF_SB) {
                if (ny < 148)   // a few large fronts: the serial step chain, so overlap its copies
                    mf_fwd_block_kernel<2, MF_BLOCK_NT_FEW><<<ny, MF_BLOCK_NT_FEW, MF_BLOCK_SMEM2, s>>>(
                        lst + y0, m->d_meta, S, k0, m->fact, m->inv, m->sw);
                else
                    mf_fwd_block_kernel<1, 256><<<ny, 256, MF_BLOCK_SMEM, s>>>(lst + y0, m->d_meta, S, k0, m->fact, m->inv, m->sw);
                dim3 gu(nblk(maxn - k0, 32 * MF_RPL), ny, sz);   // rows [k1, n) of a front: at most n - k0
                mf_fwd_update_kernel<<<gu, 256, 0, s>>>(lst + y0, m->d_meta, S, k0, m->fact, m->sw);
            }
            mf_fwd_finish_kernel<<<g, 256, 0, s>>>(lst + y0, m->d_meta, S, m->sw, m->sy, m->suv);
        }
        EMFEM_LAUNCH("multifrontal forward");
    }
    for (int L = nl - 1; L >= 0; L--) {
        const int nfl = (int)m->levels[L].size();
        const int* lst = m->d_lst + m->lvl_off[L];
        long long maxn = m->lvl_max_n[L];
        long long maxe = m->lvl_max_e[L];
        for (int y0 = 0; y0 < nfl; y0 += 65535) {
            const int ny = std::min(65535, nfl - y0);
            dim3 g(nblk(maxn * S, MF_CHUNK), ny);
            mf_bwd_gather_kernel<<<g, 256, 0, s>>>(lst + y0, m->d_meta, S, m->d_fdof, m->sy, m->sx, m->sw);
            const unsigned sz = (unsigned)((S + 7) / 8);
            const long long nsplit = (m->lvl_max_ob[L] + MF_CW - 1) / MF_CW;
            if (nsplit > 1 && nfl < 148) {
                const unsigned nrg = nblk(maxe, 32 * MF_RPL);
                dim3 gb(nrg * (unsigned)nsplit, ny, sz);
                mf_bwd_bnd_split_kernel<<<gb, 256, 0, s>>>(lst + y0, m->d_meta, S, (int)nrg, m->lvl_wv[L], m->fact,
                                                          m->sw, m->spart);
                dim3 gs(nblk(maxe * S, MF_CHUNK), ny);
                mf_bwd_bnd_sum_kernel<<<gs, 256, 0, s>>>(lst + y0, m->d_meta, S, (int)nsplit, m->lvl_wv[L], m->spart,
                                                        m->sw);
            } else {
                dim3 gb(nblk(maxe, 32 * MF_RPL), ny, sz);
                mf_bwd_bnd_kernel<<<gb, 256, 0, s>>>(lst + y0, m->d_meta, S, m->fact, m->sw);
            }
            const int nblocks = (int)((maxe + MF_SB - 1) / MF_SB);
            for (int bi = nblocks - 1; bi >= 0; bi--) {
                const int k0 = bi * MF_SB;
                if (ny < 148)
                    mf_bwd_block_kernel<2, MF_BLOCK_NT_FEW><<<ny, MF_BLOCK_NT_FEW, MF_BLOCK_SMEM2, s>>>(
                        lst + y0, m->d_meta, S, k0, m->fact, m->inv, m->sw);
                else
                    mf_bwd_block_kernel<1, 256><<<ny, 256, MF_BLOCK_SMEM, s>>>(lst + y0, m->d_meta, S, k0, m->fact, m->inv, m->sw);
                if (k0 > 0) {
                    dim3 gu(nblk(k0, 32 * MF_RPL), ny, sz);
                    mf_bwd_update_kernel<<<gu, 256, 0, s>>>(lst + y0, m->d_meta, S, k0, m->fact, m->sw);
                }
            }
            dim3 gf(nblk(maxe * S, MF_CHUNK), ny);
            mf_bwd_finish_kernel<<<gf, 256, 0, s>>>(lst + y0, m->d_meta, S, m->d_fdof, m->sw, m->sx);
        }
        EMFEM_LAUNCH("multifrontal backward");
    }
    mf_out_kernel<<<grid_for(m->n * S, 256), 256, 0, s>>>(m->n, S, m->d_free, m->d_scale, m->sx, x);
    EMFEM_LAUNCH("mf_out_kernel");
    return EMFEM_OK;
}
}  // namespace emfem

// The level loop of one factorization, fronts in workspace precision T.
template <typename T>
static int mf_factor_levels(emfem_mf_s* m, const double2* K_vals, cudaStream_t s) {
    T* ws = (T*)m->ws;
    T* upd = (T*)m->upd;
    T* invc = m->wide ? (T*)m->invc : (T*)m->inv;
    int rc = EMFEM_OK;
    const int nl = (int)m->levels.size();
    for (int L = 0; L < nl && rc == EMFEM_OK; L++) {
        const int nfl = (int)m->levels[L].size();
        long long wsz = 0;
        for (int v : m->levels[L]) wsz += (long long)m->meta[v].n * m->meta[v].n;
        rc = check_cuda(cudaMemsetAsync(ws, 0, sizeof(T) * wsz, s), "cudaMemsetAsync");
        for (int y0 = 0; y0 < nfl && rc == EMFEM_OK; y0 += 65535) {
            const int ny = std::min(65535, nfl - y0);
            const int* lst = m->d_lst + m->lvl_off[L] + y0;
            long long maxn = m->lvl_max_n[L], maxb = m->lvl_max_b[L];
            mf_asm_kernel<T><<<dim3(nblk(m->lvl_max_asm[L], MF_CHUNK), ny), 256, 0, s>>>(
                lst, m->d_meta, K_vals, m->d_slot, m->d_off, m->d_fdof, m->d_scale, ws);
            for (int c = 0; c < 2; c++)
                mf_ea_kernel<T><<<dim3(nblk(maxb * maxb, MF_CHUNK), ny), 256, 0, s>>>(lst, m->d_meta, c, m->d_ea, upd, ws);
            for (int k = 0; k < m->lvl_max_e[L]; k += MF_NB) {
                mf_diag_kernel<T><<<ny, 32, 0, s>>>(lst, m->d_meta, k, ws, m->inv, invc, m->piv, m->d_npert);
                long long mm = maxn - k - 1;
                if (mm < 1) mm = 1;
                mf_panel_kernel<T><<<dim3(nblk(2 * mm, 256), ny), 256, 0, s>>>(lst, m->d_meta, k, ws, invc, m->piv);
                long long nt = (mm + MF_TILE - 1) / MF_TILE;
                mf_trail_kernel<T><<<dim3((unsigned)std::max(1LL, nt * nt), ny), 256, 0, s>>>(lst, m->d_meta, k, ws);
            }
            mf_compact_kernel<T><<<dim3(nblk(maxn * maxn, MF_CHUNK), ny), 256, 0, s>>>(lst, m->d_meta, ws, m->fact, upd);
            rc = check_cuda(cudaGetLastError(), "multifrontal factor level");
        }
    }
    return rc;
}


extern "C" {

int emfem_mf_create(emfem_handle h, int64_t n, int n_fronts, const int32_t* e, const int32_t* b, const int32_t* parent,
                    const int32_t* level, const int64_t* fdof_ptr, const int32_t* fdof, const int32_t* ea,
                    const int64_t* asm_ptr, const int32_t* asm_slot, const int32_t* asm_off, emfem_mf* out) {
    EMFEM_REQUIRE(h && n > 0 && n_fronts > 0 && e && b && parent && level && fdof_ptr && fdof && ea && out,
                  "emfem_mf_create: bad argument");
    EMFEM_REQUIRE((asm_ptr && asm_slot && asm_off) || (!asm_ptr && !asm_slot && !asm_off),
                  "emfem_mf_create: give all three assembly arrays or none (then emfem_mf_build_lists)");
    auto* m = new emfem_mf_s();
    m->h = &h->h;
    m->n = n;
    m->nf = n_fronts;
    m->meta.resize(n_fronts);
    int nl = 0;
    long long tot_fdof = 0;
    for (int v = 0; v < n_fronts; v++) {
        if (e[v] < 0 || b[v] < 0 || e[v] + b[v] > MF_MAX_FRONT || level[v] < 0 || parent[v] >= n_fronts ||
            (parent[v] >= 0 && parent[v] <= v) || fdof_ptr[v + 1] - fdof_ptr[v] != (long long)e[v] + b[v]) {
            delete m;
            set_error("emfem_mf_create: front %d is inconsistent (e %d, b %d, parent %d)", v, e[v], b[v], parent[v]);
            return EMFEM_ERR_INVALID_ARG;
        }
        nl = std::max(nl, level[v] + 1);
        tot_fdof += e[v] + b[v];
    }
    m->levels.assign(nl, {});
    for (int v = 0; v < n_fronts; v++) m->levels[level[v]].push_back(v);
    // offsets
    long long fact = 0, inv = 0, pivo = 0, eao = 0, y = 0;
    for (int v = 0; v < n_fronts; v++) {
        FrontMeta& f = m->meta[v];
        f.e = e[v]; f.b = b[v]; f.n = e[v] + b[v]; f.parent = parent[v];
        f.child[0] = f.child[1] = -1;
        f.fdof = fdof_ptr[v];
        f.ea = eao; eao += b[v];
        f.asm0 = asm_ptr ? asm_ptr[v] : 0; f.asm1 = asm_ptr ? asm_ptr[v + 1] : 0;
        f.fact = fact; fact += (long long)f.n * f.e + (long long)f.e * f.b;
        f.inv = inv; inv += (long long)((f.e + MF_NB - 1) / MF_NB) * 2 * MF_NB * MF_NB;
        f.piv = pivo; pivo += f.e;
        f.y = y; y += f.e;
    }
    for (int v = 0; v < n_fronts; v++) {
        int p = parent[v];
        if (p < 0) continue;
        FrontMeta& f = m->meta[p];
        if (f.child[0] < 0) f.child[0] = v;
        else if (f.child[1] < 0) f.child[1] = v;
        else { delete m; set_error("emfem_mf_create: front %d has more than two children", p); return EMFEM_ERR_INVALID_ARG; }
        if (level[p] <= level[v]) { delete m; set_error("emfem_mf_create: parent below child"); return EMFEM_ERR_INVALID_ARG; }
    }
    // per-level workspace and solve-buffer offsets; update store by first-fit over the level schedule
    long long ws_max = 0, wv_max = 0;
    std::map<long long, long long> freel;   // offset -> size
    long long upd_top = 0;
    auto alloc = [&](long long sz) -> long long {
        for (auto it = freel.begin(); it != freel.end(); ++it) {
            if (it->second >= sz) {
                long long o = it->first, rem = it->second - sz;
                freel.erase(it);
                if (rem > 0) freel[o + sz] = rem;
                return o;
            }
        }
        long long o = upd_top;
        upd_top += sz;
        return o;
    };
    auto release = [&](long long o, long long sz) {
        if (sz <= 0) return;
        auto it = freel.emplace(o, sz).first;
        auto nx = std::next(it);
        if (nx != freel.end() && it->first + it->second == nx->first) { it->second += nx->second; freel.erase(nx); }
        if (it != freel.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; freel.erase(it); }
        }
    };
    long long uv = 0;
    m->lvl_max_e.assign(nl, 0); m->lvl_max_n.assign(nl, 0); m->lvl_max_asm.assign(nl, 0); m->lvl_max_b.assign(nl, 0);
    m->lvl_wv.assign(nl, 0); m->lvl_max_ob.assign(nl, 0);
    for (int L = 0; L < nl; L++) {
        long long wso = 0, wvo = 0;
        for (int v : m->levels[L]) {
            FrontMeta& f = m->meta[v];
            f.ws = wso; wso += (long long)f.n * f.n;
            f.wv = wvo; wvo += f.n;
            f.uv = uv; uv += f.b;
            m->lvl_max_e[L] = std::max(m->lvl_max_e[L], f.e);
            m->lvl_max_n[L] = std::max(m->lvl_max_n[L], f.n);
            m->lvl_max_asm[L] = std::max(m->lvl_max_asm[L], f.asm1 - f.asm0);
            long long cb = 0;
            for (int c : f.child) if (c >= 0) cb = std::max<long long>(cb, m->meta[c].b);
            m->lvl_max_b[L] = std::max(m->lvl_max_b[L], cb);
            m->lvl_max_ob[L] = std::max<long long>(m->lvl_max_ob[L], f.b);
        }
        ws_max = std::max(ws_max, wso);
        wv_max = std::max(wv_max, wvo);
        m->lvl_wv[L] = wvo;
        // levels of few fronts (the top of the tree) split their long boundary products over CTAs
        const long long nsplit = (m->lvl_max_ob[L] + MF_CW - 1) / MF_CW;
        if (nsplit > 1 && m->levels[L].size() < 148) m->part_n = std::max(m->part_n, nsplit * wvo);
        // the level's fronts get their update blocks; their children's are freed once the level assembled
        for (int v : m->levels[L]) {
            FrontMeta& f = m->meta[v];
            f.upd = alloc((long long)f.b * f.b);
        }
        for (int v : m->levels[L])
            for (int c : m->meta[v].child)
                if (c >= 0) release(m->meta[c].upd, (long long)m->meta[c].b * m->meta[c].b);
    }
    m->fact_n = fact; m->inv_n = inv; m->piv_n = pivo; m->ws_n = ws_max; m->upd_n = upd_top;
    m->wv_n = wv_max; m->uv_n = uv; m->y_n = y;
    for (int v = 0; v < n_fronts; v++) {
        double E = e[v], B = b[v];
        m->flops += 8.0 * (E * E * E / 3 + E * E * B + E * B * B);
    }
    // device arrays
    std::vector<int> lst;
    m->lvl_off.resize(nl);
    for (int L = 0; L < nl; L++) {
        m->lvl_off[L] = (long long)lst.size();
        lst.insert(lst.end(), m->levels[L].begin(), m->levels[L].end());
    }
    std::vector<uint8_t> freed(n, 0);
    for (int v = 0; v < n_fronts; v++)
        for (int i = 0; i < e[v]; i++) {
            int d = fdof[fdof_ptr[v] + i];
            if (d < 0 || d >= n) { delete m; set_error("emfem_mf_create: DOF %d out of range", d); return EMFEM_ERR_INVALID_ARG; }
            freed[d] = 1;
        }
    long long nasm = asm_ptr ? asm_ptr[n_fronts] : 0;
    m->lists = asm_ptr != nullptr;
    // elimination position of every DOF, the front of every position, each front's first position
    m->h_pos.assign(n, -1);
    m->h_fpos.reserve((size_t)std::max<long long>(1, n));
    m->h_own0.resize(n_fronts);
    for (int v = 0; v < n_fronts; v++) {
        m->h_own0[v] = (long long)m->h_fpos.size();
        for (int i = 0; i < e[v]; i++) {
            m->h_pos[fdof[fdof_ptr[v] + i]] = (int)m->h_fpos.size();
            m->h_fpos.push_back(v);
        }
    }
    int rc = EMFEM_OK;
    auto up = [&](void** dst, const void* src, size_t bytes) {
        if (rc != EMFEM_OK) return;
        rc = check_cuda(cudaMalloc(dst, std::max<size_t>(bytes, 16)), "cudaMalloc");
        if (rc == EMFEM_OK && bytes) rc = check_cuda(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
    };
    up((void**)&m->d_meta, m->meta.data(), sizeof(FrontMeta) * n_fronts);
    up((void**)&m->d_lst, lst.data(), sizeof(int) * lst.size());
    up((void**)&m->d_fdof, fdof, sizeof(int) * tot_fdof);
    up((void**)&m->d_ea, ea, sizeof(int) * eao);
    up((void**)&m->d_slot, asm_slot, sizeof(int) * nasm);
    up((void**)&m->d_off, asm_off, sizeof(int) * nasm);
    up((void**)&m->d_free, freed.data(), n);
    auto mk = [&](void** dst, size_t bytes) {
        if (rc != EMFEM_OK) return;
        rc = check_cuda(cudaMalloc(dst, std::max<size_t>(bytes, 16)), "cudaMalloc");
    };
    mk((void**)&m->fact, sizeof(float2) * fact);
    mk((void**)&m->inv, sizeof(float2) * inv);
    mk((void**)&m->piv, sizeof(int) * pivo);
    mk((void**)&m->ws, sizeof(float2) * ws_max);
    mk((void**)&m->upd, sizeof(float2) * upd_top);
    mk((void**)&m->d_npert, sizeof(int));
    mk((void**)&m->d_scale, sizeof(double) * n);
    if (rc != EMFEM_OK) { mf_free(m); delete m; return rc; }
    rc = check_cuda(cudaFuncSetAttribute(mf_fwd_block_kernel<1, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)MF_BLOCK_SMEM), "cudaFuncSetAttribute");
    if (rc == EMFEM_OK)
        rc = check_cuda(cudaFuncSetAttribute(mf_bwd_block_kernel<1, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)MF_BLOCK_SMEM), "cudaFuncSetAttribute");
    if (rc == EMFEM_OK)
        rc = check_cuda(cudaFuncSetAttribute(mf_fwd_block_kernel<2, MF_BLOCK_NT_FEW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)MF_BLOCK_SMEM2), "cudaFuncSetAttribute");
    if (rc == EMFEM_OK)
        rc = check_cuda(cudaFuncSetAttribute(mf_bwd_block_kernel<2, MF_BLOCK_NT_FEW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)MF_BLOCK_SMEM2), "cudaFuncSetAttribute");
    if (rc != EMFEM_OK) { mf_free(m); delete m; return rc; }
    *out = m;
    return EMFEM_OK;
}

int emfem_mf_info(emfem_mf m, size_t* device_bytes, double* flops, int* n_levels) {
    EMFEM_REQUIRE(m, "emfem_mf_info: bad handle");
    if (device_bytes)
        *device_bytes = sizeof(float2) * (m->fact_n + m->inv_n) + (m->wide ? sizeof(double2) : sizeof(float2)) *
                        (m->ws_n + m->upd_n) + (m->wide ? sizeof(double2) * m->inv_n : 0) + sizeof(int) * m->piv_n +
                        sizeof(double) * m->n;
    if (flops) *flops = m->flops;
    if (n_levels) *n_levels = (int)m->levels.size();
    return EMFEM_OK;
}

int emfem_mf_set_precision(emfem_mf m, int bits) {
    EMFEM_REQUIRE(m && (bits == 64 || bits == 128), "emfem_mf_set_precision: bits must be 64 or 128");
    const bool wide = bits == 128;
    if (wide == m->wide) return EMFEM_OK;
    int prev = 0;
    EMFEM_CUDA(cudaGetDevice(&prev));
    if (prev != m->h->device) EMFEM_CUDA(cudaSetDevice(m->h->device));
    EMFEM_CUDA(cudaStreamSynchronize(m->h->stream));
    void* ps[] = {m->ws, m->upd, m->invc};
    for (void* p : ps)
        if (p) cudaFree(p);
    m->ws = m->upd = m->invc = nullptr;
    m->factored = false;
    const size_t el = wide ? sizeof(double2) : sizeof(float2);
    int rc = check_cuda(cudaMalloc(&m->ws, el * std::max(1LL, m->ws_n)), "cudaMalloc");
    if (rc == EMFEM_OK) rc = check_cuda(cudaMalloc(&m->upd, el * std::max(1LL, m->upd_n)), "cudaMalloc");
    if (rc == EMFEM_OK && wide) rc = check_cuda(cudaMalloc(&m->invc, sizeof(double2) * std::max(1LL, m->inv_n)), "cudaMalloc");
    if (rc == EMFEM_OK) {
        m->wide = wide;
    } else {
        // leave a usable complex64 handle behind when the complex128 workspace does not fit
        void* qs[] = {m->ws, m->upd, m->invc};
        for (void* p : qs)
            if (p) cudaFree(p);
        m->ws = m->upd = m->invc = nullptr;
        m->wide = false;
        if (cudaMalloc(&m->ws, sizeof(float2) * std::max(1LL, m->ws_n)) != cudaSuccess ||
            cudaMalloc(&m->upd, sizeof(float2) * std::max(1LL, m->upd_n)) != cudaSuccess)
            set_error("emfem_mf_set_precision: the complex64 workspace could not be restored either");
    }
    if (prev != m->h->device) cudaSetDevice(prev);
    return rc;
}

int emfem_mf_factor(emfem_mf m, const void* K_vals, int* n_perturbed) {
    EMFEM_REQUIRE(m && K_vals, "emfem_mf_factor: bad argument");
    EMFEM_REQUIRE(m->lists, "emfem_mf_factor: no assembly lists (emfem_mf_build_lists)");
    cudaStream_t s = m->h->stream;
    int prev = 0;
    EMFEM_CUDA(cudaGetDevice(&prev));
    if (prev != m->h->device) EMFEM_CUDA(cudaSetDevice(m->h->device));
    int rc = EMFEM_OK;
    m->factored = false;
    rc = check_cuda(cudaMemsetAsync(m->d_npert, 0, sizeof(int), s), "cudaMemsetAsync");
    const int nl = (int)m->levels.size();
    // equilibration first: a front's boundary DOFs take their scale from the ancestors that eliminate them
    if (rc == EMFEM_OK) {
        mf_fill_kernel<<<grid_for(m->n, 256), 256, 0, s>>>(m->n, 1.0, m->d_scale);
        for (int L = 0; L < nl; L++)
            for (int y0 = 0; y0 < (int)m->levels[L].size(); y0 += 65535) {
                const int ny = std::min(65535, (int)m->levels[L].size() - y0);
                mf_scale_kernel<<<dim3(nblk(m->lvl_max_asm[L], MF_CHUNK), ny), 256, 0, s>>>(
                    m->d_lst + m->lvl_off[L] + y0, m->d_meta, (const double2*)K_vals, m->d_slot, m->d_off, m->d_fdof,
                    m->d_scale);
            }
        rc = check_cuda(cudaGetLastError(), "multifrontal equilibration");
    }
    if (rc == EMFEM_OK)
        rc = m->wide ? mf_factor_levels<double2>(m, (const double2*)K_vals, s)
                     : mf_factor_levels<float2>(m, (const double2*)K_vals, s);
    int np = 0;
    if (rc == EMFEM_OK) rc = check_cuda(cudaMemcpyAsync(&np, m->d_npert, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
    if (rc == EMFEM_OK) rc = check_cuda(cudaStreamSynchronize(s), "sync");
    if (rc == EMFEM_OK) {
        m->factored = true;
        if (n_perturbed) *n_perturbed = np;
    }
    if (prev != m->h->device) cudaSetDevice(prev);
    return rc;
}

int emfem_mf_build_lists(emfem_mf m, int64_t nnz, const int32_t* indptr, const int32_t* indices) {
    EMFEM_REQUIRE(m && indptr && indices && nnz > 0 && nnz < (1LL << 31), "emfem_mf_build_lists: bad argument");
    EMFEM_REQUIRE(!m->lists, "emfem_mf_build_lists: the lists exist already");
    cudaStream_t s = m->h->stream;
    const long long n = m->n;
    const int nf = m->nf;
    int *d_pos = nullptr, *d_fpos = nullptr, *cnt = nullptr, *base = nullptr, *cur = nullptr, *scratch = nullptr;
    long long* d_own0 = nullptr;
    int rc = EMFEM_OK;
    std::vector<int> hb(nf + 1);
#define LTRY(x) do { rc = (x); if (rc != EMFEM_OK) goto done; } while (0)
    LTRY(check_cuda(cudaMalloc(&d_pos, sizeof(int) * n), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&d_fpos, sizeof(int) * std::max<size_t>(1, m->h_fpos.size())), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&d_own0, sizeof(long long) * nf), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&cnt, sizeof(int) * nf), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&base, sizeof(int) * (nf + 1)), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&cur, sizeof(int) * nf), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&scratch, sizeof(int) * scan_scratch_ints(nf)), "cudaMalloc"));
    LTRY(check_cuda(cudaMemcpyAsync(d_pos, m->h_pos.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s), "copy"));
    LTRY(check_cuda(cudaMemcpyAsync(d_fpos, m->h_fpos.data(), sizeof(int) * m->h_fpos.size(), cudaMemcpyHostToDevice, s), "copy"));
    LTRY(check_cuda(cudaMemcpyAsync(d_own0, m->h_own0.data(), sizeof(long long) * nf, cudaMemcpyHostToDevice, s), "copy"));
    LTRY(check_cuda(cudaMemsetAsync(cnt, 0, sizeof(int) * nf, s), "memset"));
    LTRY(check_cuda(cudaMemsetAsync(cur, 0, sizeof(int) * nf, s), "memset"));
    LTRY(check_cuda(cudaMemsetAsync(m->h->dev_status, 0, sizeof(int), s), "memset"));
    mf_list_count_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, indptr, indices, d_pos, d_fpos, cnt);
    LTRY(check_cuda(cudaGetLastError(), "mf_list_count_kernel"));
    LTRY(exclusive_scan_i32(m->h, cnt, base, nf, scratch));
    LTRY(check_cuda(cudaMemcpyAsync(hb.data(), base, sizeof(int) * (nf + 1), cudaMemcpyDeviceToHost, s), "copy"));
    LTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
    LTRY(check_cuda(cudaMalloc(&m->d_slot, sizeof(int) * std::max(1, hb[nf])), "cudaMalloc"));
    LTRY(check_cuda(cudaMalloc(&m->d_off, sizeof(int) * std::max(1, hb[nf])), "cudaMalloc"));
    mf_list_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, indptr, indices, d_pos, d_fpos, d_own0, m->d_meta, m->d_fdof,
                                                          base, cur, m->d_slot, m->d_off, m->h->dev_status);
    LTRY(check_cuda(cudaGetLastError(), "mf_list_fill_kernel"));
    for (int v = 0; v < nf; v++) {
        m->meta[v].asm0 = hb[v];
        m->meta[v].asm1 = hb[v + 1];
    }
    for (size_t L = 0; L < m->levels.size(); L++) {
        long long mx = 0;
        for (int v : m->levels[L]) mx = std::max<long long>(mx, hb[v + 1] - hb[v]);
        m->lvl_max_asm[L] = mx;
    }
    LTRY(check_cuda(cudaMemcpyAsync(m->d_meta, m->meta.data(), sizeof(FrontMeta) * nf, cudaMemcpyHostToDevice, s), "copy"));
    {
        int st = 0;
        LTRY(check_cuda(cudaMemcpyAsync(&st, m->h->dev_status, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        LTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        if (st & DEV_BAD_INDEX) {
            cudaMemsetAsync(m->h->dev_status, 0, sizeof(int), s);
            set_error("emfem_mf_build_lists: a CSR entry's DOF is in neither the own nor the boundary set of its front");
            rc = EMFEM_ERR_DEVICE_CHECK;
            goto done;
        }
    }
    m->lists = true;
done:
    cudaFree(d_pos); cudaFree(d_fpos); cudaFree(d_own0); cudaFree(cnt); cudaFree(base); cudaFree(cur); cudaFree(scratch);
    return rc;
#undef LTRY
}

int emfem_mf_reserve(emfem_mf m, int nrhs) {
    EMFEM_REQUIRE(m && nrhs >= 1 && nrhs <= 256, "emfem_mf_reserve: bad argument");
    return mf_reserve(m, nrhs);
}

int emfem_mf_solve(emfem_mf m, int nrhs, const void* b, void* x) {
    EMFEM_REQUIRE(m && b && x && nrhs >= 1, "emfem_mf_solve: bad argument");
    EMFEM_TRY(mf_reserve(m, nrhs));
    return mf_apply(m, nrhs, (const double2*)b, (double2*)x, m->h->stream);
}

int emfem_mf_destroy(emfem_mf m) {
    if (!m) return EMFEM_OK;
    cudaStreamSynchronize(m->h->stream);
    mf_free(m);
    delete m;
    return EMFEM_OK;
}

}  // extern "C"
