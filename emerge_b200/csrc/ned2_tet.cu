// Nedelec-2 tet kernels: per-element integrator, device symbolic CSR plan, fused CSR assembly.
//
// Fused assembly design (replaces _matrix_builder + coo.tocsr(), ASM/curlcurl.py:145-173,419-466):
//   * An "entity" X is an edge (X < N_e) or a face (N_e <= X < H = N_e + N_f); it owns the two DOF
//     rows X (first kind) and X + H (second kind) (elements/nedelec2.py:42-58).
//   * Plan (once per mesh): for every entity, its incident tets sorted ascending, the sorted set
//     S_X of first-kind DOFs of those tets (row X's columns are S_X then S_X + H; row X + H has the
//     same columns), and for every (X, t) incidence the position in S_X of each of t's 10 entities.
//   * Numeric: per-tet invariants (ned2_math.cuh) are computed once per tet; then one thread per
//     (X, k) — row pair of X, column pair of S_X[k] — sums the 2x2 D/F pair blocks of X's incident
//     tets in ascending tet order and writes its 4 E and 4 B CSR values once.  No atomics, no COO
//     buffer; the pattern equals SciPy's tocsr() of the reference COO (sorted rows, zeros kept).
#include "emfem_internal.cuh"
#include "ned2_math.cuh"

#include <vector>

namespace emfem {

constexpr int INC_REC = 16;         // bytes per incidence record: 10 positions + own slot + pad
constexpr int SYM_CAP = 1024;       // max candidate columns per entity (10 x incident tets)
constexpr int SYM_WARPS = 4;        // warps per CTA in the symbolic kernels

// ---------------------------------------------------------------- per-tet invariants
__device__ __forceinline__ cd load_c(const double2* p, long long i) {
    double2 v = p[i];
    return mk(v.x, v.y);
}

__global__ void __launch_bounds__(128) tet_invariants_kernel(
    long long nt, long long nn, long long ne, const double* __restrict__ nodes,
    const int64_t* __restrict__ tets, const int64_t* __restrict__ t2e, const double* __restrict__ elen,
    const double2* __restrict__ ur, const double2* __restrict__ er, double* __restrict__ inv, int* status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int64_t ids[4];
    double xs[4], ys[4], zs[4], el[6];
    bool bad = false, finite = true;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int64_t v = tets[i * nt + t];
        if (v < 0 || v >= nn) { bad = true; v = 0; }
        ids[i] = v;
        xs[i] = nodes[v]; ys[i] = nodes[nn + v]; zs[i] = nodes[2 * nn + v];
        finite &= isfinite(xs[i]) && isfinite(ys[i]) && isfinite(zs[i]);
    }
#pragma unroll
    for (int e = 0; e < 6; e++) {
        int64_t id = t2e[e * nt + t];
        if (id < 0 || id >= ne) { bad = true; id = 0; }
        el[e] = elen[id];
        finite &= isfinite(el[e]);
    }
    if (bad) flag(status, DEV_BAD_INDEX);
    cd U[9], E[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        U[k] = load_c(ur, k * nt + t); E[k] = load_c(er, k * nt + t);
        finite &= isfinite(U[k].x) && isfinite(U[k].y) && isfinite(E[k].x) && isfinite(E[k].y);
    }
    double* out = inv + t * INV_STRIDE;
    tet_invariants(xs, ys, zs, ids, el, U, E, out);
    if (!(out[INV_SF] < 1e300)) flag(status, DEV_DEGENERATE);
    if (!finite) flag(status, DEV_NONFINITE);
}

__device__ __forceinline__ void load_vtab(double* sh) {
    for (int i = threadIdx.x; i < 625; i += blockDim.x)
        sh[i] = volume_coeff_closed(i / 125, (i / 25) % 5, (i / 5) % 5, i % 5);
}

// ---------------------------------------------------------------- per-element matrices
// 32 tets per CTA: invariants to shared memory, then 128 threads cover the 32 x 100 pair blocks.
constexpr int EL_TETS = 32;

__global__ void __launch_bounds__(128) tet_element_kernel(
    long long nt, long long nn, long long ne, const double* __restrict__ nodes,
    const int64_t* __restrict__ tets, const int64_t* __restrict__ t2e, const double* __restrict__ elen,
    const double2* __restrict__ ur, const double2* __restrict__ er, double2* __restrict__ outE,
    double2* __restrict__ outB, int* status) {
    __shared__ double vtab[625];
    __shared__ double sinv[INV_NDOUBLE * EL_TETS];
    load_vtab(vtab);
    long long t0 = (long long)blockIdx.x * EL_TETS;
    if (threadIdx.x < EL_TETS) {
        long long t = t0 + threadIdx.x;
        if (t < nt) {
            int64_t ids[4];
            double xs[4], ys[4], zs[4], el[6];
            bool bad = false;
            for (int i = 0; i < 4; i++) {
                int64_t v = tets[i * nt + t];
                if (v < 0 || v >= nn) { bad = true; v = 0; }
                ids[i] = v;
                xs[i] = nodes[v]; ys[i] = nodes[nn + v]; zs[i] = nodes[2 * nn + v];
            }
            for (int e = 0; e < 6; e++) {
                int64_t id = t2e[e * nt + t];
                if (id < 0 || id >= ne) { bad = true; id = 0; }
                el[e] = elen[id];
            }
            if (bad) flag(status, DEV_BAD_INDEX);
            cd U[9], E[9];
            for (int k = 0; k < 9; k++) { U[k] = load_c(ur, k * nt + t); E[k] = load_c(er, k * nt + t); }
            double loc[INV_NDOUBLE];
            tet_invariants(xs, ys, zs, ids, el, U, E, loc);
            if (!(loc[INV_SF] < 1e300)) flag(status, DEV_DEGENERATE);
            for (int f = 0; f < INV_NDOUBLE; f++) sinv[f * EL_TETS + threadIdx.x] = loc[f];
        }
    }
    __syncthreads();
    VTab T{vtab};
    for (int w = threadIdx.x; w < EL_TETS * 100; w += blockDim.x) {
        int lt = w / 100, pb = w % 100;
        long long t = t0 + lt;
        if (t >= nt) continue;
        InvView I{sinv + lt, EL_TETS};
        Orient o = unpack_rank((int)I.g(INV_RANK));
        int sx = pb / 10, sy = pb % 10;
        cd d[4], f[4];
        pair_block(I, o, T, sx, sy, d, f);
#pragma unroll
        for (int kx = 0; kx < 2; kx++)
#pragma unroll
            for (int ky = 0; ky < 2; ky++) {
                long long o2 = t * 400 + local_dof(sx, kx) * 20 + local_dof(sy, ky);
                cd dv = d[2 * kx + ky], fv = f[2 * kx + ky];
                outE[o2] = make_double2(dv.x, dv.y);
                outB[o2] = make_double2(fv.x, fv.y);
            }
    }
}

__global__ void coo_indices_kernel(long long nt, const int64_t* __restrict__ t2f, int64_t* rows, int64_t* cols) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nt * 400) return;
    long long t = g / 400;
    int k = (int)(g % 400), i = k / 20, j = k % 20;
    rows[g] = t2f[i * nt + t];
    cols[g] = t2f[j * nt + t];
}

__global__ void mesh_check_kernel(long long nn, long long nt, long long ne, long long nf,
                                  const int64_t* __restrict__ tets, const int64_t* __restrict__ edges,
                                  const int64_t* __restrict__ tris, const int64_t* __restrict__ t2e,
                                  const int64_t* __restrict__ t2t, int* status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int64_t v[4];
    bool bad = false;
    for (int i = 0; i < 4; i++) { v[i] = tets[i * nt + t]; if (v[i] < 0 || v[i] >= nn) bad = true; }
    for (int e = 0; e < 6 && !bad; e++) {
        int64_t id = t2e[e * nt + t];
        if (id < 0 || id >= ne) { bad = true; break; }
        int64_t a = v[tet_edge_p(e)], b = v[tet_edge_q(e)];
        int64_t lo = a < b ? a : b, hi = a < b ? b : a;
        if (edges[id] != lo || edges[ne + id] != hi) bad = true;
    }
    for (int f = 0; f < 4 && !bad; f++) {
        int64_t id = t2t[f * nt + t];
        if (id < 0 || id >= nf) { bad = true; break; }
        int64_t a = v[tet_face_v(f, 0)], b = v[tet_face_v(f, 1)], c = v[tet_face_v(f, 2)], s;
        if (b < a) { s = a; a = b; b = s; }
        if (c < b) { s = b; b = c; c = s; }
        if (b < a) { s = a; a = b; b = s; }
        if (tris[id] != a || tris[nf + id] != b || tris[2 * nf + id] != c) bad = true;
    }
    if (bad) flag(status, DEV_BAD_INDEX);
}

// ---------------------------------------------------------------- symbolic plan kernels
__global__ void inc_count_kernel(long long nt, long long ne, long long H, const int64_t* __restrict__ t2f,
                                 int* __restrict__ cnt, int* status) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nt * 10) return;
    int s = (int)(g / nt);
    long long t = g % nt;
    int64_t X = t2f[s * nt + t];
    int64_t X2 = t2f[(s + 10) * nt + t];
    bool ok = s < 6 ? (X >= 0 && X < ne) : (X >= ne && X < H);
    ok = ok && (X2 == X + H);
    if (!ok) { flag(status, DEV_BAD_INDEX); return; }
    atomicAdd(&cnt[X], 1);
}

__global__ void inc_fill_kernel(long long nt, long long ne, const int64_t* __restrict__ t2f, const int* __restrict__ inc_ptr,
                                int* __restrict__ cursor, uint32_t* __restrict__ inc_code, long long H) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nt * 10) return;
    int s = (int)(g / nt);
    long long t = g % nt;
    int64_t X = t2f[s * nt + t];
    int64_t X2 = t2f[(s + 10) * nt + t];
    bool ok = s < 6 ? (X >= 0 && X < ne) : (X >= ne && X < H);
    if (!ok || X2 != X + H) return;
    int p = atomicAdd(&cursor[X], 1);
    inc_code[inc_ptr[X] + p] = (uint32_t)(t * 16 + s);
}

__global__ void inc_sort_kernel(long long H, const int* __restrict__ inc_ptr, uint32_t* __restrict__ inc_code) {
    long long X = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (X >= H) return;
    int b = inc_ptr[X], e = inc_ptr[X + 1];
    for (int i = b + 1; i < e; i++) {
        uint32_t v = inc_code[i];
        int j = i - 1;
        while (j >= b && inc_code[j] > v) { inc_code[j + 1] = inc_code[j]; j--; }
        inc_code[j + 1] = v;
    }
}

// warp-level bitonic sort of buf[0..P) (P power of two <= SYM_CAP), ascending
__device__ void warp_bitonic(int* buf, int P) {
    int lane = threadIdx.x & 31;
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                int p = i ^ j;
                if (p > i) {
                    int a = buf[i], b = buf[p];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { buf[i] = b; buf[p] = a; }
                }
            }
            __syncwarp();
        }
    }
}

// warp per entity: candidates (10 first-kind DOFs of each incident tet) -> sorted unique list
// into tmp[10 * inc_ptr[X] ...], count into m[X].
__global__ void __launch_bounds__(32 * SYM_WARPS) cols_count_kernel(
    long long H, long long nt, const int64_t* __restrict__ t2f, const int* __restrict__ inc_ptr,
    const uint32_t* __restrict__ inc_code, int* __restrict__ tmp, int* __restrict__ m, int* status) {
    __shared__ int sbuf[SYM_WARPS][SYM_CAP];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    long long X = (long long)blockIdx.x * SYM_WARPS + warp;
    if (X >= H) return;
    int* buf = sbuf[warp];
    int b = inc_ptr[X], deg = inc_ptr[X + 1] - b;
    int nc = 10 * deg;
    if (nc > SYM_CAP) {
        if (lane == 0) { flag(status, DEV_CAPACITY); m[X] = 0; }
        return;
    }
    int P = 1;
    while (P < nc) P <<= 1;
    for (int c = lane; c < P; c += 32) {
        int v = 0x7fffffff;
        if (c < nc) {
            uint32_t code = inc_code[b + c / 10];
            long long t = code >> 4;
            v = (int)t2f[(c % 10) * nt + t];
        }
        buf[c] = v;
    }
    __syncwarp();
    warp_bitonic(buf, P);
    // compact unique values preserving order
    int base = 0;
    for (int c0 = 0; c0 < nc; c0 += 32) {
        int c = c0 + lane;
        bool first = c < nc && (c == 0 || buf[c] != buf[c - 1]);
        unsigned mask = __ballot_sync(0xffffffffu, first);
        int rank = __popc(mask & ((1u << lane) - 1));
        if (first) tmp[10LL * b + base + rank] = buf[c];
        base += __popc(mask);
    }
    if (lane == 0) m[X] = base;
}

// thread per entity: copy the unique list into S and build the incidence records.
__global__ void cols_fill_kernel(long long H, long long nt, const int64_t* __restrict__ t2f,
                                 const int* __restrict__ inc_ptr, const uint32_t* __restrict__ inc_code,
                                 const int* __restrict__ tmp, const int* __restrict__ mptr,
                                 int* __restrict__ S, uint8_t* __restrict__ rec, int* status) {
    long long X = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (X >= H) return;
    int b = inc_ptr[X], e = inc_ptr[X + 1];
    int s0 = mptr[X], m = mptr[X + 1] - s0;
    const int* src = tmp + 10LL * b;
    for (int k = 0; k < m; k++) S[s0 + k] = src[k];
    if (m > 255) { flag(status, DEV_CAPACITY); return; }
    for (int i = b; i < e; i++) {
        uint32_t code = inc_code[i];
        long long t = code >> 4;
        uint8_t r[INC_REC];
        for (int sy = 0; sy < 10; sy++) {
            int v = (int)t2f[sy * nt + t];
            int lo = 0, hi = m - 1;
            while (lo < hi) { int mid = (lo + hi) >> 1; if (src[mid] < v) lo = mid + 1; else hi = mid; }
            r[sy] = (uint8_t)lo;
        }
        r[10] = (uint8_t)(code & 15);
        for (int q = 11; q < INC_REC; q++) r[q] = 0xff;
        uint4 pk;
        memcpy(&pk, r, 16);
        reinterpret_cast<uint4*>(rec)[i] = pk;
    }
}

__global__ void export_indptr_kernel(long long H, const int* __restrict__ mptr, int* __restrict__ indptr) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long N = 2 * H;
    if (r > N) return;
    long long v;
    if (r < H) v = 2LL * mptr[r];
    else if (r < N) v = 2LL * mptr[H] + 2LL * mptr[r - H];
    else v = 4LL * mptr[H];
    indptr[r] = (int)v;
}

__device__ __forceinline__ long long find_entity(const int* __restrict__ mptr, long long H, long long j,
                                                 long long lo, long long hi) {
    // largest X in [lo, hi) with mptr[X] <= j
    while (hi - lo > 1) {
        long long mid = (lo + hi) >> 1;
        if (mptr[mid] <= j) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void export_indices_kernel(long long H, long long sum_m, const int* __restrict__ mptr,
                                      const int* __restrict__ S, int* __restrict__ indices) {
    long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= sum_m) return;
    long long X = find_entity(mptr, H, j, 0, H);
    int k = (int)(j - mptr[X]), m = mptr[X + 1] - mptr[X];
    int c = S[j];
    long long b1 = 2LL * mptr[X] + k, b2 = 2LL * mptr[H] + 2LL * mptr[X] + k;
    indices[b1] = c; indices[b1 + m] = c + (int)H;
    indices[b2] = c; indices[b2 + m] = c + (int)H;
}

// ---------------------------------------------------------------- fused numeric assembly
// One CTA per chunk of consecutive entities of one kind (all edges or all faces) holding at most
// CH incidences.  Phase 0: the chunk's incidence records and the invariants of their tets are
// copied to shared memory with coalesced loads.  Phase 1: one thread per (incidence, column entity)
// pair block, column-entity major so every warp evaluates one edge/face block type; results staged
// in shared memory.  Phase 2: one thread per output (X, k) sums its tets' staged blocks in
// ascending tet order and writes the 4 E and 4 B CSR values of its column pair.
constexpr int INV_SMEM_STRIDE = 121;  // odd stride in doubles: lanes of a warp hit distinct banks

template <int CH, bool SINV>
struct ChunkSmem {
    static constexpr size_t stage = (size_t)(CH + 1) * 10 * 8 * 16;
    static constexpr size_t inv = SINV ? (size_t)CH * INV_SMEM_STRIDE * 8 : 0;
    static constexpr size_t vtab = 625 * 8;
    static constexpr size_t rec = (size_t)CH * 16;
    static constexpr size_t code = (size_t)CH * 4;
    static constexpr size_t off_inv = stage;
    static constexpr size_t off_vtab = off_inv + inv;
    static constexpr size_t off_rec = (off_vtab + vtab + 15) & ~(size_t)15;
    static constexpr size_t off_code = off_rec + rec;
    static constexpr size_t off_ent = off_code + code;              // (CH + 1) mptr, (CH + 1) inc_ptr
    static constexpr size_t total = off_ent + (size_t)(2 * CH + 2) * 4;
};

// LM (incidence-major): consecutive threads take the 6 edge columns, then the 4 face columns, of one
// incidence before the next, so a warp's invariant loads fall on a few tets' records (few L1
// wavefronts).  Otherwise consecutive threads take one column of 32 incidences (32 records).
template <int CH, int NT, int MINB, bool SINV, bool LM>
__global__ void __launch_bounds__(NT, MINB) assemble_chunk_kernel(
    const int* __restrict__ chunk_ptr, long long H, const int* __restrict__ mptr,
    const int* __restrict__ inc_ptr, const uint32_t* __restrict__ inc_code, const uint4* __restrict__ rec,
    const double* __restrict__ inv, double2* __restrict__ Ev, double2* __restrict__ Bv) {
    typedef ChunkSmem<CH, SINV> L;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* stage = reinterpret_cast<double2*>(smem);                 // [q][sy][CH + 1] (padded rows)
    double* sinv = reinterpret_cast<double*>(smem + L::off_inv);       // [CH][INV_SMEM_STRIDE]
    double* vtab = reinterpret_cast<double*>(smem + L::off_vtab);      // 625
    uint4* srec = reinterpret_cast<uint4*>(smem + L::off_rec);         // CH
    uint32_t* scode = reinterpret_cast<uint32_t*>(smem + L::off_code); // CH
    int* smptr = reinterpret_cast<int*>(smem + L::off_ent);             // chunk entities' mptr, X0..X1
    int* sinc = smptr + CH + 1;                                          // chunk entities' inc_ptr - i0
    load_vtab(vtab);
    const int X0 = chunk_ptr[blockIdx.x], X1 = chunk_ptr[blockIdx.x + 1];
    const int i0 = inc_ptr[X0], ninc = inc_ptr[X1] - i0;
    const int nent = X1 - X0;  // <= CH: every entity has at least one incidence
    for (int li = threadIdx.x; li < ninc; li += NT) {
        srec[li] = rec[i0 + li];
        scode[li] = inc_code[i0 + li];
    }
    for (int e = threadIdx.x; e <= nent; e += NT) {
        smptr[e] = mptr[X0 + e];
        sinc[e] = inc_ptr[X0 + e] - i0;
    }
    __syncthreads();
    if (SINV) {
        // one warp per incidence: lanes copy consecutive doubles of the tet's record
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int li = warp; li < ninc; li += NT / 32) {
            const double* src = inv + (long long)(scode[li] >> 4) * INV_STRIDE;
            double* dst = sinv + li * INV_SMEM_STRIDE;
#pragma unroll
            for (int f = lane; f < INV_NDOUBLE; f += 32) dst[f] = src[f];
        }
    }
    __syncthreads();
    VTab T{vtab};
    const int npad = (ninc + 31) & ~31;
    const int nwork = LM ? 10 * ninc : 10 * npad;
    for (int w = threadIdx.x; w < nwork; w += NT) {
        int sy, li;
        if (LM) {
            if (w < 6 * ninc) { li = w / 6; sy = w - 6 * li; }
            else { int u = w - 6 * ninc; li = u >> 2; sy = 6 + (u & 3); }
        } else {
            sy = w / npad; li = w - sy * npad;
            if (li >= ninc) continue;
        }
        int sx = (int)((srec[li].z >> 16) & 0xff);  // byte 10 of the record
        cd d[4], f[4];
        if constexpr (SINV) {
            const InvView I{sinv + li * INV_SMEM_STRIDE, 1};
            pair_block(I, unpack_rank((int)I.g(INV_RANK)), T, sx, sy, d, f);
        } else {
            const InvRec I{inv + (long long)(scode[li] >> 4) * INV_STRIDE};
            pair_block(I, unpack_rank((int)I.g(INV_RANK)), T, sx, sy, d, f);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            stage[(q * 10 + sy) * (CH + 1) + li] = make_double2(d[q].x, d[q].y);
            stage[((4 + q) * 10 + sy) * (CH + 1) + li] = make_double2(f[q].x, f[q].y);
        }
    }
    __syncthreads();
    const int m0 = smptr[0], total = smptr[nent] - m0;
    const long long two_mH = 2LL * mptr[H];
    for (int o = threadIdx.x; o < total; o += NT) {
        int j = m0 + o;
        int lo = 0, hi = nent;  // largest e in [0, nent) with smptr[e] <= j
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (smptr[mid] <= j) lo = mid; else hi = mid; }
        const int mb = smptr[lo], k = j - mb, m = smptr[lo + 1] - mb;
        double2 acc[8];
#pragma unroll
        for (int q = 0; q < 8; q++) acc[q] = make_double2(0.0, 0.0);
        for (int li = sinc[lo]; li < sinc[lo + 1]; li++) {
            uint4 r4 = srec[li];
            uint32_t wds[4] = {r4.x, r4.y, r4.z, r4.w};
            int sy = -1;
#pragma unroll
            for (int q = 0; q < 10; q++) if ((int)((wds[q >> 2] >> (8 * (q & 3))) & 0xff) == k) sy = q;
            if (sy < 0) continue;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                double2 v = stage[(q * 10 + sy) * (CH + 1) + li];
                acc[q].x += v.x; acc[q].y += v.y;
            }
        }
        long long b1 = 2LL * mb + k, b2 = two_mH + 2LL * mb + k;
        Ev[b1] = acc[0]; Ev[b1 + m] = acc[1]; Ev[b2] = acc[2]; Ev[b2 + m] = acc[3];
        Bv[b1] = acc[4]; Bv[b1 + m] = acc[5]; Bv[b2] = acc[6]; Bv[b2 + m] = acc[7];
    }
}

// Kernel variants: chunk capacity CH incidences, NT threads, min resident CTAs, invariants staged in
// shared memory or read through L1.  The plan times them and keeps the fastest.
struct AsmVariant { int ch; int nt; size_t smem; };
#define EMFEM_ASM_VARIANTS(X)              \
    X(0, 32, 160, 2, true, false)          \
    X(1, 32, 160, 4, false, false)         \
    X(2, 64, 320, 1, true, false)          \
    X(3, 16, 128, 5, false, false)         \
    X(4, 32, 160, 3, false, false)         \
    X(5, 64, 320, 2, false, false)         \
    X(6, 64, 320, 2, false, true)          \
    X(7, 32, 160, 4, false, true)          \
    X(8, 32, 160, 3, false, true)          \
    X(9, 64, 320, 1, true, true)           \
    X(10, 64, 256, 2, false, true)         \
    X(11, 32, 128, 4, false, true)         \
    X(12, 64, 192, 3, false, true)
constexpr int N_ASM_VARIANTS = 13;
constexpr int DEFAULT_ASM_VARIANT = 6;
#define EMFEM_V_ENTRY(i, ch, nt, mb, si, lm) {ch, nt, ChunkSmem<ch, si>::total},
static const AsmVariant ASM_VARIANTS[N_ASM_VARIANTS] = {EMFEM_ASM_VARIANTS(EMFEM_V_ENTRY)};

static void launch_asm_variant(int v, unsigned grid, cudaStream_t s, const int* chunk_ptr, long long H, const int* mptr,
                               const int* inc_ptr, const uint32_t* inc_code, const uint4* rec, const double* inv,
                               double2* E, double2* B) {
    switch (v) {
#define EMFEM_V_LAUNCH(i, ch, nt, mb, si, lm) \
    case i: assemble_chunk_kernel<ch, nt, mb, si, lm><<<grid, nt, ASM_VARIANTS[i].smem, s>>>(chunk_ptr, H, mptr, inc_ptr, inc_code, rec, inv, E, B); break;
        EMFEM_ASM_VARIANTS(EMFEM_V_LAUNCH)
    default: break;
    }
}

static cudaError_t set_asm_smem_attributes() {
    cudaError_t e = cudaSuccess;
#define EMFEM_V_ATTR(i, ch, nt, mb, si, lm) \
    if (e == cudaSuccess) e = cudaFuncSetAttribute(assemble_chunk_kernel<ch, nt, mb, si, lm>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ASM_VARIANTS[i].smem);
    EMFEM_ASM_VARIANTS(EMFEM_V_ATTR)
    return e;
}

__global__ void find_slots_kernel(long long n, long long H, const int* __restrict__ mptr, const int* __restrict__ S,
                                  const int64_t* __restrict__ rows, const int64_t* __restrict__ cols, int* slots) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long r = rows[i], c = cols[i];
    int out = -1;
    if (r >= 0 && r < 2 * H && c >= 0 && c < 2 * H) {
        long long X = r < H ? r : r - H;
        long long cX = c < H ? c : c - H;
        int b = mptr[X], m = mptr[X + 1] - b;
        int lo = 0, hi = m - 1;
        while (lo < hi) { int mid = (lo + hi) >> 1; if (S[b + mid] < cX) lo = mid + 1; else hi = mid; }
        if (m > 0 && S[b + lo] == cX) {
            long long base = r < H ? 2LL * b : 2LL * mptr[H] + 2LL * b;
            out = (int)(base + lo + (c < H ? 0 : m));
        }
    }
    slots[i] = out;
}

}  // namespace emfem

using namespace emfem;

struct emfem_plan_s {
    Handle* h = nullptr;
    long long nt = 0, ne = 0, nf = 0, H = 0, N = 0, nnz = 0, sum_m = 0;
    int* inc_ptr = nullptr;        // H + 1
    uint32_t* inc_code = nullptr;  // 10 nt: tet * 16 + slot, sorted per entity
    uint8_t* rec = nullptr;        // 16 * 10 nt
    int* mptr = nullptr;           // H + 1
    int* S = nullptr;              // sum_m
    double* inv = nullptr;         // INV_STRIDE * nt (array of structs)
    int* chunk_ptr[N_ASM_VARIANTS] = {nullptr};   // per variant: n_chunks + 1 entity boundaries
    int n_chunks[N_ASM_VARIANTS] = {0};
    int variant = 0;                                 // kernel variant used by emfem_plan_assemble
};

static void plan_free(emfem_plan p) {
    if (!p) return;
    cudaFree(p->inc_ptr); cudaFree(p->inc_code); cudaFree(p->rec);
    cudaFree(p->mptr); cudaFree(p->S); cudaFree(p->inv);
    for (int v = 0; v < N_ASM_VARIANTS; v++) cudaFree(p->chunk_ptr[v]);
    delete p;
}

extern "C" {

int emfem_ned2_tet_matrices(emfem_handle h, int64_t n_nodes, int64_t n_tets, int64_t n_edges,
                            const double* nodes, const int64_t* tets, const int64_t* tet_to_edge,
                            const double* edge_lengths, const void* ur, const void* er,
                            void* E_out, void* B_out) {
    EMFEM_REQUIRE(h && nodes && tets && tet_to_edge && edge_lengths && ur && er && E_out && B_out,
                  "emfem_ned2_tet_matrices: null argument");
    EMFEM_REQUIRE(n_tets >= 0 && n_nodes > 0 && n_edges > 0, "emfem_ned2_tet_matrices: bad sizes");
    if (n_tets == 0) return EMFEM_OK;
    unsigned grid = (unsigned)((n_tets + EL_TETS - 1) / EL_TETS);
    tet_element_kernel<<<grid, 128, 0, h->h.stream>>>(n_tets, n_nodes, n_edges, nodes, tets, tet_to_edge,
                                                       edge_lengths, (const double2*)ur, (const double2*)er,
                                                       (double2*)E_out, (double2*)B_out, h->h.dev_status);
    EMFEM_LAUNCH("tet_element_kernel");
    return EMFEM_OK;
}

int emfem_ned2_coo_indices(emfem_handle h, int64_t n_tets, const int64_t* tet_to_field, int64_t* rows, int64_t* cols) {
    EMFEM_REQUIRE(h && tet_to_field && rows && cols && n_tets >= 0, "emfem_ned2_coo_indices: bad argument");
    if (n_tets == 0) return EMFEM_OK;
    coo_indices_kernel<<<grid_for(n_tets * 400, 256), 256, 0, h->h.stream>>>(n_tets, tet_to_field, rows, cols);
    EMFEM_LAUNCH("coo_indices_kernel");
    return EMFEM_OK;
}

int emfem_mesh_check(emfem_handle h, int64_t n_nodes, int64_t n_tets, int64_t n_edges, int64_t n_tris,
                     const int64_t* tets, const int64_t* edges, const int64_t* tris,
                     const int64_t* tet_to_edge, const int64_t* tet_to_tri) {
    EMFEM_REQUIRE(h && tets && edges && tris && tet_to_edge && tet_to_tri, "emfem_mesh_check: null argument");
    if (n_tets == 0) return EMFEM_OK;
    mesh_check_kernel<<<grid_for(n_tets, 256), 256, 0, h->h.stream>>>(n_nodes, n_tets, n_edges, n_tris, tets, edges,
                                                                     tris, tet_to_edge, tet_to_tri, h->h.dev_status);
    EMFEM_LAUNCH("mesh_check_kernel");
    return EMFEM_OK;
}

int emfem_plan_create(emfem_handle h, int64_t n_tets, int64_t n_edges, int64_t n_tris,
                      const int64_t* tet_to_field, emfem_plan* out) {
    EMFEM_REQUIRE(h && tet_to_field && out, "emfem_plan_create: null argument");
    EMFEM_REQUIRE(n_tets > 0 && n_edges > 0 && n_tris > 0, "emfem_plan_create: empty mesh");
    EMFEM_REQUIRE(n_tets < (1LL << 27), "emfem_plan_create: at most 2^27 tets supported");
    long long H = n_edges + n_tris;
    EMFEM_REQUIRE(10LL * n_tets < (1LL << 31) && 2 * H < (1LL << 31), "emfem_plan_create: mesh too large for int32 indexing");
    cudaStream_t s = h->h.stream;
    emfem_plan p = new emfem_plan_s();
    p->h = &h->h; p->nt = n_tets; p->ne = n_edges; p->nf = n_tris; p->H = H; p->N = 2 * H;
    int st = EMFEM_OK;
    int *cnt = nullptr, *cursor = nullptr, *scratch = nullptr, *tmp = nullptr, *m = nullptr;
    size_t nscr = scan_scratch_ints(H + 1);
#define PTRY(x) do { st = (x); if (st != EMFEM_OK) goto fail; } while (0)
    PTRY(check_cuda(cudaMalloc(&p->inc_ptr, (H + 1) * sizeof(int)), "cudaMalloc(inc_ptr)"));
    PTRY(check_cuda(cudaMalloc(&p->inc_code, 10 * n_tets * sizeof(uint32_t)), "cudaMalloc(inc_code)"));
    PTRY(check_cuda(cudaMalloc(&p->rec, 10 * n_tets * (size_t)INC_REC), "cudaMalloc(rec)"));
    PTRY(check_cuda(cudaMalloc(&p->mptr, (H + 1) * sizeof(int)), "cudaMalloc(mptr)"));
    PTRY(check_cuda(cudaMalloc(&p->inv, (size_t)INV_STRIDE * n_tets * sizeof(double)), "cudaMalloc(inv)"));
    PTRY(check_cuda(cudaMalloc(&cnt, H * sizeof(int)), "cudaMalloc(cnt)"));
    PTRY(check_cuda(cudaMalloc(&cursor, H * sizeof(int)), "cudaMalloc(cursor)"));
    PTRY(check_cuda(cudaMalloc(&scratch, nscr * sizeof(int)), "cudaMalloc(scan)"));
    PTRY(check_cuda(cudaMalloc(&tmp, 100 * n_tets * sizeof(int)), "cudaMalloc(tmp)"));
    PTRY(check_cuda(cudaMalloc(&m, H * sizeof(int)), "cudaMalloc(m)"));
    PTRY(check_cuda(cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), s), "memset"));
    PTRY(check_cuda(cudaMemsetAsync(cnt, 0, H * sizeof(int), s), "memset"));
    PTRY(check_cuda(cudaMemsetAsync(cursor, 0, H * sizeof(int), s), "memset"));
    inc_count_kernel<<<grid_for(10 * n_tets, 256), 256, 0, s>>>(n_tets, n_edges, H, tet_to_field, cnt, h->h.dev_status);
    PTRY(check_cuda(cudaGetLastError(), "inc_count_kernel"));
    {
        int dstat = 0;
        PTRY(check_cuda(cudaMemcpyAsync(&dstat, h->h.dev_status, sizeof(int), cudaMemcpyDeviceToHost, s), "status"));
        PTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        if (dstat & DEV_BAD_INDEX) {
            set_error("emfem_plan_create: tet_to_field is inconsistent with n_edges/n_tris (Nedelec2 layout)");
            cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), s);
            st = EMFEM_ERR_DEVICE_CHECK;
            goto fail;
        }
    }
    PTRY(exclusive_scan_i32(&h->h, cnt, p->inc_ptr, H, scratch));
    inc_fill_kernel<<<grid_for(10 * n_tets, 256), 256, 0, s>>>(n_tets, n_edges, tet_to_field, p->inc_ptr, cursor, p->inc_code, H);
    PTRY(check_cuda(cudaGetLastError(), "inc_fill_kernel"));
    inc_sort_kernel<<<grid_for(H, 256), 256, 0, s>>>(H, p->inc_ptr, p->inc_code);
    PTRY(check_cuda(cudaGetLastError(), "inc_sort_kernel"));
    cols_count_kernel<<<grid_for(H, SYM_WARPS), 32 * SYM_WARPS, 0, s>>>(H, n_tets, tet_to_field, p->inc_ptr,
                                                                       p->inc_code, tmp, m, h->h.dev_status);
    PTRY(check_cuda(cudaGetLastError(), "cols_count_kernel"));
    PTRY(exclusive_scan_i32(&h->h, m, p->mptr, H, scratch));
    {
        int summ = 0, dstat = 0;
        PTRY(check_cuda(cudaMemcpyAsync(&summ, p->mptr + H, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        PTRY(check_cuda(cudaMemcpyAsync(&dstat, h->h.dev_status, sizeof(int), cudaMemcpyDeviceToHost, s), "status"));
        PTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        if (dstat & DEV_CAPACITY) {
            set_error("emfem_plan_create: an edge or face is shared by more than %d tets", SYM_CAP / 10);
            cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), s);
            st = EMFEM_ERR_DEVICE_CHECK;
            goto fail;
        }
        p->sum_m = summ;
        p->nnz = 4LL * summ;
        if (p->nnz >= (1LL << 31)) { set_error("emfem_plan_create: nnz exceeds int32"); st = EMFEM_ERR_INVALID_ARG; goto fail; }
    }
    PTRY(check_cuda(cudaMalloc(&p->S, (size_t)p->sum_m * sizeof(int)), "cudaMalloc(S)"));
    cols_fill_kernel<<<grid_for(H, 128), 128, 0, s>>>(H, n_tets, tet_to_field, p->inc_ptr, p->inc_code, tmp, p->mptr,
                                                      p->S, p->rec, h->h.dev_status);
    PTRY(check_cuda(cudaGetLastError(), "cols_fill_kernel"));
    {
        // greedy chunks of whole entities of one kind with at most CH incidences each, per variant
        std::vector<int> hptr(H + 1);
        PTRY(check_cuda(cudaMemcpyAsync(hptr.data(), p->inc_ptr, (H + 1) * sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        PTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        int maxdeg = 0;
        for (long long X = 0; X < H; X++) maxdeg = std::max(maxdeg, hptr[X + 1] - hptr[X]);
        p->variant = -1;
        for (int v = 0; v < N_ASM_VARIANTS; v++) {
            const int CH = ASM_VARIANTS[v].ch;
            if (maxdeg > CH) continue;  // an entity must fit one chunk
            std::vector<int> cptr;
            cptr.push_back(0);
            int cur = 0;
            for (long long X = 0; X < H; X++) {
                int deg = hptr[X + 1] - hptr[X];
                bool kind_change = X == n_edges && X > cptr.back();
                bool full = (cur + deg > CH || X - cptr.back() >= CH) && X > cptr.back();
                if (full || kind_change) { cptr.push_back((int)X); cur = 0; }
                cur += deg;
            }
            cptr.push_back((int)H);
            p->n_chunks[v] = (int)cptr.size() - 1;
            PTRY(check_cuda(cudaMalloc(&p->chunk_ptr[v], cptr.size() * sizeof(int)), "cudaMalloc(chunk_ptr)"));
            PTRY(check_cuda(cudaMemcpyAsync(p->chunk_ptr[v], cptr.data(), cptr.size() * sizeof(int), cudaMemcpyHostToDevice, s), "copy"));
            PTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
            if (p->variant < 0) p->variant = v;
        }
        // default: the incidence-major 64/320 variant (fastest measured on B200) when it fits
        if (p->variant >= 0 && p->n_chunks[DEFAULT_ASM_VARIANT] > 0) p->variant = DEFAULT_ASM_VARIANT;
        if (p->variant < 0) {
            set_error("emfem_plan_create: an edge or face is shared by %d tets (at most 64 supported)", maxdeg);
            st = EMFEM_ERR_INVALID_ARG;
            goto fail;
        }
        PTRY(check_cuda(set_asm_smem_attributes(), "cudaFuncSetAttribute"));
    }
    PTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
    cudaFree(cnt); cudaFree(cursor); cudaFree(scratch); cudaFree(tmp); cudaFree(m);
    *out = p;
    return EMFEM_OK;
fail:
    cudaFree(cnt); cudaFree(cursor); cudaFree(scratch); cudaFree(tmp); cudaFree(m);
    plan_free(p);
    return st;
#undef PTRY
}

int emfem_plan_info(emfem_plan p, int64_t* n_field, int64_t* nnz) {
    EMFEM_REQUIRE(p, "emfem_plan_info: null plan");
    if (n_field) *n_field = p->N;
    if (nnz) *nnz = p->nnz;
    return EMFEM_OK;
}

int emfem_plan_destroy(emfem_plan p) {
    plan_free(p);
    return EMFEM_OK;
}

int emfem_plan_export_csr(emfem_plan p, int32_t* indptr, int32_t* indices) {
    EMFEM_REQUIRE(p && indptr && indices, "emfem_plan_export_csr: null argument");
    cudaStream_t s = p->h->stream;
    export_indptr_kernel<<<grid_for(p->N + 1, 256), 256, 0, s>>>(p->H, p->mptr, indptr);
    EMFEM_LAUNCH("export_indptr_kernel");
    export_indices_kernel<<<grid_for(p->sum_m, 256), 256, 0, s>>>(p->H, p->sum_m, p->mptr, p->S, indices);
    EMFEM_LAUNCH("export_indices_kernel");
    return EMFEM_OK;
}

int emfem_plan_assemble(emfem_plan p, int64_t n_nodes, int64_t n_edges, const double* nodes,
                        const int64_t* tets, const int64_t* tet_to_edge, const double* edge_lengths,
                        const void* ur, const void* er, void* E_vals, void* B_vals) {
    EMFEM_REQUIRE(p && nodes && tets && tet_to_edge && edge_lengths && ur && er && E_vals && B_vals,
                  "emfem_plan_assemble: null argument");
    EMFEM_REQUIRE(n_edges == p->ne, "emfem_plan_assemble: n_edges differs from the plan's");
    cudaStream_t s = p->h->stream;
    tet_invariants_kernel<<<grid_for(p->nt, 128), 128, 0, s>>>(p->nt, n_nodes, n_edges, nodes, tets, tet_to_edge,
                                                                edge_lengths, (const double2*)ur, (const double2*)er,
                                                                p->inv, p->h->dev_status);
    EMFEM_LAUNCH("tet_invariants_kernel");
    const int v = p->variant;
    launch_asm_variant(v, (unsigned)p->n_chunks[v], s, p->chunk_ptr[v], p->H, p->mptr, p->inc_ptr, p->inc_code,
                       (const uint4*)p->rec, p->inv, (double2*)E_vals, (double2*)B_vals);
    EMFEM_LAUNCH("assemble_chunk_kernel");
    return EMFEM_OK;
}

int emfem_plan_variants(emfem_plan p, int* n_variants, int* current) {
    EMFEM_REQUIRE(p, "emfem_plan_variants: null plan");
    if (n_variants) *n_variants = N_ASM_VARIANTS;
    if (current) *current = p->variant;
    return EMFEM_OK;
}

int emfem_plan_variant_info(emfem_plan p, int variant, int* chunk, int* threads, int* available) {
    EMFEM_REQUIRE(p && variant >= 0 && variant < N_ASM_VARIANTS, "emfem_plan_variant_info: bad variant");
    if (chunk) *chunk = ASM_VARIANTS[variant].ch;
    if (threads) *threads = ASM_VARIANTS[variant].nt;
    if (available) *available = p->chunk_ptr[variant] != nullptr ? 1 : 0;
    return EMFEM_OK;
}

int emfem_plan_set_variant(emfem_plan p, int variant) {
    EMFEM_REQUIRE(p && variant >= 0 && variant < N_ASM_VARIANTS, "emfem_plan_set_variant: bad variant");
    EMFEM_REQUIRE(p->chunk_ptr[variant] != nullptr, "emfem_plan_set_variant: variant %d cannot hold this mesh's incidences", variant);
    p->variant = variant;
    return EMFEM_OK;
}

int emfem_plan_find_slots(emfem_plan p, int64_t n, const int64_t* rows, const int64_t* cols, int32_t* slots) {
    EMFEM_REQUIRE(p && rows && cols && slots && n >= 0, "emfem_plan_find_slots: bad argument");
    if (n == 0) return EMFEM_OK;
    find_slots_kernel<<<grid_for(n, 256), 256, 0, p->h->stream>>>(n, p->H, p->mptr, p->S, rows, cols, slots);
    EMFEM_LAUNCH("find_slots_kernel");
    return EMFEM_OK;
}

}  // extern "C"
