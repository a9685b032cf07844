// Device mesh connectivity in Mesh3D conventions (src/emerge/_emerge/mesh3d.py:387-497).
//
// The reference builds the unique edge / triangle lists with Python sets over the tets, sorts them,
// and fills tet_to_edge, tet_to_tri, tri_to_edge, tri_to_tet and edge_lengths in Python loops.  Here
// every candidate edge (a, b) and triangle (a, b, c) of every tet (vertices sorted, a smallest) is
// bucketed by its smallest node a with a counting scatter, each bucket is sorted and deduplicated,
// and buckets are concatenated in node order — which is exactly lexicographic order of the sorted
// tuples, so edge and triangle ids equal the reference's.  Lookups are binary searches inside the
// bucket of the smallest node.  tri_to_tet keeps, per triangle, the two smallest tet ids (the
// reference appends tets in ascending order).  All steps are deterministic.
#include "emfem_internal.cuh"

#include <vector>

namespace emfem {

__device__ __forceinline__ void sort4(int64_t v[4]) {
    int64_t t;
#define CSWAP(i, j) if (v[j] < v[i]) { t = v[i]; v[i] = v[j]; v[j] = t; }
    CSWAP(0, 1) CSWAP(2, 3) CSWAP(0, 2) CSWAP(1, 3) CSWAP(1, 2)
#undef CSWAP
}

__device__ __forceinline__ void tet_vertices(const int64_t* tets, long long nt, long long t, int64_t v[4]) {
    for (int i = 0; i < 4; i++) v[i] = tets[i * nt + t];
}

__global__ void cand_count_kernel(long long nt, long long nn, const int64_t* __restrict__ tets,
                                  int* __restrict__ ecnt, int* __restrict__ fcnt, int* status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int64_t v[4];
    tet_vertices(tets, nt, t, v);
    for (int i = 0; i < 4; i++) if (v[i] < 0 || v[i] >= nn) { flag(status, DEV_BAD_INDEX); return; }
    sort4(v);
    if (v[0] == v[1] || v[1] == v[2] || v[2] == v[3]) { flag(status, DEV_DEGENERATE); return; }
    // edges (a,b) with a = smaller node: a = v0 for 3 edges, v1 for 2, v2 for 1
    atomicAdd(&ecnt[v[0]], 3); atomicAdd(&ecnt[v[1]], 2); atomicAdd(&ecnt[v[2]], 1);
    // faces (a,b,c): a = v0 for 3 faces, v1 for 1
    atomicAdd(&fcnt[v[0]], 3); atomicAdd(&fcnt[v[1]], 1);
}

__global__ void cand_fill_kernel(long long nt, const int64_t* __restrict__ tets, const int* __restrict__ eptr,
                                 int* __restrict__ ecur, int* __restrict__ ecand, const int* __restrict__ fptr,
                                 int* __restrict__ fcur, long long* __restrict__ fcand, long long nn) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int64_t v[4];
    tet_vertices(tets, nt, t, v);
    for (int i = 0; i < 4; i++) if (v[i] < 0 || v[i] >= nn) return;
    sort4(v);
    if (v[0] == v[1] || v[1] == v[2] || v[2] == v[3]) return;
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 4; j++) {
            int p = atomicAdd(&ecur[v[i]], 1);
            ecand[eptr[v[i]] + p] = (int)v[j];
        }
    const int fi[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (int f = 0; f < 4; f++) {
        int64_t a = v[fi[f][0]], b = v[fi[f][1]], c = v[fi[f][2]];
        int p = atomicAdd(&fcur[a], 1);
        fcand[fptr[a] + p] = b * nn + c;
    }
}

// per node: sort its bucket, deduplicate in place, count unique entries
template <typename K>
__global__ void bucket_unique_kernel(long long nn, const int* __restrict__ ptr, K* __restrict__ cand,
                                     int* __restrict__ nuniq) {
    long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nn) return;
    int b = ptr[a], e = ptr[a + 1];
    for (int i = b + 1; i < e; i++) {
        K v = cand[i];
        int j = i - 1;
        while (j >= b && cand[j] > v) { cand[j + 1] = cand[j]; j--; }
        cand[j + 1] = v;
    }
    int u = 0;
    for (int i = b; i < e; i++)
        if (i == b || cand[i] != cand[i - 1]) cand[b + u++] = cand[i];
    nuniq[a] = u;
}

template <typename K>
__device__ __forceinline__ int bucket_find(const K* cand, int b, int u, K key) {
    int lo = 0, hi = u - 1;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (cand[b + mid] < key) lo = mid + 1; else hi = mid; }
    return (u > 0 && cand[b + lo] == key) ? lo : -1;
}

__global__ void emit_edges_kernel(long long nn, const int* __restrict__ ptr, const int* __restrict__ cand,
                                  const int* __restrict__ uptr, const double* __restrict__ nodes,
                                  int64_t* __restrict__ edges, long long ne, double* __restrict__ elen) {
    long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nn) return;
    int b = ptr[a], u0 = uptr[a], u = uptr[a + 1] - u0;
    for (int k = 0; k < u; k++) {
        long long id = u0 + k, c = cand[b + k];
        edges[id] = a;
        edges[ne + id] = c;
        double dx = nodes[a] - nodes[c], dy = nodes[nn + a] - nodes[nn + c], dz = nodes[2 * nn + a] - nodes[2 * nn + c];
        // ((dx^2 + dy^2) + dz^2) with every operation rounded separately (no FMA contraction): the
        // reference's np.sqrt(np.sum(d**2, axis=0)) bit for bit
        elen[id] = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    }
}

__global__ void emit_tris_kernel(long long nn, const int* __restrict__ ptr, const long long* __restrict__ cand,
                                 const int* __restrict__ uptr, int64_t* __restrict__ tris, long long nf) {
    long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nn) return;
    int b = ptr[a], u0 = uptr[a], u = uptr[a + 1] - u0;
    for (int k = 0; k < u; k++) {
        long long id = u0 + k, key = cand[b + k];
        tris[id] = a;
        tris[nf + id] = key / nn;
        tris[2 * nf + id] = key % nn;
    }
}

__device__ __forceinline__ long long edge_id(const int* eptr, const int* ecand, const int* euptr, int64_t i, int64_t j) {
    int64_t a = i < j ? i : j, c = i < j ? j : i;
    int k = bucket_find<int>(ecand, eptr[a], euptr[a + 1] - euptr[a], (int)c);
    return k < 0 ? -1 : (long long)euptr[a] + k;
}

__device__ __forceinline__ long long tri_id(const int* fptr, const long long* fcand, const int* fuptr, long long nn,
                                            int64_t i, int64_t j, int64_t k) {
    int64_t v[3] = {i, j, k}, t;
    if (v[1] < v[0]) { t = v[0]; v[0] = v[1]; v[1] = t; }
    if (v[2] < v[1]) { t = v[1]; v[1] = v[2]; v[2] = t; }
    if (v[1] < v[0]) { t = v[0]; v[0] = v[1]; v[1] = t; }
    int q = bucket_find<long long>(fcand, fptr[v[0]], fuptr[v[0] + 1] - fuptr[v[0]], v[1] * nn + v[2]);
    return q < 0 ? -1 : (long long)fuptr[v[0]] + q;
}

__global__ void tet_maps_kernel(long long nt, long long nn, const int64_t* __restrict__ tets,
                                const int* eptr, const int* ecand, const int* euptr,
                                const int* fptr, const long long* fcand, const int* fuptr,
                                int64_t* __restrict__ t2e, int64_t* __restrict__ t2t,
                                long long* __restrict__ first, unsigned long long* __restrict__ count,
                                int* status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int64_t v[4];
    tet_vertices(tets, nt, t, v);
    for (int i = 0; i < 4; i++) if (v[i] < 0 || v[i] >= nn) return;
    const int ep[6] = {0, 0, 0, 1, 3, 2}, eq[6] = {1, 2, 3, 2, 1, 3};
    for (int e = 0; e < 6; e++) {
        long long id = edge_id(eptr, ecand, euptr, v[ep[e]], v[eq[e]]);
        if (id < 0) flag(status, DEV_BAD_INDEX);
        t2e[e * nt + t] = id;
    }
    const int fv[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 2, 3}};
    for (int f = 0; f < 4; f++) {
        long long id = tri_id(fptr, fcand, fuptr, nn, v[fv[f][0]], v[fv[f][1]], v[fv[f][2]]);
        if (id < 0) { flag(status, DEV_BAD_INDEX); t2t[f * nt + t] = -1; continue; }
        t2t[f * nt + t] = id;
        atomicMin((unsigned long long*)&first[id], (unsigned long long)t);
        atomicAdd(&count[id], 1ULL);
    }
}

__global__ void second_tet_kernel(long long nt, const int64_t* __restrict__ t2t, const long long* __restrict__ first,
                                  long long* __restrict__ second) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    for (int f = 0; f < 4; f++) {
        long long id = t2t[f * nt + t];
        if (id >= 0 && first[id] != t) atomicMin((unsigned long long*)&second[id], (unsigned long long)t);
    }
}

__global__ void tri_maps_kernel(long long nf, long long nn, const int64_t* __restrict__ tris,
                                const int* eptr, const int* ecand, const int* euptr,
                                const long long* __restrict__ first, const long long* __restrict__ second,
                                const unsigned long long* __restrict__ count, int64_t* __restrict__ tri2e,
                                int64_t* __restrict__ tri2tet, int* status) {
    long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nf) return;
    int64_t i1 = tris[it], i2 = tris[nf + it], i3 = tris[2 * nf + it];
    long long e1 = edge_id(eptr, ecand, euptr, i1, i2), e2 = edge_id(eptr, ecand, euptr, i2, i3),
              e3 = edge_id(eptr, ecand, euptr, i1, i3);
    if (e1 < 0 || e2 < 0 || e3 < 0) flag(status, DEV_BAD_INDEX);
    if (count[it] > 2) flag(status, DEV_CAPACITY);
    tri2e[it] = e1; tri2e[nf + it] = e2; tri2e[2 * nf + it] = e3;
    const long long NONE = 0x7fffffffffffffffLL;
    tri2tet[it] = first[it] == NONE ? EMFEM_MISSING_ID : first[it];
    tri2tet[nf + it] = second[it] == NONE ? EMFEM_MISSING_ID : second[it];
}

__global__ void fill_ll_kernel(long long n, long long* p, long long v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace emfem

using namespace emfem;

struct emfem_conn_s {
    Handle* h = nullptr;
    long long nn = 0, nt = 0, ne = 0, nf = 0;
    int *eptr = nullptr, *ecand = nullptr, *euptr = nullptr;
    int *fptr = nullptr, *fuptr = nullptr;
    long long* fcand = nullptr;
};

static void conn_free(emfem_conn c) {
    if (!c) return;
    cudaFree(c->eptr); cudaFree(c->ecand); cudaFree(c->euptr);
    cudaFree(c->fptr); cudaFree(c->fuptr); cudaFree(c->fcand);
    delete c;
}

extern "C" {

int emfem_mesh_connect_create(emfem_handle h, int64_t n_nodes, int64_t n_tets, const int64_t* tets, emfem_conn* out) {
    EMFEM_REQUIRE(h && tets && out && n_nodes > 0 && n_tets > 0, "emfem_mesh_connect_create: bad argument");
    EMFEM_REQUIRE(n_nodes < (1LL << 31) && 6 * n_tets < (1LL << 31) && n_nodes < (1LL << 31) / 4,
                  "emfem_mesh_connect_create: mesh too large for int32 indexing");
    cudaStream_t s = h->h.stream;
    emfem_conn c = new emfem_conn_s();
    c->h = &h->h; c->nn = n_nodes; c->nt = n_tets;
    long long nn = n_nodes;
    int *ecnt = nullptr, *fcnt = nullptr, *ecur = nullptr, *fcur = nullptr, *eu = nullptr, *fu = nullptr, *scratch = nullptr;
    int st = EMFEM_OK;
    size_t nscr = scan_scratch_ints(nn);
#define CTRY(x) do { st = (x); if (st != EMFEM_OK) goto fail; } while (0)
    CTRY(check_cuda(cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), s), "memset"));
    CTRY(check_cuda(cudaMalloc(&ecnt, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&fcnt, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&ecur, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&fcur, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&eu, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&fu, nn * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&scratch, nscr * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->eptr, (nn + 1) * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->fptr, (nn + 1) * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->euptr, (nn + 1) * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->fuptr, (nn + 1) * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->ecand, 6 * n_tets * sizeof(int)), "cudaMalloc"));
    CTRY(check_cuda(cudaMalloc(&c->fcand, 4 * n_tets * sizeof(long long)), "cudaMalloc"));
    CTRY(check_cuda(cudaMemsetAsync(ecnt, 0, nn * sizeof(int), s), "memset"));
    CTRY(check_cuda(cudaMemsetAsync(fcnt, 0, nn * sizeof(int), s), "memset"));
    CTRY(check_cuda(cudaMemsetAsync(ecur, 0, nn * sizeof(int), s), "memset"));
    CTRY(check_cuda(cudaMemsetAsync(fcur, 0, nn * sizeof(int), s), "memset"));
    cand_count_kernel<<<grid_for(n_tets, 256), 256, 0, s>>>(n_tets, nn, tets, ecnt, fcnt, h->h.dev_status);
    CTRY(check_cuda(cudaGetLastError(), "cand_count_kernel"));
    {
        int dstat = 0;
        CTRY(check_cuda(cudaMemcpyAsync(&dstat, h->h.dev_status, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        CTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        if (dstat) {
            set_error("emfem_mesh_connect_create: a tet has an out-of-range or repeated node id");
            cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), s);
            st = EMFEM_ERR_DEVICE_CHECK;
            goto fail;
        }
    }
    CTRY(exclusive_scan_i32(&h->h, ecnt, c->eptr, nn, scratch));
    CTRY(exclusive_scan_i32(&h->h, fcnt, c->fptr, nn, scratch));
    cand_fill_kernel<<<grid_for(n_tets, 256), 256, 0, s>>>(n_tets, tets, c->eptr, ecur, c->ecand, c->fptr, fcur, c->fcand, nn);
    CTRY(check_cuda(cudaGetLastError(), "cand_fill_kernel"));
    bucket_unique_kernel<int><<<grid_for(nn, 256), 256, 0, s>>>(nn, c->eptr, c->ecand, eu);
    bucket_unique_kernel<long long><<<grid_for(nn, 256), 256, 0, s>>>(nn, c->fptr, c->fcand, fu);
    CTRY(check_cuda(cudaGetLastError(), "bucket_unique_kernel"));
    CTRY(exclusive_scan_i32(&h->h, eu, c->euptr, nn, scratch));
    CTRY(exclusive_scan_i32(&h->h, fu, c->fuptr, nn, scratch));
    {
        int ne = 0, nf = 0;
        CTRY(check_cuda(cudaMemcpyAsync(&ne, c->euptr + nn, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        CTRY(check_cuda(cudaMemcpyAsync(&nf, c->fuptr + nn, sizeof(int), cudaMemcpyDeviceToHost, s), "copy"));
        CTRY(check_cuda(cudaStreamSynchronize(s), "sync"));
        c->ne = ne; c->nf = nf;
    }
    cudaFree(ecnt); cudaFree(fcnt); cudaFree(ecur); cudaFree(fcur); cudaFree(eu); cudaFree(fu); cudaFree(scratch);
    *out = c;
    return EMFEM_OK;
fail:
    cudaFree(ecnt); cudaFree(fcnt); cudaFree(ecur); cudaFree(fcur); cudaFree(eu); cudaFree(fu); cudaFree(scratch);
    conn_free(c);
    return st;
#undef CTRY
}

int emfem_mesh_connect_info(emfem_conn c, int64_t* n_edges, int64_t* n_tris) {
    EMFEM_REQUIRE(c, "emfem_mesh_connect_info: null");
    if (n_edges) *n_edges = c->ne;
    if (n_tris) *n_tris = c->nf;
    return EMFEM_OK;
}

int emfem_mesh_connect_export(emfem_conn c, const double* nodes, const int64_t* tets, int64_t* edges, int64_t* tris,
                              int64_t* tet_to_edge, int64_t* tet_to_tri, int64_t* tri_to_edge, int64_t* tri_to_tet,
                              double* edge_lengths) {
    EMFEM_REQUIRE(c && nodes && tets && edges && tris && tet_to_edge && tet_to_tri && tri_to_edge && tri_to_tet &&
                  edge_lengths, "emfem_mesh_connect_export: null argument");
    cudaStream_t s = c->h->stream;
    long long nn = c->nn, nt = c->nt, ne = c->ne, nf = c->nf;
    emit_edges_kernel<<<grid_for(nn, 256), 256, 0, s>>>(nn, c->eptr, c->ecand, c->euptr, nodes, edges, ne, edge_lengths);
    EMFEM_LAUNCH("emit_edges_kernel");
    emit_tris_kernel<<<grid_for(nn, 256), 256, 0, s>>>(nn, c->fptr, c->fcand, c->fuptr, tris, nf);
    EMFEM_LAUNCH("emit_tris_kernel");
    // per triangle: smallest tet id, second smallest, number of tets (3 nf words)
    long long* firstsec = nullptr;
    EMFEM_CUDA(cudaMallocAsync(&firstsec, 3 * nf * sizeof(long long), s));
    unsigned long long* count = (unsigned long long*)(firstsec + 2 * nf);
    fill_ll_kernel<<<grid_for(2 * nf, 256), 256, 0, s>>>(2 * nf, firstsec, 0x7fffffffffffffffLL);
    EMFEM_CUDA(cudaMemsetAsync(count, 0, nf * sizeof(long long), s));
    tet_maps_kernel<<<grid_for(nt, 256), 256, 0, s>>>(nt, nn, tets, c->eptr, c->ecand, c->euptr, c->fptr, c->fcand,
                                                     c->fuptr, tet_to_edge, tet_to_tri, firstsec, count,
                                                     c->h->dev_status);
    second_tet_kernel<<<grid_for(nt, 256), 256, 0, s>>>(nt, tet_to_tri, firstsec, firstsec + nf);
    tri_maps_kernel<<<grid_for(nf, 256), 256, 0, s>>>(nf, nn, tris, c->eptr, c->ecand, c->euptr, firstsec, firstsec + nf,
                                                     count, tri_to_edge, tri_to_tet, c->h->dev_status);
    EMFEM_LAUNCH("mesh connectivity maps");
    EMFEM_CUDA(cudaFreeAsync(firstsec, s));
    return EMFEM_OK;
}

int emfem_mesh_connect_destroy(emfem_conn c) {
    conn_free(c);
    return EMFEM_OK;
}

}  // extern "C"
