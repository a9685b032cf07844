// CSR compaction for the frequency-domain system matrix.
//
// The reference forms K = E - B*k0**2 and K + B_p with SciPy sparse arithmetic
// (src/emerge/_emerge/physics/microwave/assembly/assembler.py:255, :350), whose result keeps only the
// entries that are not exactly zero (E's element matrices hold exact zeros; where B is zero too the
// sum is dropped).  emfem_sweep_combine forms the values on the full E/B pattern; these two calls then
// drop the exact zeros in row order, so the device matrix has the reference's CSR layout.
// A warp owns a row: it walks the row in chunks of 32 entries, votes on the nonzero ones and writes
// them at the offset given by the prefix count, so the kept entries stay in column order.
#include "emfem_internal.cuh"

namespace emfem {

__device__ __forceinline__ bool nonzero(double2 v) { return v.x != 0.0 || v.y != 0.0; }

__global__ void count_nonzero_kernel(long long n, const int* __restrict__ indptr, const double2* __restrict__ vals,
                                     int* __restrict__ counts) {
    long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= n) return;
    int b = indptr[row], e = indptr[row + 1];
    int c = 0;
    for (int k = b + lane; k < e; k += 32) c += nonzero(vals[k]) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[row] = c;
}

__global__ void compact_nonzero_kernel(long long n, const int* __restrict__ indptr, const int* __restrict__ indices,
                                       const double2* __restrict__ vals, const int* __restrict__ out_ptr,
                                       int* __restrict__ out_idx, double2* __restrict__ out_vals) {
    long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= n) return;
    int b = indptr[row], e = indptr[row + 1];
    int w = out_ptr[row];
    for (int k0 = b; k0 < e; k0 += 32) {
        int k = k0 + lane;
        bool keep = false;
        double2 v = make_double2(0.0, 0.0);
        if (k < e) {
            v = vals[k];
            keep = nonzero(v);
        }
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            int pos = w + __popc(m & ((1u << lane) - 1u));
            out_idx[pos] = indices[k];
            out_vals[pos] = v;
        }
        w += __popc(m);
    }
}

}  // namespace emfem

using namespace emfem;

extern "C" {

int emfem_csr_drop_zeros_workspace(int64_t n, size_t* bytes) {
    EMFEM_REQUIRE(n > 0 && bytes, "emfem_csr_drop_zeros_workspace: bad argument");
    *bytes = sizeof(int) * ((size_t)n + scan_scratch_ints(n));
    return EMFEM_OK;
}

int emfem_csr_count_nonzero(emfem_handle h, int64_t n, const int32_t* indptr, const void* vals, int32_t* out_indptr,
                            void* workspace, size_t workspace_bytes, int64_t* nnz_out) {
    EMFEM_REQUIRE(h && n > 0 && indptr && vals && out_indptr && workspace && nnz_out,
                  "emfem_csr_count_nonzero: bad argument");
    size_t need = 0;
    EMFEM_TRY(emfem_csr_drop_zeros_workspace(n, &need));
    if (workspace_bytes < need) {
        set_error("emfem_csr_count_nonzero: workspace %zu bytes < %zu", workspace_bytes, need);
        return EMFEM_ERR_WORKSPACE;
    }
    int* counts = (int*)workspace;
    int* scratch = counts + n;
    cudaStream_t s = h->h.stream;
    const int TB = 256;
    count_nonzero_kernel<<<grid_for(n * 32, TB), TB, 0, s>>>(n, indptr, (const double2*)vals, counts);
    EMFEM_LAUNCH("count_nonzero_kernel");
    EMFEM_TRY(exclusive_scan_i32(&h->h, counts, out_indptr, n, scratch));
    int total = 0;
    EMFEM_CUDA(cudaMemcpyAsync(&total, out_indptr + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    EMFEM_CUDA(cudaStreamSynchronize(s));
    *nnz_out = total;
    return EMFEM_OK;
}

int emfem_csr_compact_nonzero(emfem_handle h, int64_t n, const int32_t* indptr, const int32_t* indices,
                              const void* vals, const int32_t* out_indptr, int32_t* out_indices, void* out_vals) {
    EMFEM_REQUIRE(h && n > 0 && indptr && indices && vals && out_indptr && out_indices && out_vals,
                  "emfem_csr_compact_nonzero: bad argument");
    const int TB = 256;
    compact_nonzero_kernel<<<grid_for(n * 32, TB), TB, 0, h->h.stream>>>(
        n, indptr, indices, (const double2*)vals, out_indptr, out_indices, (double2*)out_vals);
    EMFEM_LAUNCH("compact_nonzero_kernel");
    return EMFEM_OK;
}

}  // extern "C"
