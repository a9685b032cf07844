// Handle, error reporting, device status word, and small generic kernels (scan, gather-sum).
#include "emfem_internal.cuh"

namespace emfem {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

// ---- exclusive scan (three passes: block sums, scan of block sums, add) -----------------
constexpr int SCAN_BLOCK = 1024;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh, int& total) {
    // warp-level inclusive scan, then across warps
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        int s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    int base = warp > 0 ? sh[warp - 1] : 0;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void scan_blocks_kernel(const int* __restrict__ in, int* __restrict__ out, long long n,
                                   int* __restrict__ block_sums) {
    __shared__ int sh[32];
    long long i = (long long)blockIdx.x * SCAN_BLOCK + threadIdx.x;
    int v = i < n ? in[i] : 0;
    int total;
    int ex = block_exclusive_scan(v, sh, total);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void scan_add_kernel(int* __restrict__ out, long long n, const int* __restrict__ block_off) {
    long long i = (long long)blockIdx.x * SCAN_BLOCK + threadIdx.x;
    if (i < n) out[i] += block_off[blockIdx.x];
}

__global__ void scan_total_kernel(int* out, long long n, const int* block_off, const int* block_sums, int nb) {
    out[n] = block_off[nb - 1] + block_sums[nb - 1];
}

size_t scan_scratch_ints(long long n) {
    long long nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    if (nb < 1) nb = 1;
    return (size_t)(2 * nb + 1) + (nb > 1 ? scan_scratch_ints(nb) : 0);
}

int exclusive_scan_i32(Handle* h, const int* in, int* out, long long n, int* scratch) {
    long long nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    if (nb < 1) nb = 1;
    int* bsum = scratch;
    int* boff = scratch + nb;
    if (n > 0) {
        scan_blocks_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, h->stream>>>(in, out, n, bsum);
        EMFEM_LAUNCH("scan_blocks_kernel");
    } else {
        EMFEM_CUDA(cudaMemsetAsync(bsum, 0, sizeof(int), h->stream));
    }
    if (nb == 1) {
        EMFEM_CUDA(cudaMemsetAsync(boff, 0, sizeof(int), h->stream));
    } else {
        EMFEM_TRY(exclusive_scan_i32(h, bsum, boff, nb, scratch + 2 * nb + 1));
        scan_add_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, h->stream>>>(out, n, boff);
        EMFEM_LAUNCH("scan_add_kernel");
    }
    scan_total_kernel<<<1, 1, 0, h->stream>>>(out, n, boff, bsum, (int)nb);
    EMFEM_LAUNCH("scan_total_kernel");
    return EMFEM_OK;
}

// ---- deterministic segmented gather-sum ----------------------------------------------------
__global__ void gather_sum_kernel(long long n_out, const int* __restrict__ seg, const int* __restrict__ idx,
                                  const double2* __restrict__ src, double2* __restrict__ out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = seg[i]; k < seg[i + 1]; k++) {
        double2 v = src[idx[k]];
        acc.x += v.x;
        acc.y += v.y;
    }
    out[i] = acc;
}

}  // namespace emfem

using namespace emfem;

extern "C" {

int emfem_version(void) { return 10000; }

int emfem_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return EMFEM_ERR_INVALID_ARG;
    strncpy(buf, g_err, len - 1);
    buf[len - 1] = 0;
    return EMFEM_OK;
}

int emfem_create(emfem_handle* out, int device, void* stream) {
    EMFEM_REQUIRE(out != nullptr, "emfem_create: null output pointer");
    EMFEM_CUDA(cudaSetDevice(device));
    emfem_handle h = new emfem_handle_s();
    h->h.device = device;
    h->h.stream = (cudaStream_t)stream;
    int st = check_cuda(cudaMalloc(&h->h.dev_status, sizeof(int)), "cudaMalloc(status)");
    if (st != EMFEM_OK) { delete h; return st; }
    st = check_cuda(cudaMemset(h->h.dev_status, 0, sizeof(int)), "cudaMemset(status)");
    if (st != EMFEM_OK) { cudaFree(h->h.dev_status); delete h; return st; }
    cudaDeviceGetAttribute(&h->h.num_sms, cudaDevAttrMultiProcessorCount, device);
    *out = h;
    return EMFEM_OK;
}

int emfem_set_stream(emfem_handle h, void* stream) {
    EMFEM_REQUIRE(h != nullptr, "emfem_set_stream: null handle");
    h->h.stream = (cudaStream_t)stream;
    return EMFEM_OK;
}

int emfem_destroy(emfem_handle h) {
    if (!h) return EMFEM_OK;
    cudaSetDevice(h->h.device);
    if (h->h.dev_status) cudaFree(h->h.dev_status);
    delete h;
    return EMFEM_OK;
}

int emfem_device_status(emfem_handle h, int* status) {
    EMFEM_REQUIRE(h != nullptr && status != nullptr, "emfem_device_status: null argument");
    int v = 0;
    EMFEM_CUDA(cudaMemcpyAsync(&v, h->h.dev_status, sizeof(int), cudaMemcpyDeviceToHost, h->h.stream));
    EMFEM_CUDA(cudaStreamSynchronize(h->h.stream));
    EMFEM_CUDA(cudaMemsetAsync(h->h.dev_status, 0, sizeof(int), h->h.stream));
    *status = v;
    return EMFEM_OK;
}

int emfem_segmented_gather_sum(emfem_handle h, int64_t n_out, const int32_t* seg, const int32_t* idx,
                               const void* src, void* out) {
    EMFEM_REQUIRE(h && seg && idx && src && out && n_out >= 0, "emfem_segmented_gather_sum: bad argument");
    if (n_out == 0) return EMFEM_OK;
    gather_sum_kernel<<<grid_for(n_out, 256), 256, 0, h->h.stream>>>(n_out, seg, idx, (const double2*)src, (double2*)out);
    EMFEM_LAUNCH("gather_sum_kernel");
    return EMFEM_OK;
}

}  // extern "C"
