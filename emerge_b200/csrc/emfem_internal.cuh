// Internal plumbing shared by the libemfem translation units: handle, error text, launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <stdarg.h>

#include "../../include/emfem.h"

namespace emfem {

// Sticky device-side status bits (written by kernels instead of trapping).
enum : int {
    DEV_OK = 0,
    DEV_BAD_INDEX = 1,        // an index read from an input was outside its declared range
    DEV_DEGENERATE = 2,       // zero-volume tet / zero-area triangle
    DEV_NONFINITE = 4,        // NaN or Inf in an input tensor
    DEV_CAPACITY = 8,         // a per-entity list exceeded its fixed capacity
    DEV_BREAKDOWN = 16,       // Krylov breakdown (rho or p.q == 0)
};

void set_error(const char* fmt, ...);

struct Handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int* dev_status = nullptr;      // one int, sticky bits above
    int num_sms = 148;
};

inline int check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return EMFEM_ERR_CUDA;
    }
    return EMFEM_OK;
}

#define EMFEM_TRY(expr)                                   \
    do {                                                  \
        int _st = (expr);                                 \
        if (_st != EMFEM_OK) return _st;                  \
    } while (0)

#define EMFEM_CUDA(call) EMFEM_TRY(::emfem::check_cuda((call), #call))
#define EMFEM_LAUNCH(what) EMFEM_TRY(::emfem::check_cuda(cudaGetLastError(), what))

#define EMFEM_REQUIRE(cond, ...)                          \
    do {                                                  \
        if (!(cond)) {                                    \
            ::emfem::set_error(__VA_ARGS__);              \
            return EMFEM_ERR_INVALID_ARG;                 \
        }                                                 \
    } while (0)

inline unsigned grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (unsigned)g;
}

__device__ __forceinline__ void flag(int* st, int bit) { atomicOr(st, bit); }

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total) on the handle's stream,
// using scratch of scan_scratch_ints(n) ints.  Deterministic; total must fit int32.
size_t scan_scratch_ints(long long n);
int exclusive_scan_i32(Handle* h, const int* in, int* out, long long n, int* scratch);

}  // namespace emfem

struct emfem_handle_s { emfem::Handle h; };
