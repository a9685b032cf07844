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

// patch row map (sweep_solve.cu): pmap[rows[k]] = k for the Robin patch rows
void launch_patch_map(long long np, const int* rows, int* pmap, cudaStream_t s);

}  // namespace emfem

struct emfem_handle_s { emfem::Handle h; };

// Auxiliary nodal space (aux_space.cu); the Krylov solver reads it directly.
struct emfem_aux_s {
    emfem::Handle* h = nullptr;
    long long nn = 0, ne = 0, nf = 0, n = 0, na = 0, nnz_gt = 0, nnz_inc = 0;
    int* gcol = nullptr;        // G rows, ELL [n][6]
    double* gval = nullptr;
    int* gt_ptr = nullptr;      // G^T, CSR [na + 1]
    int* gt_row = nullptr;
    double* gt_val = nullptr;
    int* inc_ptr = nullptr;     // vertex-edge incidence graph, CSR [na + 1]
    int* inc = nullptr;
    float* inv_deg = nullptr;   // [na]
    uint8_t* atype = nullptr;   // [na] 0 vertex, 1 edge
    uint8_t* amask = nullptr;   // [na] usable (support entirely on free DOFs)
    double2* dE = nullptr;      // [na] diag(G^T E G)
    double2* dB = nullptr;      // [na] diag(G^T B G)
    double2* dR = nullptr;      // [EMFEM_MAX_PORTS][na] diag(G^T R_p G)
    int nports = 0;
    bool have_operator = false;
    float* params = nullptr;    // [EMFEM_MPNN_NPARAMS], caller-owned device memory
    void* kbuf = nullptr;       // solve-time buffers (emfem_aux_reserve)
    size_t kbuf_bytes = 0;
    int* agroup = nullptr;      // [na] group of every aux node in a grouped (multi-mesh) solve, or null
    int ngroups = 1;
};

namespace emfem {
template <typename T>
int aux_correct(const emfem_aux_s* a, int S, bool learned, const T* dinv, const T* v, const uint8_t* mask, T* z,
                cudaStream_t s);
template <typename T>
int aux_setup_dinv(const emfem_aux_s* a, int S, int nsys, const double* k0sq, const double* gamma, T* dinv,
                   cudaStream_t s);
size_t aux_solve_bytes(const emfem_aux_s* a, int S);
void* aux_dinv_buffer(const emfem_aux_s* a, int S);
}  // namespace emfem

// Multifrontal LU (multifrontal.cu); the Krylov solver applies it as a right preconditioner.
struct emfem_mf_s;
namespace emfem {
int mf_apply(emfem_mf_s* m, int S, const double2* r, double2* x, cudaStream_t s);
int mf_reserved(const emfem_mf_s* m);
}  // namespace emfem
