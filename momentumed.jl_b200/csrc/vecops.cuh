// Kernel (c): Lanczos vector operations on the device-resident Krylov basis.
//
// The basis V is column-major: column i is V + i * N (N complex entries), stored
// as double2 (FP64) or float2 (mixed precision); every reduction accumulates in
// FP64.  Reductions are two-stage (per-block partials, then one ordered block
// reduction), so results are deterministic run to run.
//
// One Lanczos step j with full reorthogonalisation (classical Gram-Schmidt,
// a second pass only when the norm drops by more than 1/sqrt(2), the
// Daniel-Gragg-Kaufman-Stewart criterion):
//   w = H v_j                      (matvec writes straight into column j+1)
//   c = V[0..j]^H w, |w|^2          k_proj  + k_reduce
//   w -= V[0..j] c, |w|^2           k_update + k_decide
//   (repeat if the norm dropped)   predicated on a device flag
//   alpha_j = Re c_j, beta_j = |w|  k_finalize
//   v_{j+1} = w / beta_j            k_scale
#pragma once
#include "momed_internal.cuh"

namespace momed {

constexpr int kVecThreads = 256;
constexpr int kMaxCols = 136;              // krylovdim + 1 supported by k_proj
constexpr int kColsPerWarp = (kMaxCols + 7) / 8;

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <typename VT> __device__ __forceinline__ VT from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// Host launchers (vecops.cu)
struct RedBuf {
    DevBuf<double2> partial;    // [grid][kMaxCols + 1]
    int grid = 0;
};

template <typename VT>
void vec_proj(const VT* V, int64_t N, int ncols, const VT* w, double2* partial, int grid, const int* active,
              cudaStream_t st);
void vec_reduce(const double2* partial, int grid, int ncols1, double2* out, const int* active, cudaStream_t st);
template <typename VT>
void vec_update(const VT* V, int64_t N, int ncols, const double2* coef, VT* w, double2* partial, int grid,
                const int* active, cudaStream_t st);
// flag = (|w|^2 after < 0.5 |w|^2 before); stores |w|^2 after into scal[1]
void vec_decide(const double2* coefA, int ncols, const double2* partial, int grid, int* flag, double* scal,
                cudaStream_t st);
// alpha/beta of step j; scal[0] = 1 / beta
void vec_finalize(const double2* coefA, const double2* coefB, int ncols, const double2* partial2, int grid,
                  const int* flag, double* scal, double* alpha, double* beta, int j, cudaStream_t st);
template <typename VT>
void vec_scale(VT* v, int64_t N, const double* scal, cudaStream_t st);
template <typename VT>
void vec_random(VT* v, int64_t N, uint64_t seed, cudaStream_t st);
// out[:, i] = sum_a U[a + i*m] V[:, a] for i < nout (U column-major m x nout, FP64);
// when copy_col >= 0 also out[:, nout] = V[:, copy_col].  In place (out == V) is allowed.
template <typename VIN, typename VOUT>
void vec_combine(const VIN* V, int64_t N, int m, const double* U, int nout, VOUT* out, int64_t out_ld, int copy_col,
                 cudaStream_t st);
// complex combination: out[:, i] = sum_a Y[a + i*k] X[:, a] (Y complex column-major k x k), out != X
void vec_combine_complex(const double2* X, int64_t N, int k, const double2* Y, double2* out, cudaStream_t st);
template <typename VT>
void vec_copy_convert(const VT* src, double2* dst, int64_t n, cudaStream_t st);
template <typename VT>
void vec_convert_from(const double2* src, VT* dst, int64_t n, cudaStream_t st);
// r_i = ||W_i - theta_i X_i|| for i < k (columns of length N)
void vec_residual_norms(const double2* W, const double2* X, int64_t N, int k, const double* theta, double* out_norms,
                        cudaStream_t st);
int vec_grid(int64_t N);

}  // namespace momed
