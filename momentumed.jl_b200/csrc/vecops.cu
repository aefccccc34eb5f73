// Kernel (c): fused Lanczos vector operations (see vecops.cuh).
#include <algorithm>

#include "vecops.cuh"

namespace momed {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double2 cmul_conj(double2 a, double2 b) {   // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t seed, uint64_t idx) {
    return (double)(mix64(seed + (idx + 1) * 0x9E3779B97F4A7C15ULL) >> 11) * (1.0 / 9007199254740992.0);
}

// rows [r0, r1) handled by block b
__device__ __forceinline__ void block_rows(int64_t N, int64_t& r0, int64_t& r1) {
    int64_t per = (N + gridDim.x - 1) / gridDim.x;
    per = (per + kVecThreads - 1) / kVecThreads * kVecThreads;
    r0 = (int64_t)blockIdx.x * per;
    r1 = min(N, r0 + per);
}

// Grid: x = row blocks, y = groups of 8 columns; warp w of group g owns column 8g + w (one
// accumulator per lane, 8 loads of V in flight per warp); group 0 also sums |w|^2.
template <typename VT>
__global__ void __launch_bounds__(kVecThreads)
k_proj(const VT* __restrict__ V, int64_t N, int ncols, const VT* __restrict__ w, double2* partial,
       const int* active) {
    if (active && *active == 0) return;
    constexpr int TR = 2048;                     // rows of w staged per tile
    __shared__ double2 ws[TR];
    __shared__ double red[kVecThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int i = blockIdx.y * 8 + wid;
    double ax = 0.0, ay = 0.0, wn2 = 0.0;
    int64_t r0, r1;
    block_rows(N, r0, r1);
    const VT* colbase = V + (int64_t)(i < ncols ? i : 0) * N;
    for (int64_t t0 = r0; t0 < r1; t0 += TR) {
#pragma unroll
        for (int e = threadIdx.x; e < TR; e += kVecThreads) {
            int64_t n = t0 + e;
            double2 wv = (n < r1) ? to_d2(w[n]) : make_double2(0.0, 0.0);
            ws[e] = wv;
            wn2 += wv.x * wv.x + wv.y * wv.y;
        }
        __syncthreads();
        const int rows = (int)((r1 - t0) < (int64_t)TR ? (r1 - t0) : (int64_t)TR);
        if (i < ncols) {
            const VT* col = colbase + t0;
#pragma unroll 8
            for (int r = lane; r < rows; r += 32) {
                double2 p = cmul_conj(to_d2(col[r]), ws[r]);
                ax += p.x;
                ay += p.y;
            }
        }
        __syncthreads();
    }
    double2* out = partial + (int64_t)blockIdx.x * (kMaxCols + 1);
    ax = warp_sum(ax);
    ay = warp_sum(ay);
    if (i < ncols && lane == 0) out[i] = make_double2(ax, ay);
    if (blockIdx.y != 0) return;
    wn2 = warp_sum(wn2);
    if (lane == 0) red[wid] = wn2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kVecThreads / 32; ++q) s += red[q];
        out[ncols] = make_double2(s, 0.0);
    }
}

// One warp per column: lanes stride over the blocks' partials, then a fixed shuffle tree
// (deterministic order).
__global__ void k_reduce(const double2* partial, int grid, int ncols1, double2* out, const int* active) {
    if (active && *active == 0) return;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= ncols1) return;
    double sx = 0.0, sy = 0.0;
    for (int b = lane; b < grid; b += 32) {
        double2 v = partial[(int64_t)b * (kMaxCols + 1) + i];
        sx += v.x;
        sy += v.y;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (lane == 0) out[i] = make_double2(sx, sy);
}

template <typename VT>
__global__ void __launch_bounds__(kVecThreads)
k_update(const VT* __restrict__ V, int64_t N, int ncols, const double2* __restrict__ coef, VT* __restrict__ w,
         double2* partial, const int* active) {
    if (active && *active == 0) return;
    __shared__ double2 c[kMaxCols];
    __shared__ double red[kVecThreads / 32];
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) c[i] = coef[i];
    __syncthreads();
    int64_t r0, r1;
    block_rows(N, r0, r1);
    double wn2 = 0.0;
    for (int64_t n = r0 + threadIdx.x; n < r1; n += kVecThreads) {
        double2 acc = to_d2(w[n]);
#pragma unroll 8
        for (int i = 0; i < ncols; ++i) {
            double2 p = cmul(c[i], to_d2(V[(int64_t)i * N + n]));
            acc.x -= p.x;
            acc.y -= p.y;
        }
        VT st = from_d2<VT>(acc);
        w[n] = st;
        double2 back = to_d2(st);
        wn2 += back.x * back.x + back.y * back.y;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    wn2 = warp_sum(wn2);
    if (lane == 0) red[wid] = wn2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kVecThreads / 32; ++q) s += red[q];
        partial[(int64_t)blockIdx.x * (kMaxCols + 1)] = make_double2(s, 0.0);
    }
}

// Warp-wide sum of the per-block norm partials (call with all 32 lanes).
__device__ double sum_norm_partials(const double2* partial, int grid) {
    double s = 0.0;
    for (int b = threadIdx.x & 31; b < grid; b += 32) s += partial[(int64_t)b * (kMaxCols + 1)].x;
    return warp_sum(s);
}

__global__ void k_decide(const double2* coefA, int ncols, const double2* partial, int grid, int* flag,
                         double* scal) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    double after = sum_norm_partials(partial, grid);
    if (threadIdx.x != 0) return;
    double before = coefA[ncols].x;
    scal[1] = after;
    // second pass when the first removed more than 1 - 0.1 of the squared norm (|w'| < 0.32 |w|);
    // the classical 1/2 flags nearly every Lanczos step (w = H v carries alpha and beta along the
    // two newest columns) without changing the eigenpairs
    *flag = (after < 0.1 * before) ? 1 : 0;
}

__global__ void k_finalize(const double2* coefA, const double2* coefB, int ncols, const double2* partial2, int grid,
                           const int* flag, double* scal, double* alpha, double* beta, int j) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const bool second = *flag != 0;
    double s2 = second ? sum_norm_partials(partial2, grid) : 0.0;   // warp-uniform branch
    if (threadIdx.x != 0) return;
    double a = coefA[ncols - 1].x + (second ? coefB[ncols - 1].x : 0.0);
    double wn2 = second ? s2 : scal[1];
    double b = sqrt(max(wn2, 0.0));
    alpha[j] = a;
    beta[j] = b;
    scal[0] = b > 0.0 ? 1.0 / b : 0.0;
}

template <typename VT>
__global__ void k_scale(VT* v, int64_t N, const double* scal) {
    const double s = *scal;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        double2 x = to_d2(v[n]);
        v[n] = from_d2<VT>(make_double2(x.x * s, x.y * s));
    }
}

template <typename VT>
__global__ void k_random(VT* v, int64_t N, uint64_t seed) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
        v[n] = from_d2<VT>(make_double2(u01(seed, 2 * (uint64_t)n), u01(seed, 2 * (uint64_t)n + 1)));
}

// Tile of TR rows of all m (+1) columns staged in shared memory, then every
// (row, output) pair is a length-m dot product from shared memory.
template <typename VIN, typename VOUT, int TR>
__global__ void __launch_bounds__(kVecThreads)
k_combine(const VIN* V, int64_t N, int m, const double* __restrict__ U, int nout, VOUT* out, int64_t out_ld,
          int copy_col) {
    extern __shared__ double2 tile[];   // [(m + 1) * TR]
    const int ncopy = copy_col >= 0 ? 1 : 0;
    for (int64_t t0 = (int64_t)blockIdx.x * TR; t0 < N; t0 += (int64_t)gridDim.x * TR) {
        const int rows = (int)((N - t0) < (int64_t)TR ? (N - t0) : (int64_t)TR);
#pragma unroll 4
        for (int e = threadIdx.x; e < (m + ncopy) * TR; e += blockDim.x) {
            int a = e / TR, r = e % TR;
            int col = (a < m) ? a : copy_col;
            tile[e] = (r < rows) ? to_d2(V[(int64_t)col * N + t0 + r]) : make_double2(0.0, 0.0);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nout * TR; e += blockDim.x) {
            int i = e / TR, r = e % TR;
            if (r < rows) {
                double sx = 0.0, sy = 0.0;
                const double* u = U + (int64_t)i * m;
                for (int a = 0; a < m; ++a) {
                    double2 v = tile[a * TR + r];
                    double c = __ldg(u + a);
                    sx += c * v.x;
                    sy += c * v.y;
                }
                out[(int64_t)i * out_ld + t0 + r] = from_d2<VOUT>(make_double2(sx, sy));
            }
        }
        if (ncopy) {
            for (int r = threadIdx.x; r < rows; r += blockDim.x)
                out[(int64_t)nout * out_ld + t0 + r] = from_d2<VOUT>(tile[m * TR + r]);
        }
        __syncthreads();
    }
}

__global__ void k_combine_complex(const double2* __restrict__ X, int64_t N, int k, const double2* __restrict__ Y,
                                  double2* __restrict__ out) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        for (int i = 0; i < k; ++i) {
            double sx = 0.0, sy = 0.0;
            for (int a = 0; a < k; ++a) {
                double2 y = Y[(int64_t)i * k + a];
                double2 x = X[(int64_t)a * N + n];
                sx += y.x * x.x - y.y * x.y;
                sy += y.x * x.y + y.y * x.x;
            }
            out[(int64_t)i * N + n] = make_double2(sx, sy);
        }
    }
}

template <typename VT>
__global__ void k_to_d2(const VT* src, double2* dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = to_d2(src[i]);
}
template <typename VT>
__global__ void k_from_d2(const double2* src, VT* dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = from_d2<VT>(src[i]);
}

__global__ void k_residual(const double2* W, const double2* X, int64_t N, int k, const double* theta,
                           double* partial /* [grid][k] */) {
    __shared__ double red[kVecThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = 0; i < k; ++i) {
        double th = theta[i], s = 0.0;
        for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
            double2 w = W[(int64_t)i * N + n], x = X[(int64_t)i * N + n];
            double rx = w.x - th * x.x, ry = w.y - th * x.y;
            s += rx * rx + ry * ry;
        }
        s = warp_sum(s);
        if (lane == 0) red[wid] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int q = 0; q < kVecThreads / 32; ++q) t += red[q];
            partial[(int64_t)blockIdx.x * k + i] = t;
        }
        __syncthreads();
    }
}

int sm_count() {
    static const int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    return sms;
}

int flat_grid(int64_t n) {
    int64_t b = (n + kVecThreads - 1) / kVecThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * 8));
}

}  // namespace

int vec_grid(int64_t N) {
    int64_t b = (N + kVecThreads - 1) / kVecThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * 4));
}

template <typename VT>
void vec_proj(const VT* V, int64_t N, int ncols, const VT* w, double2* partial, int grid, const int* active,
              cudaStream_t st) {
    MOMED_REQUIRE(ncols <= kMaxCols, MOMED_EINVAL, "krylovdim too large");
    k_proj<VT><<<dim3(grid, (unsigned)std::max(1, (ncols + 7) / 8)), kVecThreads, 0, st>>>(V, N, ncols, w, partial,
                                                                                            active);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
void vec_reduce(const double2* partial, int grid, int ncols1, double2* out, const int* active, cudaStream_t st) {
    k_reduce<<<(ncols1 + 7) / 8, 256, 0, st>>>(partial, grid, ncols1, out, active);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VT>
void vec_update(const VT* V, int64_t N, int ncols, const double2* coef, VT* w, double2* partial, int grid,
                const int* active, cudaStream_t st) {
    k_update<VT><<<grid, kVecThreads, 0, st>>>(V, N, ncols, coef, w, partial, active);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
void vec_decide(const double2* coefA, int ncols, const double2* partial, int grid, int* flag, double* scal,
                cudaStream_t st) {
    k_decide<<<1, 32, 0, st>>>(coefA, ncols, partial, grid, flag, scal);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
void vec_finalize(const double2* coefA, const double2* coefB, int ncols, const double2* partial2, int grid,
                  const int* flag, double* scal, double* alpha, double* beta, int j, cudaStream_t st) {
    k_finalize<<<1, 32, 0, st>>>(coefA, coefB, ncols, partial2, grid, flag, scal, alpha, beta, j);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VT>
void vec_scale(VT* v, int64_t N, const double* scal, cudaStream_t st) {
    k_scale<VT><<<flat_grid(N), kVecThreads, 0, st>>>(v, N, scal);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VT>
void vec_random(VT* v, int64_t N, uint64_t seed, cudaStream_t st) {
    k_random<VT><<<flat_grid(N), kVecThreads, 0, st>>>(v, N, seed);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VIN, typename VOUT>
void vec_combine(const VIN* V, int64_t N, int m, const double* U, int nout, VOUT* out, int64_t out_ld, int copy_col,
                 cudaStream_t st) {
    // The shared-memory limit is a process-wide attribute of the kernel: it is always set to the
    // largest tile the kernel can get, so callers on other threads never lower it under a launch.
    const int ncopy = copy_col >= 0 ? 1 : 0;
    MOMED_REQUIRE(m + ncopy <= kMaxCols + 1, MOMED_EINVAL, "krylovdim too large");
    if (m + ncopy <= 100) {
        constexpr int TR = 64;
        size_t smem = (size_t)(m + ncopy) * TR * sizeof(double2);
        auto k = k_combine<VIN, VOUT, TR>;
        MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(100 * TR * sizeof(double2))));
        int grid = (int)std::max<int64_t>(1, std::min<int64_t>((N + TR - 1) / TR, (int64_t)sm_count() * 2));
        k<<<grid, kVecThreads, smem, st>>>(V, N, m, U, nout, out, out_ld, copy_col);
    } else {
        constexpr int TR = 32;
        size_t smem = (size_t)(m + ncopy) * TR * sizeof(double2);
        auto k = k_combine<VIN, VOUT, TR>;
        MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)((kMaxCols + 1) * TR * sizeof(double2))));
        int grid = (int)std::max<int64_t>(1, std::min<int64_t>((N + TR - 1) / TR, (int64_t)sm_count() * 2));
        k<<<grid, kVecThreads, smem, st>>>(V, N, m, U, nout, out, out_ld, copy_col);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
void vec_combine_complex(const double2* X, int64_t N, int k, const double2* Y, double2* out, cudaStream_t st) {
    k_combine_complex<<<flat_grid(N), kVecThreads, 0, st>>>(X, N, k, Y, out);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VT>
void vec_copy_convert(const VT* src, double2* dst, int64_t n, cudaStream_t st) {
    k_to_d2<VT><<<flat_grid(n), kVecThreads, 0, st>>>(src, dst, n);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
template <typename VT>
void vec_convert_from(const double2* src, VT* dst, int64_t n, cudaStream_t st) {
    k_from_d2<VT><<<flat_grid(n), kVecThreads, 0, st>>>(src, dst, n);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}
void vec_residual_norms(const double2* W, const double2* X, int64_t N, int k, const double* theta, double* out_norms,
                        cudaStream_t st) {
    int grid = std::min(vec_grid(N), 512);
    DevBuf<double> part, th;
    part.resize((size_t)grid * k);
    th.resize(k);
    MOMED_CUDA_TRY(cudaMemcpyAsync(th.p, theta, k * sizeof(double), cudaMemcpyHostToDevice, st));
    k_residual<<<grid, kVecThreads, 0, st>>>(W, X, N, k, th.p, part.p);
    MOMED_CUDA_TRY(cudaGetLastError());
    std::vector<double> h((size_t)grid * k);
    MOMED_CUDA_TRY(cudaMemcpyAsync(h.data(), part.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < k; ++i) {
        double s = 0.0;
        for (int b = 0; b < grid; ++b) s += h[(size_t)b * k + i];
        out_norms[i] = std::sqrt(s);
    }
}

// explicit instantiations
template void vec_proj<double2>(const double2*, int64_t, int, const double2*, double2*, int, const int*, cudaStream_t);
template void vec_proj<float2>(const float2*, int64_t, int, const float2*, double2*, int, const int*, cudaStream_t);
template void vec_update<double2>(const double2*, int64_t, int, const double2*, double2*, double2*, int, const int*,
                                  cudaStream_t);
template void vec_update<float2>(const float2*, int64_t, int, const double2*, float2*, double2*, int, const int*,
                                 cudaStream_t);
template void vec_scale<double2>(double2*, int64_t, const double*, cudaStream_t);
template void vec_scale<float2>(float2*, int64_t, const double*, cudaStream_t);
template void vec_random<double2>(double2*, int64_t, uint64_t, cudaStream_t);
template void vec_random<float2>(float2*, int64_t, uint64_t, cudaStream_t);
template void vec_combine<double2, double2>(const double2*, int64_t, int, const double*, int, double2*, int64_t, int,
                                            cudaStream_t);
template void vec_combine<float2, float2>(const float2*, int64_t, int, const double*, int, float2*, int64_t, int,
                                          cudaStream_t);
template void vec_combine<float2, double2>(const float2*, int64_t, int, const double*, int, double2*, int64_t, int,
                                           cudaStream_t);
template void vec_copy_convert<float2>(const float2*, double2*, int64_t, cudaStream_t);
template void vec_copy_convert<double2>(const double2*, double2*, int64_t, cudaStream_t);
template void vec_convert_from<float2>(const double2*, float2*, int64_t, cudaStream_t);
template void vec_convert_from<double2>(const double2*, double2*, int64_t, cudaStream_t);

}  // namespace momed
