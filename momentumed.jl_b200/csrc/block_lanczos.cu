// Block thick-restart Lanczos for ONE operator and several wanted eigenpairs.
//
// The single-vector solver (lanczos.cu) multiplies one Krylov vector per map launch; the map
// then gathers one x value per (row, term) hit from a random 16-byte location and is bound by
// L1 wavefronts, not HBM.  Here every launch multiplies a block of B vectors stored
// interleaved ([row][B]), so each hit reads B contiguous values: the same block map that the
// batched solver uses for its B parameter values, with one parameter.  This is the block
// Krylov method that KrylovKit's Lanczos (krylov_map_solve, MomentumEDCUDAExt.jl:159-179)
// does with block size 1, restarted the same way (Krylov-Schur: keep the leading Ritz
// vectors, reduce the projected matrix to an arrow; basistransform!, 210-244).
//
// One block step j (basis blocks Q_0..Q_j, each N x B):
//   W = H Q_j                                   block map (B right-hand sides)
//   C = Q^H W,  W -= Q C      (twice)           k_bl_proj + k_bl_reduce, k_bl_update
//   W = Q_{j+1} R   (Cholesky QR, twice)        Gram W^H W with k_bl_proj, k_bl_chol, k_bl_rmul
// The projected matrix is block tridiagonal and Hermitian: diagonal blocks A_j = Q_j^H H Q_j
// (the projections on block j), sub-diagonal blocks R_j.  Reorthogonalisation coefficients,
// Gram matrices and every reduction accumulate in FP64.  A step runs on the device without a
// host round trip (the B x B Cholesky factors included); the host reads the factors once per
// restart cycle and solves the m x m projected eigenproblem in FP64.
//
// Precision forms (the same contract as the single-vector solver):
//   FP64  - c128 block map and basis.
//   MIXED - c64 block map (FP32 accumulate) and c64 basis with FP64 reductions, run to the
//           FP32 floor; then FP64 Rayleigh-Ritz on the Ritz vectors, and if that misses the
//           target, FP64 block Lanczos warm-started from the refined vectors.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "vecops.cuh"

namespace momed {

void ensure_ready(momed_handle* h);
void rayleigh_ritz_fp64(momed_handle* h, double2* X, double2* W, double2* scratch, int k, std::vector<double>& theta,
                        std::vector<double>& resid, int64_t& matvecs);

namespace {

using cd = std::complex<double>;
constexpr int kBT = 256;           // threads per block of the block-vector kernels
constexpr int kProjRows = 64;      // rows of W staged per tile in k_bl_proj
constexpr int kMaxBlkCols = 256;   // basis columns one projection covers (m <= 256)
constexpr int kMaxCoef = 2048;     // m * B coefficients one update holds in shared memory

// row phases of a projection over ncol columns: all 256 threads busy for wide bases, at most 16
// for the Gram matrix of one block (fewer partial sums to reduce)
__host__ __device__ inline int proj_phases(int ncol) {
    const int p = kBT / ncol;
    return p < 16 ? p : 16;
}

template <typename VT> struct Real;
template <> struct Real<float2> { using T = float; };
template <> struct Real<double2> { using T = double; };

__device__ __forceinline__ double2 ld2(const float2* p) { float2 v = *p; return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 ld2(const double2* p) { return *p; }
__device__ __forceinline__ void st2(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ void st2(double2* p, double2 v) { *p = v; }

// Projection of the block W [N][B] on ncol basis columns: column c is entry c % B of block
// c / B (blocks blk_stride elements apart).  Thread (c, p) accumulates conj(Q_c[n]) W[n][r] for
// all r over the rows n = p, p + P, ... of each staged tile, in FP64; each (CTA, p) writes
// its partial sums partial[(cta * P + p)][c][r].
template <typename VT, int B>
__global__ void __launch_bounds__(kBT)
k_bl_proj(const VT* __restrict__ Q, int64_t blk_stride, int ncol, int64_t N, const VT* __restrict__ W,
          double2* __restrict__ partial) {
    __shared__ double2 wt[kProjRows * B];
    const int P = proj_phases(ncol);                // row phases (ncol <= kBT)
    const int t = threadIdx.x;
    const int c = t % ncol, p = t / ncol;
    const bool active = p < P;
    const VT* qc = Q + (size_t)(c / B) * blk_stride + (c % B);
    double are[B], aim[B];
#pragma unroll
    for (int r = 0; r < B; ++r) { are[r] = 0.0; aim[r] = 0.0; }
    const int64_t tiles = (N + kProjRows - 1) / kProjRows;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t n0 = tile * kProjRows;
        const int rows = (int)(N - n0 < kProjRows ? N - n0 : kProjRows);
        __syncthreads();
        for (int e = t; e < rows * B; e += kBT) wt[e] = ld2(W + n0 * B + e);
        __syncthreads();
        if (active) {
#pragma unroll 4
            for (int i = p; i < rows; i += P) {
                const double2 q = ld2(qc + (n0 + i) * B);
#pragma unroll
                for (int r = 0; r < B; ++r) {
                    const double2 w = wt[i * B + r];
                    are[r] = fma(q.x, w.x, fma(q.y, w.y, are[r]));
                    aim[r] = fma(q.x, w.y, fma(-q.y, w.x, aim[r]));
                }
            }
        }
    }
    if (active) {
        double2* out = partial + ((size_t)blockIdx.x * P + p) * ncol * B + (size_t)c * B;
#pragma unroll
        for (int r = 0; r < B; ++r) out[r] = make_double2(are[r], aim[r]);
    }
}

// out[e] = sum over g < nparts of partial[g][e]: one CTA per output, the threads take parts in
// a fixed stride and a fixed tree combines them (deterministic; thousands of parts per output
// for the Gram matrices of one block)
__global__ void __launch_bounds__(256) k_bl_reduce(const double2* __restrict__ partial, int nparts, int count,
                                                   double2* __restrict__ out) {
    __shared__ double sx[256], sy[256];
    const int e = blockIdx.x, t = threadIdx.x;
    double ax = 0.0, ay = 0.0;
    for (int g = t; g < nparts; g += 256) {
        const double2 v = partial[(size_t)g * count + e];
        ax += v.x;
        ay += v.y;
    }
    sx[t] = ax;
    sy[t] = ay;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (t < o) {
            sx[t] += sx[t + o];
            sy[t] += sy[t + o];
        }
        __syncthreads();
    }
    if (t == 0) out[e] = make_double2(sx[0], sy[0]);
}

// W[n][r] -= sum_c Q_c[n] C[c][r]  (c < ncol; C [ncol][B] FP64, staged in shared memory as ACC)
template <typename VT, typename ACC, int B>
__global__ void __launch_bounds__(kBT)
k_bl_update(const VT* __restrict__ Q, int64_t blk_stride, int ncol, int64_t N, const double2* __restrict__ C,
            VT* __restrict__ W) {
    extern __shared__ unsigned char smem_raw[];
    ACC* cs = reinterpret_cast<ACC*>(smem_raw);     // [ncol * B] complex as (re, im) pairs
    for (int e = threadIdx.x; e < ncol * B; e += blockDim.x) {
        cs[2 * e] = (ACC)C[e].x;
        cs[2 * e + 1] = (ACC)C[e].y;
    }
    __syncthreads();
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        ACC are[B], aim[B];
#pragma unroll
        for (int r = 0; r < B; ++r) {
            const double2 w = ld2(W + n * B + r);
            are[r] = (ACC)w.x;
            aim[r] = (ACC)w.y;
        }
        for (int c = 0; c < ncol; ++c) {
            const double2 q = ld2(Q + (size_t)(c / B) * blk_stride + n * B + (c % B));
            const ACC qx = (ACC)q.x, qy = (ACC)q.y;
            const ACC* cc = cs + 2 * c * B;
#pragma unroll
            for (int r = 0; r < B; ++r) {
                const ACC cx = cc[2 * r], cy = cc[2 * r + 1];
                are[r] -= qx * cx - qy * cy;
                aim[r] -= qx * cy + qy * cx;
            }
        }
#pragma unroll
        for (int r = 0; r < B; ++r) st2(W + n * B + r, make_double2((double)are[r], (double)aim[r]));
    }
}

// W[n][:] <- W[n][:] M   (M [B][B] complex FP64, row a column r), in place: thread (n, r)
// reads row n, the warp (which holds whole rows: B divides 32) synchronises, then writes.
template <typename VT, int B>
__global__ void __launch_bounds__(kBT) k_bl_rmul(VT* __restrict__ W, int64_t N, const double2* __restrict__ M) {
    __shared__ double2 ms[B * B];
    for (int e = threadIdx.x; e < B * B; e += blockDim.x) ms[e] = M[e];
    __syncthreads();
    const int r = threadIdx.x % B;
    const int64_t total = N * B;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x; e0 < total; e0 += stride) {
        const int64_t e = e0 + threadIdx.x;          // every thread of the warp takes part in __syncwarp
        const bool in = e < total;
        const int64_t n = e / B;
        double sx = 0.0, sy = 0.0;
        if (in) {
            for (int a = 0; a < B; ++a) {
                const double2 w = ld2(W + n * B + a);
                const double2 m = ms[a * B + r];
                sx = fma(w.x, m.x, fma(-w.y, m.y, sx));
                sy = fma(w.x, m.y, fma(w.y, m.x, sy));
            }
        }
        __syncwarp();
        if (in) st2(W + e, make_double2(sx, sy));
    }
}

// Ritz vectors: out_i = sum_c Q_c Y[c][i] for the B outputs i = blockIdx.y * B + r (r < B,
// i < nout); Y [ncol][nout] complex FP64.  BLOCKED: out block blockIdx.y ([N][B], VOUT = VT,
// blocks out_stride apart); else out[i][N] (VOUT = double2).  FP64 accumulation.
template <typename VT, typename VOUT, int B, bool BLOCKED>
__global__ void __launch_bounds__(kBT)
k_bl_combine(const VT* __restrict__ Q, int64_t blk_stride, int ncol, int64_t N, const double2* __restrict__ Y,
             int nout, VOUT* __restrict__ out, int64_t out_stride) {
    extern __shared__ unsigned char smem_raw[];
    double2* ys = reinterpret_cast<double2*>(smem_raw);   // [ncol][B] of this output group
    const int i0 = blockIdx.y * B;
    for (int e = threadIdx.x; e < ncol * B; e += blockDim.x) {
        const int c = e / B, r = e % B;
        ys[e] = (i0 + r < nout) ? Y[(size_t)c * nout + i0 + r] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        double are[B], aim[B];
#pragma unroll
        for (int r = 0; r < B; ++r) { are[r] = 0.0; aim[r] = 0.0; }
        for (int c = 0; c < ncol; ++c) {
            const double2 q = ld2(Q + (size_t)(c / B) * blk_stride + n * B + (c % B));
            const double2* yc = ys + c * B;
#pragma unroll
            for (int r = 0; r < B; ++r) {
                const double2 y = yc[r];
                are[r] = fma(q.x, y.x, fma(-q.y, y.y, are[r]));
                aim[r] = fma(q.x, y.y, fma(q.y, y.x, aim[r]));
            }
        }
        if (BLOCKED) {
#pragma unroll
            for (int r = 0; r < B; ++r)
                st2(reinterpret_cast<VT*>(out) + (size_t)blockIdx.y * out_stride + n * B + r,
                    make_double2(are[r], aim[r]));
        } else {
#pragma unroll
            for (int r = 0; r < B; ++r)
                if (i0 + r < nout)
                    reinterpret_cast<double2*>(out)[(size_t)(i0 + r) * N + n] = make_double2(are[r], aim[r]);
        }
    }
}

// block [N][B] from columns [k][N] c128: dst[n][r] = src[r][n] for r < k, untouched beyond
template <typename VT, int B>
__global__ void k_bl_from_cols(const double2* __restrict__ src, int k, int64_t N, VT* __restrict__ dst) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N * B; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % B);
        if (r < k) st2(dst + e, src[(size_t)r * N + e / B]);
    }
}

// One Cholesky QR pass on the device (one warp; B <= 16): G = R^H R for the Gram matrix
// G[a][r] = w_a^H w_r, Rinv = R^-1 (applied by k_bl_rmul), and the accumulated factor
// Racc <- R (pass 0) or R Racc (pass 1), so that W_in = W_out Racc.  Sets *flag when the block
// lost rank: a pivot below rel * max diag(G), or (gpre given) a column whose squared norm fell
// below lost * its norm before the Gram-Schmidt passes.
template <int B>
__global__ void k_bl_chol(const double2* __restrict__ G, const double2* __restrict__ gpre, double rel, double lost,
                          int pass, double2* __restrict__ Rinv, double2* __restrict__ Racc, int* __restrict__ flag) {
    __shared__ double2 R[B * B], X[B * B], P[B * B];
    __shared__ int bad;
    const int l = threadIdx.x;                      // one warp; lanes >= B idle in the column loops
    for (int e = l; e < B * B; e += 32) { R[e] = make_double2(0.0, 0.0); X[e] = make_double2(0.0, 0.0); }
    if (l == 0) {
        double tr = 0.0;
        for (int i = 0; i < B; ++i) tr = fmax(tr, G[i * B + i].x);
        bad = !(tr > 0.0);
        if (gpre)
            for (int i = 0; i < B; ++i)
                if (!(G[i * B + i].x > lost * gpre[i * B + i].x)) bad = 1;
    }
    __syncwarp();
    double tr = 0.0;
    for (int i = 0; i < B; ++i) tr = fmax(tr, G[i * B + i].x);
    for (int j = 0; j < B && !bad; ++j) {
        if (l == 0) {
            double d = G[j * B + j].x;
            for (int p = 0; p < j; ++p) d -= R[p * B + j].x * R[p * B + j].x + R[p * B + j].y * R[p * B + j].y;
            if (!(d > rel * tr)) bad = 1;
            else R[j * B + j] = make_double2(sqrt(d), 0.0);
        }
        __syncwarp();
        if (bad) break;
        if (l > j && l < B) {
            double vx = G[j * B + l].x, vy = G[j * B + l].y;      // minus sum_p conj(R[p][j]) R[p][l]
            for (int p = 0; p < j; ++p) {
                const double2 a = R[p * B + j], b = R[p * B + l];
                vx -= a.x * b.x + a.y * b.y;
                vy -= a.x * b.y - a.y * b.x;
            }
            const double inv = 1.0 / R[j * B + j].x;
            R[j * B + l] = make_double2(vx * inv, vy * inv);
        }
        __syncwarp();
    }
    if (bad) {
        if (l == 0) *flag = 1;
        for (int e = l; e < B * B; e += 32) Rinv[e] = make_double2((e / B == e % B) ? 1.0 : 0.0, 0.0);
        return;
    }
    if (l < B) {                                    // column l of X = R^-1 by back substitution
        const int c = l;
        X[c * B + c] = make_double2(1.0 / R[c * B + c].x, 0.0);
        for (int r = c - 1; r >= 0; --r) {
            double sx = 0.0, sy = 0.0;
            for (int p = r + 1; p <= c; ++p) {
                const double2 a = R[r * B + p], b = X[p * B + c];
                sx += a.x * b.x - a.y * b.y;
                sy += a.x * b.y + a.y * b.x;
            }
            const double inv = 1.0 / R[r * B + r].x;
            X[r * B + c] = make_double2(-sx * inv, -sy * inv);
        }
    }
    __syncwarp();
    for (int e = l; e < B * B; e += 32) Rinv[e] = X[e];
    if (pass == 0) {
        for (int e = l; e < B * B; e += 32) Racc[e] = R[e];
        return;
    }
    if (l < B) {                                    // column l of R Racc
        for (int a = 0; a < B; ++a) {
            double sx = 0.0, sy = 0.0;
            for (int p = a; p < B; ++p) {
                const double2 x = R[a * B + p], y = Racc[p * B + l];
                sx += x.x * y.x - x.y * y.y;
                sy += x.x * y.y + x.y * y.x;
            }
            P[a * B + l] = make_double2(sx, sy);
        }
    }
    __syncwarp();
    for (int e = l; e < B * B; e += 32) Racc[e] = P[e];
}

// A = C1 + C2 (the projections of both Gram-Schmidt passes on the newest block)
__global__ void k_bl_add(const double2* __restrict__ a, const double2* __restrict__ b, int count,
                         double2* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < count) out[e] = make_double2(a[e].x + b[e].x, a[e].y + b[e].y);
}

int blk_sms() {
    static const int s = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    return s;
}

// Breakdown of the block recurrence (a block lost rank): the caller falls back to the
// single-vector solver.
struct Breakdown {};

template <typename VT, int B>
struct BlockKrylov {
    using RT = typename Real<VT>::T;
    static constexpr bool kF32 = std::is_same<VT, float2>::value;
    momed_handle* h;
    int64_t N;
    int mb;          // basis blocks of a full cycle
    int m;           // mb * B columns
    cudaStream_t st;
    int pgrid;       // CTAs of one projection
    DevBuf<VT> Q, Q2;
    DevBuf<double2> partial, C1, C2, Gd, Gpre, Rinv, Astore, Rstore, Yd;
    DevBuf<RT> ud;
    DevBuf<int> flag, tcerr;
    int64_t matvecs = 0;
    bool tc = false;          // basis projections on the tensor cores (FP32 basis, B = 8 or 16)
    bool tc_check = false;    // diagnostics: also run the CUDA-core projection and compare
    double tc_maxdiff = 0.0;

    BlockKrylov(momed_handle* hh, int blocks) : h(hh), N(hh->n), mb(blocks), m(blocks * B), st(hh->stream) {
        const int64_t tiles = (N + kProjRows - 1) / kProjRows;
        pgrid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)blk_sms() * 2));
        Q.resize((size_t)(mb + 1) * N * B);
        partial.resize((size_t)pgrid * kBT * B);
        C1.resize((size_t)kMaxBlkCols * B);
        C2.resize((size_t)kMaxBlkCols * B);
        Gd.resize((size_t)B * B);
        Gpre.resize((size_t)B * B);
        Rinv.resize((size_t)B * B);
        Astore.resize((size_t)(mb + 1) * B * B);
        Rstore.resize((size_t)(mb + 1) * B * B);
        flag.resize(1);
        tcerr.resize(1);
        MOMED_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        MOMED_CUDA_TRY(cudaMemsetAsync(tcerr.p, 0, sizeof(int), st));
        if constexpr (kF32 && (B == 8 || B == 16)) {
            const char* e = std::getenv("MOMED_TC_PROJ");
            tc = !(e && e[0] == '0');
            const char* c = std::getenv("MOMED_TC_CHECK");
            tc_check = tc && c && c[0] == '1';
        }
        ud.resize(B);
        std::vector<RT> uh(B, (RT)(h->op.has_b ? h->u : 0.0));
        MOMED_CUDA_TRY(cudaMemcpyAsync(ud.p, uh.data(), B * sizeof(RT), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    VT* blk(int i) { return Q.p + (size_t)i * N * B; }
    int ugrid() const { return (int)std::max<int64_t>(1, std::min<int64_t>((N + kBT - 1) / kBT, (int64_t)blk_sms() * 8)); }
    int rgrid() const { return (int)std::max<int64_t>(1, std::min<int64_t>((N * B + kBT - 1) / kBT, (int64_t)blk_sms() * 8)); }

    void map(const VT* x, VT* y) {
        prof_begin(h);
        if constexpr (kF32) {
            const float* u = h->op.has_b ? reinterpret_cast<const float*>(ud.p) : nullptr;
            if (h->sparse.built) {
                launch_block_spmv_c64(h->sparse, reinterpret_cast<const float2*>(x), reinterpret_cast<float2*>(y), u,
                                      B, N, st);
                prof_end(h, MOMED_KERNEL_BLOCK_SPMV_C64);
            } else if (h->hcache.full()) {
                launch_block_hc_c64(h, reinterpret_cast<const float2*>(x), reinterpret_cast<float2*>(y), u, B, N, st);
                prof_end(h, MOMED_KERNEL_HC_BLOCK_C64);
            } else {
                launch_block_matvec_c64(index_view(h), h->op.view(), reinterpret_cast<const float2*>(x),
                                        reinterpret_cast<float2*>(y), u, B, N, st);
                prof_end(h, MOMED_KERNEL_BLOCK_MATVEC_C64);
            }
        } else {
            const double* u = h->op.has_b ? reinterpret_cast<const double*>(ud.p) : nullptr;
            if (h->hcache.full()) {
                launch_block_hc_c128(h, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), u, B, N,
                                     st);
                prof_end(h, MOMED_KERNEL_HC_BLOCK_C128);
            } else {
                launch_block_matvec_c128(index_view(h), h->op.view(), reinterpret_cast<const double2*>(x),
                                         reinterpret_cast<double2*>(y), u, B, N, st);
                prof_end(h, MOMED_KERNEL_BLOCK_MATVEC_C128);
            }
        }
        matvecs += B;
    }
    // out[c][r] = basis^H W over ncol columns starting at `base` (blocks N*B apart); the basis
    // projections of an FP32 basis run on the tensor cores (the Gram matrices of one block on
    // the CUDA cores)
    void proj(const VT* base, int ncol, const VT* W, double2* out) {
        if constexpr (kF32) {
            if (tc && ncol > B) {
                int ns = 0;
                launch_proj_tc_c64(reinterpret_cast<const float2*>(base), ncol, N, reinterpret_cast<const float2*>(W),
                                   B, partial.p, pgrid * kBT / 64, &ns, tcerr.p, st);
                const int count = ncol * B;
                k_bl_reduce<<<count, 256, 0, st>>>(partial.p, ns, count, out);
                MOMED_CUDA_TRY(cudaGetLastError());
                note_launches(1);
                if (tc_check) check_tc(base, ncol, W, out);
                return;
            }
        }
        proj_cuda(base, ncol, W, out);
    }
    // the same projection on the CUDA cores, compared with the tensor-core result `out`
    void check_tc(const VT* base, int ncol, const VT* W, const double2* out) {
        DevBuf<double2> ref;
        ref.resize((size_t)ncol * B);
        proj_cuda(base, ncol, W, ref.p);
        std::vector<double2> a((size_t)ncol * B), b((size_t)ncol * B);
        MOMED_CUDA_TRY(cudaMemcpyAsync(a.data(), out, a.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(b.data(), ref.p, b.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        double mx = 0.0, d = 0.0;
        for (size_t i = 0; i < a.size(); ++i) {
            mx = std::max(mx, std::hypot(b[i].x, b[i].y));
            d = std::max(d, std::hypot(a[i].x - b[i].x, a[i].y - b[i].y));
        }
        // scale: the largest coefficient or the largest column norm of W (|q^H w| <= |w|), so that
        // the tiny coefficients of a second Gram-Schmidt pass are compared with |w|
        proj_cuda(W, B, W, ref.p);
        std::vector<double2> g((size_t)B * B);
        MOMED_CUDA_TRY(cudaMemcpyAsync(g.data(), ref.p, g.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        for (int r = 0; r < B; ++r) mx = std::max(mx, std::sqrt(std::max(g[(size_t)r * B + r].x, 0.0)));
        // split-TF32 products carry ~2^-21 and the tensor-memory sums over 256 rows are FP32:
        // a few 1e-6 relative to the largest coefficient (H-scaled vectors reach |C| ~ |H|)
        const double rel = d / std::max(mx, 1e-30);
        tc_maxdiff = std::max(tc_maxdiff, d);
        if (!(rel <= 1e-5))
            throw Error{MOMED_ECUDA, "tensor-core projection differs from the CUDA-core projection: max |diff| " +
                                         std::to_string(d) + " (relative " + std::to_string(rel) + ")"};
    }
    void proj_cuda(const VT* base, int ncol, const VT* W, double2* out) {
        k_bl_proj<VT, B><<<pgrid, kBT, 0, st>>>(base, N * B, ncol, N, W, partial.p);
        const int P = proj_phases(ncol);
        const int count = ncol * B;
        k_bl_reduce<<<count, 256, 0, st>>>(partial.p, pgrid * P, count, out);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(2);
    }
    void update(int ncol, const double2* C, VT* W) {
        using ACC = typename std::conditional<kF32, float, double>::type;
        const size_t smem = (size_t)ncol * B * 2 * sizeof(ACC);
        auto k = k_bl_update<VT, ACC, B>;
        constexpr size_t smem_max = (size_t)kMaxCoef * 2 * sizeof(ACC);
        if (smem_max > 48 * 1024)
            MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
        k<<<ugrid(), kBT, smem, st>>>(Q.p, N * B, ncol, N, C, W);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(1);
    }
    // one Cholesky QR pass of W: Gram, factor on the device, W <- W R^-1; R accumulates in Racc
    void cholqr_pass(VT* W, int pass, const double2* gpre, double2* Racc) {
        proj(W, B, W, Gd.p);
        k_bl_chol<B><<<1, 32, 0, st>>>(Gd.p, gpre, pass == 0 ? 1e-24 : 1e-12, kF32 ? 1e-10 : 1e-24, pass, Rinv.p,
                                       Racc, flag.p);
        k_bl_rmul<VT, B><<<rgrid(), kBT, 0, st>>>(W, N, Rinv.p);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(2);
    }
    // W against the first nb blocks (two classical Gram-Schmidt passes), then Cholesky QR twice,
    // all on the device.  Astore[slot] receives the projection on block nb-1 (both passes),
    // Rstore[slot] the triangular factor (W = Q_new R); a rank loss sets the device flag.
    void orth(VT* W, int nb, int slot) {
        const double2* gpre = nullptr;
        if (nb > 0) {
            proj(W, B, W, Gpre.p);
            gpre = Gpre.p;
            const int ncol = nb * B;
            proj(Q.p, ncol, W, C1.p);
            update(ncol, C1.p, W);
            proj(Q.p, ncol, W, C2.p);
            update(ncol, C2.p, W);
            k_bl_add<<<(B * B + 255) / 256, 256, 0, st>>>(C1.p + (size_t)(nb - 1) * B * B,
                                                          C2.p + (size_t)(nb - 1) * B * B, B * B,
                                                          Astore.p + (size_t)slot * B * B);
            note_launches(1);
        }
        double2* Racc = Rstore.p + (size_t)slot * B * B;
        cholqr_pass(W, 0, gpre, Racc);
        cholqr_pass(W, 1, nullptr, Racc);
    }
    // the factors of steps [j0, j1) on the host; throws Breakdown when a block lost rank
    void fetch_factors(int j0, int j1, std::vector<std::vector<cd>>& A, std::vector<std::vector<cd>>& R) {
        const size_t bb = (size_t)B * B, cnt = (size_t)(j1 - j0) * bb;
        std::vector<double2> ah(cnt), rh(cnt);
        int fl = 0;
        if (cnt) {
            MOMED_CUDA_TRY(cudaMemcpyAsync(ah.data(), Astore.p + j0 * bb, cnt * sizeof(double2), cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaMemcpyAsync(rh.data(), Rstore.p + j0 * bb, cnt * sizeof(double2), cudaMemcpyDeviceToHost, st));
        }
        int te = 0;
        MOMED_CUDA_TRY(cudaMemcpyAsync(&fl, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(&te, tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        if (te) throw Error{MOMED_ETIMEOUT, "tensor-core projection: an mbarrier wait timed out"};
        if (fl) throw Breakdown{};
        for (int j = j0; j < j1; ++j) {
            A[j].assign(bb, 0.0);
            R[j].assign(bb, 0.0);
            for (size_t e = 0; e < bb; ++e) {
                const double2 a = ah[(j - j0) * bb + e], r = rh[(j - j0) * bb + e];
                A[j][e] = cd(a.x, a.y);
                R[j][e] = cd(r.x, r.y);
            }
        }
    }
    void combine_blocked(const std::vector<cd>& Y, int ncol, int nout, VT* out) {
        upload_y(Y);
        launch_combine<VT, true>(ncol, nout, out, N * B);
    }
    void combine_cols(const std::vector<cd>& Y, int ncol, int nout, double2* out) {
        upload_y(Y);
        launch_combine<double2, false>(ncol, nout, out, 0);
    }
    void upload_y(const std::vector<cd>& Y) {
        std::vector<double2> yh(Y.size());
        for (size_t i = 0; i < Y.size(); ++i) yh[i] = make_double2(Y[i].real(), Y[i].imag());
        Yd.resize(yh.size());
        MOMED_CUDA_TRY(cudaMemcpyAsync(Yd.p, yh.data(), yh.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    template <typename VOUT, bool BLOCKED>
    void launch_combine(int ncol, int nout, VOUT* out, int64_t out_stride) {
        auto k = k_bl_combine<VT, VOUT, B, BLOCKED>;
        const size_t smem = (size_t)ncol * B * sizeof(double2);
        constexpr size_t smem_max = (size_t)kMaxCoef * sizeof(double2);
        if (smem_max > 48 * 1024)
            MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
        dim3 g((unsigned)ugrid(), (unsigned)((nout + B - 1) / B));
        k<<<g, kBT, smem, st>>>(Q.p, N * B, ncol, N, Yd.p, nout, out, out_stride);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(1);
    }

    struct Out {
        std::vector<double> theta, resid;
        int nconv = 0, restarts = 0;
        int kept = 0;
    };

    // Runs to convergence.  start: optional columns [ns][N] c128 (ns <= B) for the first block,
    // the rest random from seed.  Convergence on residual <= max(tol, rel_floor * max|theta|).
    // vectors (nullable, device c128 [nwant][N]): the nwant lowest Ritz vectors.
    Out run(int nev, double tol, double rel_floor, int maxiter, const double2* start, int ns, uint64_t seed,
            int nwant, double2* vectors) {
        Out out;
        vec_random<VT>(blk(0), N * B, seed, st);
        if (start && ns > 0) {
            const int g = (int)std::max<int64_t>(1, std::min<int64_t>((N * B + kBT - 1) / kBT, (int64_t)blk_sms() * 8));
            k_bl_from_cols<VT, B><<<g, kBT, 0, st>>>(start, std::min(ns, B), N, blk(0));
            note_launches(1);
        }
        orth(blk(0), 0, mb);
        std::vector<std::vector<cd>> Ablk(mb), Rblk(mb);
        std::vector<double> kept_theta;
        std::vector<cd> S;            // [B][k] coupling of the residual block to the kept vectors
        int kb = 0;                   // kept blocks
        int restarts = 0;
        std::vector<cd> T, Z;
        std::vector<double> th(m);
        for (;;) {
            for (int j = kb; j < mb; ++j) {
                VT* W = blk(j + 1);
                map(blk(j), W);
                orth(W, j + 1, j);
            }
            fetch_factors(kb, mb, Ablk, Rblk);
            // projected matrix
            T.assign((size_t)m * m, 0.0);
            const int k = kb * B;
            for (int i = 0; i < k; ++i) T[(size_t)i * m + i] = kept_theta[i];
            if (kb > 0)
                for (int a = 0; a < B; ++a)
                    for (int i = 0; i < k; ++i) {
                        T[(size_t)(k + a) * m + i] = S[(size_t)a * k + i];
                        T[(size_t)i * m + k + a] = std::conj(S[(size_t)a * k + i]);
                    }
            for (int j = kb; j < mb; ++j) {
                for (int a = 0; a < B; ++a)
                    for (int r = 0; r < B; ++r) {
                        // A[a][r] = q_{j,a}^H H q_{j,r}: Hermitian up to rounding
                        const cd v = 0.5 * (Ablk[j][(size_t)a * B + r] + std::conj(Ablk[j][(size_t)r * B + a]));
                        T[(size_t)(j * B + a) * m + j * B + r] = v;
                    }
                if (j + 1 < mb)
                    for (int a = 0; a < B; ++a)
                        for (int r = 0; r < B; ++r) {
                            const cd v = Rblk[j][(size_t)a * B + r];
                            T[(size_t)((j + 1) * B + a) * m + j * B + r] = v;
                            T[(size_t)(j * B + r) * m + (j + 1) * B + a] = std::conj(v);
                        }
            }
            Z.assign((size_t)m * m, 0.0);
            herm_eig(m, T.data(), th.data(), Z.data());
            // residual of Ritz pair i: || R_last Z[last block rows, i] ||
            const std::vector<cd>& Rl = Rblk[mb - 1];
            std::vector<double> res(m);
            double tmax = 0.0;
            for (int i = 0; i < m; ++i) tmax = std::max(tmax, std::fabs(th[i]));
            for (int i = 0; i < m; ++i) {
                double s2 = 0.0;
                for (int a = 0; a < B; ++a) {
                    cd v = 0.0;
                    for (int r = 0; r < B; ++r) v += Rl[(size_t)a * B + r] * Z[(size_t)((mb - 1) * B + r) * m + i];
                    s2 += std::norm(v);
                }
                res[i] = std::sqrt(s2);
            }
            const double eff = std::max(tol, rel_floor * tmax);
            int nconv = 0;
            while (nconv < nev && nconv < m && res[nconv] <= eff) ++nconv;
            if (nconv >= nev || restarts >= maxiter) {
                out.theta = th;
                out.resid = res;
                out.nconv = nconv;
                out.restarts = restarts;
                const int nv = std::min(nwant, m);
                out.kept = nv;
                if (vectors && nv > 0) {
                    std::vector<cd> Y((size_t)m * nv);
                    for (int c = 0; c < m; ++c)
                        for (int i = 0; i < nv; ++i) Y[(size_t)c * nv + i] = Z[(size_t)c * m + i];
                    combine_cols(Y, m, nv, vectors);
                    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                }
                return out;
            }
            // restart: keep the leading Ritz vectors (whole blocks), the residual block follows
            int keep = nev + (m - nev) / 3;
            keep = std::max(keep, std::min(nwant, m - B));
            keep = std::min(keep, m - 3 * B);          // at least three new blocks per cycle
            int nkb = (keep + B - 1) / B;
            nkb = std::max(1, std::min(nkb, mb - 1));
            const int nk = nkb * B;
            std::vector<cd> Y((size_t)m * nk);
            for (int c = 0; c < m; ++c)
                for (int i = 0; i < nk; ++i) Y[(size_t)c * nk + i] = Z[(size_t)c * m + i];
            Q2.resize((size_t)(mb + 1) * N * B);
            combine_blocked(Y, m, nk, Q2.p);
            MOMED_CUDA_TRY(cudaMemcpyAsync(Q2.p + (size_t)nkb * N * B, blk(mb), (size_t)N * B * sizeof(VT),
                                           cudaMemcpyDeviceToDevice, st));
            std::swap(Q.p, Q2.p);
            std::swap(Q.n, Q2.n);
            kept_theta.assign(th.begin(), th.begin() + nk);
            S.assign((size_t)B * nk, 0.0);
            for (int a = 0; a < B; ++a)
                for (int i = 0; i < nk; ++i) {
                    cd v = 0.0;
                    for (int r = 0; r < B; ++r) v += Rl[(size_t)a * B + r] * Z[(size_t)((mb - 1) * B + r) * m + i];
                    S[(size_t)a * nk + i] = v;
                }
            kb = nkb;
            ++restarts;
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        }
    }
};

// Basis blocks of a cycle.  A block Krylov space of mb blocks carries polynomials of degree mb
// only, so a block basis must hold many more vectors than a single-vector one of the same
// convergence: emulated on a 3x6 sector (nev 4-10), restarts with 20 blocks of 4 or 16 of 8
// needed 1.1-1.7x the maps of the single-vector solver at krylovdim 30 (in 1/B of the
// launches), 8 blocks of 8 needed 2-6x.  Capped by the kernels' column limits and by device
// memory (the basis and its restart copy); 0 when even 6 blocks do not fit.
int pick_blocks(int64_t N, int nev, int krylovdim, int B, size_t elem_bytes) {
    int mb = B <= 4 ? 20 : (B <= 8 ? 16 : 8);
    mb = std::max(mb, (krylovdim + B - 1) / B + 2);
    mb = std::max(mb, (nev + B - 1) / B + 4);
    mb = std::min(mb, std::min(kMaxBlkCols, kMaxCoef / B) / B);
    if ((int64_t)(mb + 1) * B > N) mb = (int)std::max<int64_t>(1, N / B - 1);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b > 0)
        while (mb > 6 && 2.0 * (mb + 1) * (double)N * B * elem_bytes > 0.6 * (double)free_b) --mb;
    if (mb < 6 || 2.0 * (mb + 1) * (double)N * B * elem_bytes > 0.6 * (double)(free_b ? free_b : ~size_t(0)))
        return 0;
    return mb;
}

template <int B>
int solve_blocked(momed_handle* h, const momed_solve_opts* o, int nev, const double2* start64, double2* X,
                  std::vector<double>& theta, std::vector<double>& res, int& nconv, int& restarts, int64_t& matvecs,
                  int64_t& matvecs64) {
    const int64_t N = h->n;
    const double tol = o->tol > 0 ? o->tol : 1e-12;
    const int maxiter = o->maxiter > 0 ? o->maxiter : 100;
    const int mb = pick_blocks(N, nev, o->krylovdim > 0 ? o->krylovdim : 30, B,
                               o->precision == MOMED_PREC_MIXED ? sizeof(float2) : sizeof(double2));
    if (mb == 0) throw Breakdown{};           // no room for a block basis: the single-vector solver
    cudaStream_t st = h->stream;
    if (o->precision == MOMED_PREC_MIXED) {
        const int extra = std::min(4, std::max(0, mb * B - 2 * B - nev));
        const int k1 = nev + extra;
        DevBuf<double2> X1, W1, S1;
        X1.resize((size_t)k1 * N);
        W1.resize((size_t)k1 * N);
        S1.resize((size_t)k1 * N);
        typename BlockKrylov<float2, B>::Out r1;
        {
            // converge the nev wanted pairs to the FP32 floor and return k1 Ritz vectors: the
            // extra ones need not reach the floor (asking it of them stalled the phase when
            // k1 = B: 3x9, nev 4, B = 8 forced ran 14 s)
            BlockKrylov<float2, B> K(h, mb);
            r1 = K.run(nev, 0.0, 2e-6, maxiter, start64, start64 ? 1 : 0, o->seed, k1, X1.p);
            matvecs += K.matvecs;
        }
        restarts += r1.restarts;
        const int kk = std::min(k1, r1.kept);
        std::vector<double> th2, rs2;
        rayleigh_ritz_fp64(h, X1.p, W1.p, S1.p, kk, th2, rs2, matvecs64);
        matvecs += kk;
        const double outside = (int)r1.theta.size() > kk ? r1.theta[kk] : th2.back() + 1.0;
        bool ok = true;
        nconv = 0;
        for (int i = 0; i < nev; ++i) {
            double gap = std::fabs(outside - th2[i]);
            for (int j = 0; j < kk; ++j)
                if (j != i && std::fabs(th2[j] - th2[i]) > 1e-9 * std::max(1.0, std::fabs(th2[i])))
                    gap = std::min(gap, std::fabs(th2[j] - th2[i]));
            const double est = rs2[i] * rs2[i] / std::max(gap, 1e-300);
            const bool good = rs2[i] <= tol || est <= 1e-11 * std::max(1.0, std::fabs(th2[i]));
            if (good && nconv == i) ++nconv;
            ok = ok && good;
        }
        if (ok) {
            theta = th2;
            res = rs2;
            MOMED_CUDA_TRY(cudaMemcpyAsync(X, X1.p, (size_t)nev * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
            return 0;
        }
        // FP64 block Lanczos warm-started from the refined vectors
        const int mb64 = pick_blocks(N, nev, o->krylovdim > 0 ? o->krylovdim : 30, B, sizeof(double2));
        if (mb64 == 0) throw Breakdown{};
        BlockKrylov<double2, B> K(h, mb64);
        auto r3 = K.run(nev, tol, 0.0, maxiter, X1.p, std::min(kk, B), o->seed, nev, X);
        theta = r3.theta;
        res = r3.resid;
        nconv = r3.nconv;
        matvecs += K.matvecs;
        matvecs64 += K.matvecs;
        restarts += r3.restarts;
        return 0;
    }
    BlockKrylov<double2, B> K(h, mb);
    auto r = K.run(nev, tol, 0.0, maxiter, start64, start64 ? 1 : 0, o->seed, nev, X);
    theta = r.theta;
    res = r.resid;
    nconv = r.nconv;
    restarts = r.restarts;
    matvecs = matvecs64 = K.matvecs;
    return 0;
}

}  // namespace

// Block size for a solve of nev pairs on N states (0: the single-vector solver).  The block
// method needs the matrix-free block map (or, in mixed precision, the block SpMV): an FP64
// solve while a sparse matrix is built stays single-vector.  MOMED_BLOCK (environment) forces a
// size (0 disables).
int block_size_for(momed_handle* h, int nev, int precision) {
    if (h->sparse_only || h->block_solver == 0) return 0;
    // on a sparse matrix the single-vector SpMV paths win (the mixed block solver's FP64 phase would
    // run on the candidate block map: plain_3x10 mixed 0.55 against 2.0 solves/s)
    if (h->sparse.built) return 0;
    if (const char* e = std::getenv("MOMED_BLOCK")) {
        const int b = std::atoi(e);
        return (b == 4 || b == 8 || b == 16) && h->n >= 16 * b ? b : 0;
    }
    // Measured on B200 (FP64 / mixed solves per second, single-vector -> block) with the candidate
    // map: 3x9 (174k states, nev 4) 6.69 -> 4.35 with B = 4 (the block needs 2.8x the maps: 464
    // against 165); 3x10 (1.0M, nev 6) 0.487 -> 0.647 with B = 4, 0.527 with B = 8 (mixed 0.34 /
    // 0.50); two-component 4x6 (4.7M, nev 8) 0.063 -> 0.080 with B = 4, 0.067 with B = 8 (mixed
    // 0.040 -> 0.058); 4x9 Ne = 12 (34.8M, nev 4) 69.9 s -> 108.7 s with B = 4 (560 maps against
    // 209).  With few wanted pairs per block vector the block Krylov space needs too many more
    // vectors.  The block map's saving is the candidate stage shared by B vectors; over a hit
    // cache there is no candidate stage and the saving is the B-wide gathers only: 3x10 1.93
    // single-vector against 1.60 with B = 4, two-component 4x6 0.181 against 0.250.  So: the
    // block solver for nev >= 6, from 500k states on the candidate map, from 2M over a hit cache.
    // Mixed precision goes to the batched solver with one right-hand side instead (its anchored
    // FP64 refinement): two-component 4x6, nev 8: 2.73 s against 7.56 s for the mixed block solver
    // (whose FP64 phase restarts from B of the refined vectors) and 4.2 s for the FP64 one.
    if (nev < 6 || h->n < (h->hcache.full() ? 2000000 : 500000)) return 0;
    if (precision == MOMED_PREC_MIXED) return 0;
    return nev <= 10 ? 4 : 8;
}

// The block solver's part of momed_eigsolve: fills theta/res (at least nev entries) and X
// [nev][N]; returns false when the block recurrence broke down (the caller then runs the
// single-vector solver).
bool eigsolve_block(momed_handle* h, const momed_solve_opts* o, int nev, int B, const double2* start64, double2* X,
                    std::vector<double>& theta, std::vector<double>& res, int& nconv, int& restarts, int64_t& matvecs,
                    int64_t& matvecs64) {
    try {
        switch (B) {
            case 4: solve_blocked<4>(h, o, nev, start64, X, theta, res, nconv, restarts, matvecs, matvecs64); break;
            case 8: solve_blocked<8>(h, o, nev, start64, X, theta, res, nconv, restarts, matvecs, matvecs64); break;
            case 16: solve_blocked<16>(h, o, nev, start64, X, theta, res, nconv, restarts, matvecs, matvecs64); break;
            default: throw Error{MOMED_EINVAL, "block size must be 4, 8 or 16"};
        }
    } catch (const Breakdown&) {
        return false;
    }
    return true;
}

}  // namespace momed
