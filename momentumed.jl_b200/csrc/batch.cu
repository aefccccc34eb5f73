// Batched solver: one sector, nu values of a parameter u, H(u) = A + u B.
//
// The sweep form of the reference workflow (EDsolve called in a loop over
// interaction strengths, examples/landau level torus notebooks) as one
// device job: the nu Lanczos processes advance in lockstep on block vectors
// x[row * NB + r] (NB = nu rounded up to a power of two <= 32), so every
// index lookup of the block matvec serves all NB right-hand sides and every
// gather reads NB contiguous values.  Recurrences, reorthogonalisation and
// restarts are independent per right-hand side (per-r coefficients, per-r
// projected matrices and per-r restart combinations).
//
// Precision: the mixed form runs the lockstep Lanczos in complex64 (FP64
// dot products), then an FP64 block Rayleigh-Ritz on the Ritz vectors; right-hand
// sides whose estimated eigenvalue error stays above the target are finished by an
// FP64 single-vector Lanczos warm-started from their refined vectors.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <future>
#include <thread>
#include <type_traits>

#include "vecops.cuh"

namespace momed {

void ensure_ready(momed_handle* h);
bool gen_herm_eig(int k, const std::vector<std::complex<double>>& G, const std::vector<std::complex<double>>& S,
                  std::vector<double>& theta, std::vector<std::complex<double>>& Y);

namespace {

constexpr int kT = 256;
constexpr int kRowsTile = 64;   // rows of W staged per tile in k_bproj
// Accepted eigenvalue error estimate (relative, r^2/gap) of the mixed-precision batch: 10x
// below the 1e-10 target.
constexpr double kEigTarget = 1e-11;

__device__ __forceinline__ double2 to2(double2 v) { return v; }
__device__ __forceinline__ double2 to2(float2 v) { return make_double2(v.x, v.y); }
template <typename VT> __device__ __forceinline__ VT fr2(double2 v);
template <> __device__ __forceinline__ double2 fr2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 fr2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// partial[b][i][r] (i <= ncols: column ncols holds |w_r|^2)
template <typename VT, int NB>
__global__ void __launch_bounds__(kT)
k_bproj(const VT* __restrict__ V, int64_t N, int ncols, const VT* __restrict__ W, double2* partial,
        const int* active_any) {
    if (active_any && *active_any == 0) return;
    constexpr int RS = 32 / NB;                 // row subsets per warp
    __shared__ double2 ws[kRowsTile * NB];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int r = lane % NB, rs = lane / NB;
    double2 acc[kColsPerWarp];
#pragma unroll
    for (int k = 0; k < kColsPerWarp; ++k) acc[k] = make_double2(0.0, 0.0);
    double wn2 = 0.0;
    int64_t per = (N + gridDim.x - 1) / gridDim.x;
    int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(N, r0 + per);
    for (int64_t t0 = r0; t0 < r1; t0 += kRowsTile) {
        const int rows = (int)((r1 - t0) < kRowsTile ? (r1 - t0) : kRowsTile);
        for (int e = threadIdx.x; e < kRowsTile * NB; e += kT) {
            int t = e / NB;
            double2 v = (t < rows) ? to2(W[(t0 + t) * NB + (e % NB)]) : make_double2(0.0, 0.0);
            ws[e] = v;
        }
        __syncthreads();
        if (wid == 0) {
            for (int t = rs; t < rows; t += RS) {
                double2 v = ws[t * NB + r];
                wn2 += v.x * v.x + v.y * v.y;
            }
        }
#pragma unroll
        for (int k = 0; k < kColsPerWarp; ++k) {
            int i = wid + 8 * k;
            if (i < ncols) {
                const VT* col = V + (int64_t)i * N * NB + t0 * NB;
                for (int t = rs; t < rows; t += RS) {
                    double2 v = to2(col[t * NB + r]);
                    double2 w = ws[t * NB + r];
                    acc[k].x += v.x * w.x + v.y * w.y;
                    acc[k].y += v.x * w.y - v.y * w.x;
                }
            }
        }
        __syncthreads();
    }
    double2* out = partial + (int64_t)blockIdx.x * (kMaxCols + 1) * NB;
#pragma unroll
    for (int k = 0; k < kColsPerWarp; ++k) {
        int i = wid + 8 * k;
        double sx = acc[k].x, sy = acc[k].y;
#pragma unroll
        for (int o = NB; o < 32; o <<= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (i < ncols && rs == 0) out[i * NB + r] = make_double2(sx, sy);
    }
    if (wid == 0) {
#pragma unroll
        for (int o = NB; o < 32; o <<= 1) wn2 += __shfl_xor_sync(0xffffffffu, wn2, o);
        if (rs == 0) out[ncols * NB + r] = make_double2(wn2, 0.0);
    }
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one warp per (column, right-hand side) element; fixed reduction order
template <int NB>
__global__ void k_breduce(const double2* partial, int grid, int ncols1, double2* out, const int* active_any) {
    if (active_any && *active_any == 0) return;
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= ncols1 * NB) return;
    double sx = 0.0, sy = 0.0;
    for (int b = lane; b < grid; b += 32) {
        double2 v = partial[(int64_t)b * (kMaxCols + 1) * NB + e];
        sx += v.x;
        sy += v.y;
    }
    sx = wsum(sx);
    sy = wsum(sy);
    if (lane == 0) out[e] = make_double2(sx, sy);
}

inline int breduce_grid(int ncols1, int nb) { return (ncols1 * nb + 7) / 8; }

// W[n][r] -= sum_i coef[i][r] V_i[n][r] for active r; per-block |W_r|^2 partials
template <typename VT, int NB>
__global__ void __launch_bounds__(kT)
k_bupdate(const VT* __restrict__ V, int64_t N, int ncols, const double2* __restrict__ coef, VT* __restrict__ W,
          double* npartial /* [grid][NB] */, const int* active /* [NB] or null */, const int* active_any) {
    if (active_any && *active_any == 0) return;
    extern __shared__ double2 c[];   // [ncols * NB]
    __shared__ double nrm[32];
    for (int e = threadIdx.x; e < ncols * NB; e += kT) c[e] = coef[e];
    if (threadIdx.x < 32) nrm[threadIdx.x] = 0.0;
    __syncthreads();
    const int r = threadIdx.x % NB;
    const bool on = !active || active[r];
    double wn2 = 0.0;
    const int64_t total = N * NB;
    for (int64_t e = (int64_t)blockIdx.x * kT + threadIdx.x; e < total; e += (int64_t)gridDim.x * kT) {
        double2 acc = to2(W[e]);
        if (on) {
            const int64_t n = e / NB;
            for (int i = 0; i < ncols; ++i) {
                double2 cf = c[i * NB + r];
                double2 v = to2(V[(int64_t)i * N * NB + n * NB + r]);
                acc.x -= cf.x * v.x - cf.y * v.y;
                acc.y -= cf.x * v.y + cf.y * v.x;
            }
            VT st = fr2<VT>(acc);
            W[e] = st;
            acc = to2(st);
        }
        wn2 += acc.x * acc.x + acc.y * acc.y;
    }
    atomicAdd(&nrm[r], wn2);
    __syncthreads();
    if (threadIdx.x < NB) npartial[(int64_t)blockIdx.x * NB + threadIdx.x] = nrm[threadIdx.x];
}

// launched with NB warps: warp r reduces the norm partials of right-hand side r
template <int NB>
__global__ void k_bdecide(const double2* coefA, int ncols, const double* npartial, int grid, int* flag, int* any,
                          double* after) {
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    double a = 0.0;
    for (int b = lane; b < grid; b += 32) a += npartial[(int64_t)b * NB + r];
    a = wsum(a);
    if (lane == 0) {
        double before = coefA[ncols * NB + r].x;
        after[r] = a;
        int f = (a < 0.5 * before) ? 1 : 0;
        flag[r] = f;
        if (f) atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *any = s_any;
}

template <int NB>
__global__ void k_bfinalize(const double2* coefA, const double2* coefB, int ncols, const double* npartial2, int grid,
                            const int* flag, const int* any, const double* after, double* scal, double* alpha,
                            double* beta, int j, int m) {
    // launched with NB warps: warp r finalises right-hand side r
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    const bool anyp = *any != 0;
    double s = 0.0;
    if (anyp) {   // uniform: the second pass recomputed every r's norm (inactive r unchanged)
        for (int b = lane; b < grid; b += 32) s += npartial2[(int64_t)b * NB + r];
        s = wsum(s);
    }
    if (lane != 0) return;
    bool second = anyp && flag[r];
    double a = coefA[(ncols - 1) * NB + r].x + (second ? coefB[(ncols - 1) * NB + r].x : 0.0);
    double wn2 = anyp ? s : after[r];
    double bt = sqrt(max(wn2, 0.0));
    alpha[r * m + j] = a;
    beta[r * m + j] = bt;
    scal[r] = bt > 0.0 ? 1.0 / bt : 0.0;
}

template <typename VT, int NB>
__global__ void k_bscale(VT* W, int64_t N, const double* scal) {
    const int64_t total = N * NB;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        double s = scal[e % NB];
        double2 v = to2(W[e]);
        W[e] = fr2<VT>(make_double2(v.x * s, v.y * s));
    }
}

template <typename VT>
__global__ void k_brandom(VT* v, int64_t total, uint64_t seed) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        auto mix = [](uint64_t z) {
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            return z ^ (z >> 31);
        };
        double a = (double)(mix(seed + (2 * (uint64_t)e + 1) * 0x9E3779B97F4A7C15ULL) >> 11) * (1.0 / 9007199254740992.0);
        double b = (double)(mix(seed + (2 * (uint64_t)e + 2) * 0x9E3779B97F4A7C15ULL) >> 11) * (1.0 / 9007199254740992.0);
        v[e] = fr2<VT>(make_double2(a, b));
    }
}

// out[i][n][r] = sum_a U[i][a][r] V[a][n][r]  (U: [nout][m][NB], r fastest so a warp's coefficient
// loads are coalesced), optionally out[nout] = V[copy_col].  A tile of TR rows x (m+1) columns is
// staged in shared memory; each thread owns RPT rows of one right-hand side and accumulates OC
// outputs at a time in registers.  In place (out == V) is safe: a tile is read whole before any
// of its rows is written.
template <typename VIN, typename VOUT, int NB, int RPT>
__global__ void __launch_bounds__(kT)
k_bcombine(const VIN* V, int64_t N, int m, const double* __restrict__ U, int nout, VOUT* out, int copy_col) {
    constexpr int TPR = kT / NB;        // row slots per pass
    constexpr int TR = TPR * RPT;       // rows per tile
    constexpr int OC = 8;               // outputs per register chunk
    extern __shared__ unsigned char smem_raw[];
    VIN* tile = reinterpret_cast<VIN*>(smem_raw);   // [(m + 1)][TR][NB]
    const int ncopy = copy_col >= 0 ? 1 : 0;
    const int r = threadIdx.x % NB, tl = threadIdx.x / NB;
    for (int64_t t0 = (int64_t)blockIdx.x * TR; t0 < N; t0 += (int64_t)gridDim.x * TR) {
        const int rows = (int)((N - t0) < TR ? (N - t0) : TR);
        for (int e = threadIdx.x; e < (m + ncopy) * TR * NB; e += kT) {
            int a = e / (TR * NB), rem = e % (TR * NB);
            int t = rem / NB;
            int col = a < m ? a : copy_col;
            VIN z;
            z.x = 0;
            z.y = 0;
            tile[e] = (t < rows) ? V[(int64_t)col * N * NB + (t0 + t) * NB + (rem % NB)] : z;
        }
        __syncthreads();
        for (int c0 = 0; c0 < nout; c0 += OC) {
            double ax[RPT][OC], ay[RPT][OC];
#pragma unroll
            for (int j = 0; j < RPT; ++j)
#pragma unroll
                for (int k = 0; k < OC; ++k) { ax[j][k] = 0.0; ay[j][k] = 0.0; }
            for (int a = 0; a < m; ++a) {
                double u[OC];
#pragma unroll
                for (int k = 0; k < OC; ++k)
                    u[k] = (c0 + k < nout) ? __ldg(U + ((int64_t)(c0 + k) * m + a) * NB + r) : 0.0;
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    double2 v = to2(tile[(a * TR + tl + j * TPR) * NB + r]);
#pragma unroll
                    for (int k = 0; k < OC; ++k) {
                        ax[j][k] += u[k] * v.x;
                        ay[j][k] += u[k] * v.y;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                const int t = tl + j * TPR;
                if (t < rows) {
#pragma unroll
                    for (int k = 0; k < OC; ++k)
                        if (c0 + k < nout)
                            out[(int64_t)(c0 + k) * N * NB + (t0 + t) * NB + r] =
                                fr2<VOUT>(make_double2(ax[j][k], ay[j][k]));
                }
            }
        }
        if (ncopy) {
            for (int e = threadIdx.x; e < rows * NB; e += kT)
                out[(int64_t)nout * N * NB + t0 * NB + e] = fr2<VOUT>(to2(tile[(m * TR) * NB + e]));
        }
        __syncthreads();
    }
}

template <int NB>
__global__ void k_binv(const double2* c, double* scal) {
    int r = threadIdx.x;
    if (r < NB) {
        double v = c[r].x;
        scal[r] = v > 0.0 ? 1.0 / sqrt(v) : 0.0;
    }
}

// deinterleave one right-hand side: dst[i][n] = src[i][n][r] (c128)
template <int NB>
__global__ void k_extract(const double2* src, int64_t N, int k, int r, double2* dst) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)k * N; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = e / N, n = e % N;
        dst[e] = src[i * N * NB + n * NB + r];
    }
}

int sms() {
    static int s = 0;
    if (!s) {
        int d = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, d);
        if (s <= 0) s = 148;
    }
    return s;
}

template <typename VT> struct BlockMv;
template <> struct BlockMv<float2> {
    static void run(momed_handle* h, const float2* x, float2* y, const float* u, int nb) {
        prof_begin(h);
        launch_block_matvec_c64(index_view(h), h->op.view(), x, y, u, nb, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_BLOCK_MATVEC_C64);
    }
};
template <> struct BlockMv<double2> {
    static void run(momed_handle* h, const double2* x, double2* y, const double* u, int nb) {
        prof_begin(h);
        launch_block_matvec_c128(index_view(h), h->op.view(), x, y, u, nb, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_BLOCK_MATVEC_C128);
    }
};

template <typename VT, int NB>
struct BlockLanczos {
    using RT = typename std::conditional<std::is_same<VT, float2>::value, float, double>::type;
    momed_handle* h;
    int64_t N;
    int m;
    cudaStream_t st;
    int grid, ugrid;
    DevBuf<VT> V;
    DevBuf<double2> partial, coefA, coefB;
    DevBuf<double> npart, after, scal, alpha, beta, Ud;
    DevBuf<int> flag, any;
    DevBuf<RT> ud;
    int64_t launches = 0;

    BlockLanczos(momed_handle* hh, int mm, const std::vector<double>& u) : h(hh), N(hh->n), m(mm), st(hh->stream) {
        grid = std::max(1, std::min<int>((int)((N + kRowsTile - 1) / kRowsTile), sms() * 2));
        ugrid = std::max(1, std::min<int>((int)((N * NB + kT - 1) / kT), sms() * 8));
        V.resize((size_t)(m + 1) * N * NB);
        partial.resize((size_t)grid * (kMaxCols + 1) * NB);
        coefA.resize((size_t)(kMaxCols + 1) * NB);
        coefB.resize((size_t)(kMaxCols + 1) * NB);
        npart.resize((size_t)ugrid * NB);
        after.resize(NB);
        scal.resize(NB);
        alpha.resize((size_t)NB * m);
        beta.resize((size_t)NB * m);
        Ud.resize((size_t)NB * m * m);
        flag.resize(NB);
        any.resize(1);
        ud.resize(NB);
        std::vector<RT> uh(NB, (RT)0);
        for (size_t r = 0; r < u.size() && r < (size_t)NB; ++r) uh[r] = (RT)u[r];
        MOMED_CUDA_TRY(cudaMemcpyAsync(ud.p, uh.data(), NB * sizeof(RT), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    VT* col(int i) { return V.p + (size_t)i * N * NB; }

    void proj(int ncols, const VT* w, double2* out, const int* act) {
        k_bproj<VT, NB><<<grid, kT, 0, st>>>(V.p, N, ncols, w, partial.p, act);
        k_breduce<NB><<<breduce_grid(ncols + 1, NB), 256, 0, st>>>(partial.p, grid, ncols + 1, out, act);
        launches += 2;
    }
    void update(int ncols, const double2* coef, VT* w, const int* active, const int* act) {
        size_t smem = (size_t)ncols * NB * sizeof(double2);
        auto k = k_bupdate<VT, NB>;
        if (smem > 48 * 1024) MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<ugrid, kT, smem, st>>>(V.p, N, ncols, coef, w, npart.p, active, act);
        ++launches;
    }
    void normalize(VT* v) {
        proj(0, v, coefA.p, nullptr);
        k_binv<NB><<<1, 32, 0, st>>>(coefA.p, scal.p);
        k_bscale<VT, NB><<<ugrid, kT, 0, st>>>(v, N, scal.p);
        launches += 2;
    }
    void step(int j) {
        VT* w = col(j + 1);
        BlockMv<VT>::run(h, col(j), w, ud.p, NB);   // counted by its launcher
        const int nc = j + 1;
        proj(nc, w, coefA.p, nullptr);
        update(nc, coefA.p, w, nullptr, nullptr);
        k_bdecide<NB><<<1, NB * 32, 0, st>>>(coefA.p, nc, npart.p, ugrid, flag.p, any.p, after.p);
        proj(nc, w, coefB.p, any.p);
        update(nc, coefB.p, w, flag.p, any.p);
        k_bfinalize<NB><<<1, NB * 32, 0, st>>>(coefA.p, coefB.p, nc, npart.p, ugrid, flag.p, any.p, after.p, scal.p,
                                          alpha.p, beta.p, j, m);
        k_bscale<VT, NB><<<ugrid, kT, 0, st>>>(w, N, scal.p);
        launches += 3;
    }
    template <typename VOUT>
    void combine(const std::vector<double>& Uh, int nout, VOUT* out, int copy_col, int mm) {
        MOMED_CUDA_TRY(cudaMemcpyAsync(Ud.p, Uh.data(), Uh.size() * 8, cudaMemcpyHostToDevice, st));
        constexpr int TPR = kT / NB;
        const size_t per_row = (size_t)(mm + 1) * NB * sizeof(VT);
        const size_t limit = 200 * 1024;
        if (per_row * TPR * 2 <= limit) {
            constexpr int TR = TPR * 2;
            size_t smem = per_row * TR;
            auto k = k_bcombine<VT, VOUT, NB, 2>;
            MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int g = (int)std::max<int64_t>(1, std::min<int64_t>((N + TR - 1) / TR, (int64_t)sms()));
            k<<<g, kT, smem, st>>>(V.p, N, mm, Ud.p, nout, out, copy_col);
        } else {
            constexpr int TR = TPR;
            size_t smem = per_row * TR;
            MOMED_REQUIRE(smem <= 227 * 1024, MOMED_EINVAL, "krylovdim too large for the batched restart tile");
            auto k = k_bcombine<VT, VOUT, NB, 1>;
            MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int g = (int)std::max<int64_t>(1, std::min<int64_t>((N + TR - 1) / TR, (int64_t)sms()));
            k<<<g, kT, smem, st>>>(V.p, N, mm, Ud.p, nout, out, copy_col);
        }
        MOMED_CUDA_TRY(cudaGetLastError());
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        ++launches;
    }

    struct Out {
        std::vector<std::vector<double>> theta, resid;
        std::vector<int> nconv;
        std::vector<int> broken;   // right-hand sides whose Krylov space became invariant
        int restarts = 0;
        int64_t steps = 0;
    };

    // Lockstep thick-restart Lanczos for all NB right-hand sides.  vectors: [nwant][N][NB] c128.
    // start: optional device block [N][NB] of start vectors (normalised here); else random from seed
    // eig_target > 0 also accepts a pair whose Rayleigh-quotient error estimate res^2 / gap is
    // below eig_target * max(1, |theta|) (gap: distance to the nearest other Ritz value outside
    // its degenerate cluster), i.e. converges on eigenvalue accuracy rather than residual size.
    Out run(int nev, int nu, double tol, double rel_floor, int maxiter, uint64_t seed, int nwant, double2* vectors,
            const VT* start = nullptr, double eig_target = 0.0) {
        Out out;
        if (start) MOMED_CUDA_TRY(cudaMemcpyAsync(col(0), start, (size_t)N * NB * sizeof(VT), cudaMemcpyDeviceToDevice, st));
        else k_brandom<VT><<<ugrid, kT, 0, st>>>(col(0), N * NB, seed);
        normalize(col(0));
        std::vector<std::vector<double>> kept(NB), arrow(NB);
        std::vector<double> ha((size_t)NB * m), hb((size_t)NB * m);
        int k = 0, restarts = 0;
        int64_t steps = 0;
        std::vector<std::vector<double>> th(NB, std::vector<double>(m)), U(NB, std::vector<double>((size_t)m * m));
        std::vector<std::vector<double>> res(NB);
        std::vector<int> nconv(NB, 0);
        out.broken.assign(NB, 0);
        for (;;) {
            for (int j = k; j < m; ++j) { step(j); ++steps; }
            MOMED_CUDA_TRY(cudaMemcpyAsync(ha.data(), alpha.p, ha.size() * 8, cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaMemcpyAsync(hb.data(), beta.p, hb.size() * 8, cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            // per right-hand side projected eigenproblems, in parallel on the host
            auto solve_r = [&](int r) {
                std::vector<double> T((size_t)m * m, 0.0);
                for (int i = 0; i < k; ++i) {
                    T[(size_t)i * m + i] = kept[r][i];
                    T[(size_t)i * m + k] = arrow[r][i];
                    T[(size_t)k * m + i] = arrow[r][i];
                }
                for (int j = k; j < m; ++j) {
                    T[(size_t)j * m + j] = ha[(size_t)r * m + j];
                    if (j + 1 < m) {
                        T[(size_t)j * m + j + 1] = hb[(size_t)r * m + j];
                        T[(size_t)(j + 1) * m + j] = hb[(size_t)r * m + j];
                    }
                }
                symeig(m, T.data(), th[r].data(), U[r].data());
                double bl = hb[(size_t)r * m + m - 1];
                double tmax = 0.0;
                for (int i = 0; i < m; ++i) tmax = std::max(tmax, std::fabs(th[r][i]));
                double eff = std::max(tol, rel_floor * tmax);
                res[r].assign(m, 0.0);
                for (int i = 0; i < m; ++i) res[r][i] = std::fabs(bl * U[r][(size_t)(m - 1) * m + i]);
                auto good = [&](int i) {
                    if (res[r][i] <= eff) return true;
                    if (eig_target <= 0.0) return false;
                    const double ti = th[r][i], scale = std::max(1.0, std::fabs(ti));
                    double gap = 1e300;
                    for (int j = 0; j < m; ++j)
                        if (j != i && std::fabs(th[r][j] - ti) > 1e-9 * scale) gap = std::min(gap, std::fabs(th[r][j] - ti));
                    return res[r][i] * res[r][i] <= eig_target * scale * gap;
                };
                int c = 0;
                while (c < nev && c < m && good(c)) ++c;
                nconv[r] = c;
                double sc = tmax > 0 ? tmax : 1.0;
                for (int j = k; j + 1 < m; ++j)
                    if (hb[(size_t)r * m + j] <= 1e-13 * sc) out.broken[r] = 1;
                if (out.broken[r]) nconv[r] = nev;   // finished separately by the single-vector solver
            };
            {
                std::vector<std::future<void>> fs;
                for (int r = 0; r < NB; ++r) fs.push_back(std::async(std::launch::async, solve_r, r));
                for (auto& f : fs) f.get();
            }
            int minconv = nev;
            for (int r = 0; r < nu; ++r) minconv = std::min(minconv, nconv[r]);
            if (minconv >= nev || restarts >= maxiter) {
                out.theta = th;
                out.resid = res;
                out.nconv = nconv;
                out.restarts = restarts;
                out.steps = steps;
                if (vectors && nwant > 0) {
                    int nv = std::min(nwant, m);
                    std::vector<double> Uh((size_t)NB * nv * m);
                    for (int r = 0; r < NB; ++r)
                        for (int i = 0; i < nv; ++i)
                            for (int a = 0; a < m; ++a) Uh[((size_t)i * m + a) * NB + r] = U[r][(size_t)a * m + i];
                    combine<double2>(Uh, nv, vectors, -1, m);
                }
                return out;
            }
            int keep = (3 * m + 2 * minconv) / 5;
            keep = std::max(keep, std::min(nwant, m - 2));
            keep = std::max(keep, nev);
            keep = std::min(keep, m - 2);
            keep = std::max(keep, 1);
            std::vector<double> Uh((size_t)NB * keep * m);
            for (int r = 0; r < NB; ++r) {
                for (int i = 0; i < keep; ++i)
                    for (int a = 0; a < m; ++a) Uh[((size_t)i * m + a) * NB + r] = U[r][(size_t)a * m + i];
                kept[r].assign(th[r].begin(), th[r].begin() + keep);
                arrow[r].resize(keep);
                double bl = hb[(size_t)r * m + m - 1];
                for (int i = 0; i < keep; ++i) arrow[r][i] = bl * U[r][(size_t)(m - 1) * m + i];
            }
            combine<VT>(Uh, keep, V.p, m, m);
            k = keep;
            ++restarts;
        }
    }
};

// out[i][n][r] = sum_a Y[r][i][a] X[a][n][r]   (Y: [NB][k][k] complex, out != X)
template <int NB>
__global__ void k_bcombine_c(const double2* __restrict__ X, int64_t N, int k, const double2* __restrict__ Y,
                             double2* __restrict__ out) {
    const int64_t total = N * NB;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % NB);
        for (int i = 0; i < k; ++i) {
            double sx = 0.0, sy = 0.0;
            for (int a = 0; a < k; ++a) {
                double2 y = Y[((int64_t)r * k + i) * k + a];
                double2 x = X[(int64_t)a * total + e];
                sx += y.x * x.x - y.y * x.y;
                sy += y.x * x.y + y.y * x.x;
            }
            out[(int64_t)i * total + e] = make_double2(sx, sy);
        }
    }
}

// out[n][r] = sum_{i < k} X[i][n][r]  (warm-start block from refined Ritz vectors)
template <int NB>
__global__ void k_bsum(const double2* __restrict__ X, int64_t N, int k, double2* __restrict__ out) {
    const int64_t total = N * NB;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        double sx = 0.0, sy = 0.0;
        for (int i = 0; i < k; ++i) {
            double2 x = X[(int64_t)i * total + e];
            sx += x.x;
            sy += x.y;
        }
        out[e] = make_double2(sx, sy);
    }
}

// part[b][i][r] = sum over the block's rows of |W[i][n][r] - th[r][i] X[i][n][r]|^2
template <int NB>
__global__ void k_bresid(const double2* __restrict__ W, const double2* __restrict__ X, int64_t N, int k,
                         const double* __restrict__ th, double* part) {
    __shared__ double acc[32];
    const int64_t total = N * NB;
    const int r = threadIdx.x % NB;   // blockDim and the grid stride are multiples of NB
    for (int i = 0; i < k; ++i) {
        if (threadIdx.x < 32) acc[threadIdx.x] = 0.0;
        __syncthreads();
        const double t = th[r * k + i];
        double s = 0.0;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
            double2 w = W[(int64_t)i * total + e], x = X[(int64_t)i * total + e];
            double rx = w.x - t * x.x, ry = w.y - t * x.y;
            s += rx * rx + ry * ry;
        }
        atomicAdd(&acc[r], s);
        __syncthreads();
        if (threadIdx.x < NB) part[((int64_t)blockIdx.x * k + i) * NB + threadIdx.x] = acc[threadIdx.x];
        __syncthreads();
    }
}

template <int NB>
int run_batch(momed_handle* h, const momed_solve_opts* o, const double* u, int32_t nu, double* vals, double* resid,
              double* vecs, momed_info* info) {
    const int64_t N = h->n;
    const int nev = (int)std::min<int64_t>(o->nev, N);
    int m = o->krylovdim > 0 ? o->krylovdim : 30;
    m = (int)std::min<int64_t>(m, std::min<int64_t>(N, kMaxCols - 1));
    if (m < nev + 2 && m < N) m = (int)std::min<int64_t>(N, nev + 2);
    const double tol = o->tol > 0 ? o->tol : 1e-12;
    const int maxiter = o->maxiter > 0 ? o->maxiter : 100;
    cudaStream_t st = h->stream;
    std::vector<double> uv(u, u + nu);
    MOMED_CUDA_TRY(cudaEventRecord(h->ev0, st));
    int64_t matvecs = 0, matvecs64 = 0;
    int restarts = 0;
    const bool mixed = o->precision == MOMED_PREC_MIXED;
    const int extra = mixed ? std::min<int>(4, std::max<int>(0, m - 2 - nev)) : 0;
    const int k1 = nev + extra;
    const int64_t stride = N * NB;
    DevBuf<double2> Xb, Wb, Sb;      // [k1][N][NB] c128
    Xb.resize((size_t)k1 * stride);
    Wb.resize((size_t)k1 * stride);
    Sb.resize((size_t)k1 * stride);
    std::vector<std::vector<double>> theta1;
    std::vector<int> broken(NB, 0), nconv1(NB, nev);
    if (mixed) {
        BlockLanczos<float2, NB> L(h, m, uv);
        auto r = L.run(nev, nu, 0.0, 2e-6, maxiter, o->seed, k1, Xb.p);
        matvecs += r.steps * nu;
        restarts += r.restarts;
        theta1 = r.theta;
        broken = r.broken;
        note_launches(L.launches);
    } else {
        BlockLanczos<double2, NB> L(h, m, uv);
        auto r = L.run(nev, nu, tol, 0.0, maxiter, o->seed, k1, Xb.p);
        matvecs += r.steps * nu;
        matvecs64 += r.steps * nu;
        restarts += r.restarts;
        theta1 = r.theta;
        broken = r.broken;
        nconv1 = r.nconv;
        note_launches(L.launches);
    }
    // FP64 block map W = H(u_r) X for every Ritz vector of every parameter at once
    DevBuf<double> ud64;
    ud64.resize(NB);
    {
        std::vector<double> uh(NB, 0.0);
        for (int q = 0; q < nu; ++q) uh[q] = uv[q];
        MOMED_CUDA_TRY(cudaMemcpyAsync(ud64.p, uh.data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (int i = 0; i < k1; ++i) BlockMv<double2>::run(h, Xb.p + (size_t)i * stride, Wb.p + (size_t)i * stride, ud64.p, NB);
    matvecs += (int64_t)k1 * nu;
    matvecs64 += (int64_t)k1 * nu;
    std::vector<std::vector<double>> th(NB, std::vector<double>(k1, 0.0));
    for (int q = 0; q < nu; ++q)
        for (int i = 0; i < k1 && i < (int)theta1[q].size(); ++i) th[q][i] = theta1[q][i];
    const int eg = std::max(1, std::min<int>((int)((stride + 255) / 256), sms() * 8));
    if (mixed) {
        // Gram matrices G_r = X_r^H W_r and S_r = X_r^H X_r, all r at once
        const int grid = std::max(1, std::min<int>((int)((N + kRowsTile - 1) / kRowsTile), sms() * 2));
        DevBuf<double2> part, red;
        part.resize((size_t)grid * (kMaxCols + 1) * NB);
        red.resize((size_t)(kMaxCols + 1) * NB);
        std::vector<std::vector<std::complex<double>>> G(NB, std::vector<std::complex<double>>((size_t)k1 * k1)),
            S(NB, std::vector<std::complex<double>>((size_t)k1 * k1));
        std::vector<double2> hr((size_t)(k1 + 1) * NB);
        for (int pass = 0; pass < 2; ++pass) {
            for (int i = 0; i < k1; ++i) {
                const double2* rhs = (pass == 0 ? Wb.p : Xb.p) + (size_t)i * stride;
                k_bproj<double2, NB><<<grid, kT, 0, st>>>(Xb.p, N, k1, rhs, part.p, nullptr);
                k_breduce<NB><<<breduce_grid(k1 + 1, NB), 256, 0, st>>>(part.p, grid, k1 + 1, red.p, nullptr);
                note_launches(2);
                MOMED_CUDA_TRY(cudaMemcpyAsync(hr.data(), red.p, hr.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
                MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                for (int q = 0; q < nu; ++q)
                    for (int a = 0; a < k1; ++a)
                        (pass == 0 ? G : S)[q][(size_t)i * k1 + a] = std::complex<double>(hr[a * NB + q].x, hr[a * NB + q].y);
            }
        }
        std::vector<double2> Yh((size_t)NB * k1 * k1, make_double2(0.0, 0.0));
        for (int q = 0; q < NB; ++q)
            for (int i = 0; i < k1; ++i) Yh[((size_t)q * k1 + i) * k1 + i] = make_double2(1.0, 0.0);
        {
            std::vector<std::future<void>> fs;
            for (int q = 0; q < nu; ++q) {
                if (broken[q]) continue;
                fs.push_back(std::async(std::launch::async, [&, q]() {
                    std::vector<double> t;
                    std::vector<std::complex<double>> Y;
                    if (!gen_herm_eig(k1, G[q], S[q], t, Y)) { broken[q] = 1; return; }
                    th[q] = t;
                    for (int i = 0; i < k1; ++i)
                        for (int a = 0; a < k1; ++a) {
                            auto y = Y[(size_t)i * k1 + a];
                            Yh[((size_t)q * k1 + i) * k1 + a] = make_double2(y.real(), y.imag());
                        }
                }));
            }
            for (auto& f : fs) f.get();
        }
        DevBuf<double2> Yd;
        Yd.resize(Yh.size());
        MOMED_CUDA_TRY(cudaMemcpyAsync(Yd.p, Yh.data(), Yh.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
        k_bcombine_c<NB><<<eg, 256, 0, st>>>(Xb.p, N, k1, Yd.p, Sb.p);
        std::swap(Xb.p, Sb.p);
        k_bcombine_c<NB><<<eg, 256, 0, st>>>(Wb.p, N, k1, Yd.p, Sb.p);
        std::swap(Wb.p, Sb.p);
        note_launches(2);
        MOMED_CUDA_TRY(cudaGetLastError());
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    // residual norms ||W_i - theta_i X_i|| per (i, r) in FP64
    std::vector<std::vector<double>> rs(NB, std::vector<double>(k1, 0.0));
    {
        const int rg = std::max(1, std::min<int>((int)((stride + 255) / 256), 512));
        DevBuf<double> thd, part;
        thd.resize((size_t)NB * k1);
        part.resize((size_t)rg * k1 * NB);
        std::vector<double> thh((size_t)NB * k1, 0.0);
        for (int q = 0; q < nu; ++q)
            for (int i = 0; i < k1; ++i) thh[(size_t)q * k1 + i] = th[q][i];
        MOMED_CUDA_TRY(cudaMemcpyAsync(thd.p, thh.data(), thh.size() * 8, cudaMemcpyHostToDevice, st));
        k_bresid<NB><<<rg, 256, 0, st>>>(Wb.p, Xb.p, N, k1, thd.p, part.p);
        note_launches(1);
        MOMED_CUDA_TRY(cudaGetLastError());
        std::vector<double> hp((size_t)rg * k1 * NB);
        MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 8, cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        for (int q = 0; q < nu; ++q)
            for (int i = 0; i < k1; ++i) {
                double s = 0.0;
                for (int b = 0; b < rg; ++b) s += hp[((size_t)b * k1 + i) * NB + q];
                rs[q][i] = std::sqrt(s);
            }
    }
    // acceptance per parameter
    int converged_min = nev;
    DevBuf<double2> X1;
    X1.resize((size_t)std::max(k1, nev) * N);
    std::vector<int> okv(NB, 0), convv(NB, 0);
    for (int q = 0; q < nu; ++q) {
        int conv = 0;
        bool ok = !broken[q];
        if (ok) {
            double outside = (int)theta1[q].size() > k1 ? theta1[q][k1] : th[q][k1 - 1] + 1.0;
            for (int i = 0; i < nev; ++i) {
                bool good;
                if (mixed) {
                    double gap = std::fabs(outside - th[q][i]);
                    for (int j = 0; j < k1; ++j)
                        if (j != i && std::fabs(th[q][j] - th[q][i]) > 1e-9 * std::max(1.0, std::fabs(th[q][i])))
                            gap = std::min(gap, std::fabs(th[q][j] - th[q][i]));
                    double est = rs[q][i] * rs[q][i] / std::max(gap, 1e-300);
                    good = rs[q][i] <= tol || est <= kEigTarget * std::max(1.0, std::fabs(th[q][i]));
                } else {
                    good = i < nconv1[q] || rs[q][i] <= std::max(tol, 1e-10 * std::max(1.0, std::fabs(th[q][i])));
                }
                if (good && conv == i) ++conv;
                ok = ok && good;
            }
        }
        okv[q] = ok ? 1 : 0;
        convv[q] = conv;
    }
    // Parameters that missed the target are finished together: a lockstep FP64 block Lanczos
    // warm-started, per parameter, from the sum of its refined Ritz vectors.
    int nfail = 0;
    for (int q = 0; q < nu; ++q) nfail += (!okv[q] && !broken[q]) ? 1 : 0;
    DevBuf<double2> X3;
    std::vector<std::vector<double>> th3, rs3(NB, std::vector<double>(nev, 0.0));
    std::vector<int> nconv3(NB, 0), broken3(NB, 0);
    if (nfail > 0) {
        DevBuf<double2> v0;
        v0.resize((size_t)stride);
        k_bsum<NB><<<eg, 256, 0, st>>>(Xb.p, N, k1, v0.p);
        MOMED_CUDA_TRY(cudaGetLastError());
        X3.resize((size_t)nev * stride);
        BlockLanczos<double2, NB> L3(h, m, uv);
        auto r3 = L3.run(nev, nu, tol, 0.0, maxiter, o->seed, nev, X3.p, v0.p, kEigTarget);
        matvecs += r3.steps * nu;
        matvecs64 += r3.steps * nu;
        restarts += r3.restarts;
        note_launches(L3.launches + 1);
        th3 = r3.theta;
        nconv3 = r3.nconv;
        broken3 = r3.broken;
        // FP64 residuals of the phase-3 pairs
        for (int i = 0; i < nev; ++i)
            BlockMv<double2>::run(h, X3.p + (size_t)i * stride, Wb.p + (size_t)i * stride, ud64.p, NB);
        matvecs += (int64_t)nev * nu;
        matvecs64 += (int64_t)nev * nu;
        const int rg = std::max(1, std::min<int>((int)((stride + 255) / 256), 512));
        DevBuf<double> thd, part;
        thd.resize((size_t)NB * nev);
        part.resize((size_t)rg * nev * NB);
        std::vector<double> thh((size_t)NB * nev, 0.0);
        for (int q = 0; q < nu; ++q)
            for (int i = 0; i < nev; ++i) thh[(size_t)q * nev + i] = th3[q][i];
        MOMED_CUDA_TRY(cudaMemcpyAsync(thd.p, thh.data(), thh.size() * 8, cudaMemcpyHostToDevice, st));
        k_bresid<NB><<<rg, 256, 0, st>>>(Wb.p, X3.p, N, nev, thd.p, part.p);
        note_launches(1);
        MOMED_CUDA_TRY(cudaGetLastError());
        std::vector<double> hp((size_t)rg * nev * NB);
        MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 8, cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        for (int q = 0; q < nu; ++q)
            for (int i = 0; i < nev; ++i) {
                double s = 0.0;
                for (int b = 0; b < rg; ++b) s += hp[((size_t)b * nev + i) * NB + q];
                rs3[q][i] = std::sqrt(s);
            }
    }
    for (int q = 0; q < nu; ++q) {
        const bool from3 = !okv[q] && !broken[q] && !broken3[q];
        int conv = convv[q];
        if (from3) {
            k_extract<NB><<<eg, 256, 0, st>>>(X3.p, N, nev, q, X1.p);
        } else {
            k_extract<NB><<<eg, 256, 0, st>>>(Xb.p, N, k1, q, X1.p);
        }
        note_launches(1);
        MOMED_CUDA_TRY(cudaGetLastError());
        std::vector<double> tq(th[q].begin(), th[q].begin() + nev), rq(rs[q].begin(), rs[q].begin() + nev);
        if (from3) {
            tq.assign(th3[q].begin(), th3[q].begin() + nev);
            rq = rs3[q];
            conv = 0;
            while (conv < nev && (conv < nconv3[q] || rq[conv] <= tol)) ++conv;
        } else if (!okv[q]) {
            // invariant Krylov space: this parameter is solved on its own by the single-vector solver
            double uq = uv[q];
            float uf = (float)uq;
            MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &uq, sizeof(double), cudaMemcpyHostToDevice, st));
            MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &uf, sizeof(float), cudaMemcpyHostToDevice, st));
            momed_solve_opts o2 = *o;
            o2.precision = MOMED_PREC_FP64;
            o2.want_vectors = 1;
            o2.vecs_on_device = 1;
            momed_info i2{};
            momed_eigsolve_impl(h, &o2, nullptr, tq.data(), rq.data(), X1.p, &i2);
            matvecs += i2.matvecs;
            matvecs64 += i2.matvecs_fp64;
            restarts += i2.restarts;
            conv = i2.converged;
        }
        converged_min = std::min(converged_min, conv);
        for (int i = 0; i < nev; ++i) {
            vals[(size_t)q * nev + i] = tq[i];
            if (resid) resid[(size_t)q * nev + i] = rq[i];
        }
        if (vecs)
            MOMED_CUDA_TRY(cudaMemcpyAsync(vecs + (size_t)q * nev * N * 2, X1.p, (size_t)nev * N * sizeof(double2),
                                           cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    double one = 1.0;
    float onef = 1.0f;
    MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &one, sizeof(double), cudaMemcpyHostToDevice, st));
    MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &onef, sizeof(float), cudaMemcpyHostToDevice, st));
    MOMED_CUDA_TRY(cudaEventRecord(h->ev1, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (info) {
        info->converged = converged_min;
        info->restarts = restarts;
        info->matvecs = matvecs;
        info->matvecs_fp64 = matvecs64;
        info->seconds = ms * 1e-3;
    }
    return converged_min >= nev ? MOMED_OK : MOMED_ENOTCONV;
}

}  // namespace
}  // namespace momed

using namespace momed;

int momed_batch_solve_impl(momed_handle* h, const momed_solve_opts* o, const double* u, int32_t nu, double* vals,
                           double* resid, double* vecs, momed_info* info) {
    ensure_ready(h);
    MOMED_REQUIRE(h->op.has_b, MOMED_ESTATE, "batched solves need an operator pair (momed_set_scatter_pair)");
    MOMED_REQUIRE(nu >= 1 && nu <= 32, MOMED_EINVAL, "nu must be 1..32 per call");
    int nb = 1;
    while (nb < nu) nb <<= 1;
    switch (nb) {
        case 1: return run_batch<1>(h, o, u, nu, vals, resid, vecs, info);
        case 2: return run_batch<2>(h, o, u, nu, vals, resid, vecs, info);
        case 4: return run_batch<4>(h, o, u, nu, vals, resid, vecs, info);
        case 8: return run_batch<8>(h, o, u, nu, vals, resid, vecs, info);
        case 16: return run_batch<16>(h, o, u, nu, vals, resid, vecs, info);
        default: return run_batch<32>(h, o, u, nu, vals, resid, vecs, info);
    }
}
