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
#include <atomic>
#include <cstdlib>
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
constexpr int kTileElems = 2048;   // values of W (rows x right-hand sides) staged per tile in k_bproj
template <int NB> __host__ __device__ constexpr int rows_tile() { return kTileElems / NB; }
// Accepted eigenvalue error estimate (relative, r^2/gap) of the mixed-precision batch: 10x
// below the 1e-10 target.
constexpr double kEigTarget = 1e-11;
// Anchored refinement cycles of the mixed-precision batch before the FP64 block Lanczos takes over.
constexpr int kRefineCycles = 6;

__device__ __forceinline__ double2 to2(double2 v) { return v; }
__device__ __forceinline__ double2 to2(float2 v) { return make_double2(v.x, v.y); }
template <typename VT> __device__ __forceinline__ VT fr2(double2 v);
template <> __device__ __forceinline__ double2 fr2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 fr2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// 16-byte packets of a block vector: two c64 values (adjacent right-hand sides of one row) when
// NB is even, else one value.
template <typename VT, int NB> struct Pack {
    static constexpr int E = 1;
    using T = VT;
    static __device__ __forceinline__ void get(const T& p, double2* v) { v[0] = to2(p); }
    static __device__ __forceinline__ T put(const double2* v) { return fr2<VT>(v[0]); }
};
template <int NB> struct PackF2 {
    static constexpr int E = 2;
    using T = float4;
    static __device__ __forceinline__ void get(const float4& p, double2* v) {
        v[0] = make_double2(p.x, p.y);
        v[1] = make_double2(p.z, p.w);
    }
    static __device__ __forceinline__ float4 put(const double2* v) {
        return make_float4((float)v[0].x, (float)v[0].y, (float)v[1].x, (float)v[1].y);
    }
};
template <> struct Pack<float2, 2> : PackF2<2> {};
template <> struct Pack<float2, 4> : PackF2<4> {};
template <> struct Pack<float2, 8> : PackF2<8> {};
template <> struct Pack<float2, 16> : PackF2<16> {};
template <> struct Pack<float2, 32> : PackF2<32> {};

// partial[b][i][r] (i <= ncols: column ncols holds |w_r|^2).  Grid: x = row blocks, y = groups
// of 8 columns; warp w of group g owns column 8g + w over the block's rows, reading 16-byte
// packets of V (lanes: NB / E packets per row, 32 E / NB rows at a time) and the matching values
// of W straight from global memory (the block's 8 warps read the same rows of W, which L1
// serves), so there is no shared-memory staging and no barrier; the unrolled row loop keeps 8
// loads of V in flight per warp.  Warp 0 of group 0 also sums |w|^2.
template <typename VT, typename WT, int NB>
__global__ void __launch_bounds__(kT)
k_bproj(const VT* __restrict__ V, int64_t N, int ncols, const WT* __restrict__ W, double2* partial,
        const int* active_any) {
    if (active_any && *active_any == 0) return;
    using P = Pack<VT, NB>;
    constexpr int E = P::E;
    constexpr int PR = NB / E;                  // packets per row
    constexpr int RS = 32 / PR;                 // rows per warp pass
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int rp = lane % PR, rs = lane / PR;
    const int i = blockIdx.y * 8 + wid;
    const bool norm = blockIdx.y == 0 && wid == 0;
    if (i >= ncols && !norm) return;            // warp-uniform: this warp has no column
    double ax[E], ay[E], wn2[E];
#pragma unroll
    for (int q = 0; q < E; ++q) { ax[q] = 0.0; ay[q] = 0.0; wn2[q] = 0.0; }
    int64_t per = (N + gridDim.x - 1) / gridDim.x;
    int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(N, r0 + per);
    const typename P::T* col = reinterpret_cast<const typename P::T*>(V + (int64_t)(i < ncols ? i : 0) * N * NB);
    const WT* wr = W + rp * E;
    if (i < ncols) {
#pragma unroll 8
        for (int64_t t = r0 + rs; t < r1; t += RS) {
            double2 v[E];
            P::get(col[t * PR + rp], v);
#pragma unroll
            for (int q = 0; q < E; ++q) {
                const double2 w = to2(__ldg(wr + t * NB + q));
                ax[q] += v[q].x * w.x + v[q].y * w.y;
                ay[q] += v[q].x * w.y - v[q].y * w.x;
                if (norm) wn2[q] += w.x * w.x + w.y * w.y;
            }
        }
    } else {
        for (int64_t t = r0 + rs; t < r1; t += RS) {
#pragma unroll
            for (int q = 0; q < E; ++q) {
                const double2 w = to2(__ldg(wr + t * NB + q));
                wn2[q] += w.x * w.x + w.y * w.y;
            }
        }
    }
    double2* out = partial + (int64_t)blockIdx.x * (kMaxCols + 1) * NB;
#pragma unroll
    for (int q = 0; q < E; ++q) {
#pragma unroll
        for (int o = PR; o < 32; o <<= 1) {
            ax[q] += __shfl_xor_sync(0xffffffffu, ax[q], o);
            ay[q] += __shfl_xor_sync(0xffffffffu, ay[q], o);
            wn2[q] += __shfl_xor_sync(0xffffffffu, wn2[q], o);
        }
        if (rs == 0) {
            if (i < ncols) out[i * NB + rp * E + q] = make_double2(ax[q], ay[q]);
            if (norm) out[ncols * NB + rp * E + q] = make_double2(wn2[q], 0.0);
        }
    }
}

inline dim3 bproj_grid(int rowblocks, int ncols) { return dim3(rowblocks, (unsigned)std::max(1, (ncols + 7) / 8)); }

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

// W[n][r] -= sum_i coef[i][r] V_i[n][r] for active r; per-block |W_r|^2 partials.  A thread
// owns one 16-byte packet (E right-hand sides of a row) per grid-stride step; the unrolled
// column loop keeps 8 packet loads in flight.
template <typename VT, int NB>
__global__ void __launch_bounds__(kT)
k_bupdate(const VT* __restrict__ V, int64_t N, int ncols, const double2* __restrict__ coef, VT* __restrict__ W,
          double* npartial /* [grid][NB] */, const int* active /* [NB] or null */, const int* active_any) {
    if (active_any && *active_any == 0) return;
    using P = Pack<VT, NB>;
    using PT = typename P::T;
    constexpr int E = P::E;
    extern __shared__ double2 c[];   // [ncols * NB]
    __shared__ double nrm[32];
    for (int e = threadIdx.x; e < ncols * NB; e += kT) c[e] = coef[e];
    if (threadIdx.x < 32) nrm[threadIdx.x] = 0.0;
    __syncthreads();
    const int r0 = (threadIdx.x * E) % NB;     // fixed: the grid stride is a multiple of NB / E packets
    bool on[E];
    bool anyon = false;
#pragma unroll
    for (int q = 0; q < E; ++q) { on[q] = !active || active[r0 + q]; anyon = anyon || on[q]; }
    double wn2[E];
#pragma unroll
    for (int q = 0; q < E; ++q) wn2[q] = 0.0;
    const int64_t total = N * NB / E;           // packets per column
    const PT* Vp = reinterpret_cast<const PT*>(V);
    PT* Wp = reinterpret_cast<PT*>(W);
    for (int64_t e = (int64_t)blockIdx.x * kT + threadIdx.x; e < total; e += (int64_t)gridDim.x * kT) {
        double2 acc[E], orig[E];
        P::get(Wp[e], orig);
#pragma unroll
        for (int q = 0; q < E; ++q) acc[q] = orig[q];
        if (anyon) {
#pragma unroll 8
            for (int i = 0; i < ncols; ++i) {
                double2 v[E];
                P::get(Vp[(int64_t)i * total + e], v);
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const double2 cf = c[i * NB + r0 + q];
                    acc[q].x -= cf.x * v[q].x - cf.y * v[q].y;
                    acc[q].y -= cf.x * v[q].y + cf.y * v[q].x;
                }
            }
#pragma unroll
            for (int q = 0; q < E; ++q)
                if (!on[q]) acc[q] = orig[q];
            const PT st = P::put(acc);
            Wp[e] = st;
            P::get(st, acc);
        }
#pragma unroll
        for (int q = 0; q < E; ++q) wn2[q] += acc[q].x * acc[q].x + acc[q].y * acc[q].y;
    }
#pragma unroll
    for (int q = 0; q < E; ++q) atomicAdd(&nrm[r0 + q], wn2[q]);
    __syncthreads();
    if (threadIdx.x < NB) npartial[(int64_t)blockIdx.x * NB + threadIdx.x] = nrm[threadIdx.x];
}

// launched with NB warps: warp r reduces the norm partials of right-hand side r
template <int NB>
__global__ void k_bdecide(const double2* coefA, int ncols, const double* npartial, int grid, int* flag, int* any,
                          double* after, double keep_frac) {
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
        // second pass when less than keep_frac of the squared norm survived the first
        int f = (a < keep_frac * before) ? 1 : 0;
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

// out[i][n][r] = sum_a U[i][a][r] V[a][n][r]  (U: [nout][m][NB] real, r fastest so a warp's
// coefficient loads are coalesced), optionally out[nout] = V[copy_col].  Each thread owns RPT rows
// of one right-hand side and accumulates OC outputs at a time in registers of type ACC, streaming
// V straight from HBM (the unrolled a-loop keeps several loads in flight).  out must not overlap V.
template <typename VIN, typename VOUT, typename ACC, int NB, int RPT, int OC>
__global__ void __launch_bounds__(kT)
k_bcombine(const VIN* __restrict__ V, int64_t N, int m, const double* __restrict__ U, int nout,
           VOUT* __restrict__ out, int copy_col) {
    constexpr int TPR = kT / NB;        // row slots per block pass
    const int r = threadIdx.x % NB, slot = threadIdx.x / NB;
    const int64_t stride = N * NB;
    for (int64_t t0 = (int64_t)blockIdx.x * TPR * RPT; t0 < N; t0 += (int64_t)gridDim.x * TPR * RPT) {
        int64_t off[RPT];
        bool ok[RPT];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int64_t row = t0 + slot + (int64_t)j * TPR;
            ok[j] = row < N;
            off[j] = (ok[j] ? row : 0) * NB + r;
        }
        for (int c0 = 0; c0 < nout; c0 += OC) {
            ACC ax[RPT][OC], ay[RPT][OC];
#pragma unroll
            for (int j = 0; j < RPT; ++j)
#pragma unroll
                for (int k = 0; k < OC; ++k) { ax[j][k] = 0; ay[j][k] = 0; }
#pragma unroll 2
            for (int a = 0; a < m; ++a) {
                ACC u[OC];
#pragma unroll
                for (int k = 0; k < OC; ++k)
                    u[k] = (c0 + k < nout) ? (ACC)__ldg(U + ((int64_t)(c0 + k) * m + a) * NB + r) : (ACC)0;
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const VIN v = V[(int64_t)a * stride + off[j]];
#pragma unroll
                    for (int k = 0; k < OC; ++k) {
                        ax[j][k] += u[k] * (ACC)v.x;
                        ay[j][k] += u[k] * (ACC)v.y;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                if (!ok[j]) continue;
#pragma unroll
                for (int k = 0; k < OC; ++k)
                    if (c0 + k < nout)
                        out[(int64_t)(c0 + k) * stride + off[j]] = fr2<VOUT>(make_double2((double)ax[j][k], (double)ay[j][k]));
            }
        }
        if (copy_col >= 0) {
#pragma unroll
            for (int j = 0; j < RPT; ++j)
                if (ok[j]) out[(int64_t)nout * stride + off[j]] = fr2<VOUT>(to2(V[(int64_t)copy_col * stride + off[j]]));
        }
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
    static const int s = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();   // thread-safe first use (serving slots call concurrently)
    return s;
}

template <typename VT> struct BlockMv;
template <> struct BlockMv<float2> {
    static void run(momed_handle* h, const float2* x, float2* y, const float* u, int nb) {
        prof_begin(h);
        if (h->sparse.built) {   // the sparse method's entries (momed_build_sparse)
            launch_block_spmv_c64(h->sparse, x, y, h->op.has_b ? u : nullptr, nb, h->n, h->stream);
            prof_end(h, MOMED_KERNEL_BLOCK_SPMV_C64);
            return;
        }
        if (h->hcache.full()) {
            launch_block_hc_c64(h, x, y, u, nb, h->n, h->stream);
            prof_end(h, MOMED_KERNEL_HC_BLOCK_C64);
            return;
        }
        launch_block_matvec_c64(index_view(h), h->op.view(), x, y, u, nb, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_BLOCK_MATVEC_C64);
    }
};
template <> struct BlockMv<double2> {
    static void run(momed_handle* h, const double2* x, double2* y, const double* u, int nb) {
        prof_begin(h);
        if (h->hcache.full()) {
            launch_block_hc_c128(h, x, y, u, nb, h->n, h->stream);
            prof_end(h, MOMED_KERNEL_HC_BLOCK_C128);
            return;
        }
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
    int last_ugrid = 1;   // CTAs of the latest update: the count of its norm partials
    DevBuf<VT> V, V2;
    DevBuf<double2> partial, coefA, coefB;
    DevBuf<double> npart, after, scal, alpha, beta, Ud;
    DevBuf<int> flag, any;
    DevBuf<RT> ud;
    int64_t launches = 0;
    double dgks = 0.5;   // second Gram-Schmidt pass when |w'|^2 < dgks |w|^2 (set by run)
    // The steps of a restart cycle (k .. m-1) as one CUDA graph: captured the first time a cycle
    // starts at k on a given basis buffer (the restart alternates two), replayed afterwards.  A
    // step needs no host decision (the second Gram-Schmidt pass is predicated on a device flag),
    // so the cycle's ~12 launches per step go to the device as one graph launch.  The first
    // cycle runs eagerly (the block map's autotuner times its candidates there, outside capture).
    struct CycleGraph {
        int k;
        const VT* base;
        cudaGraphExec_t exec;
        int64_t kernels;
    };
    std::vector<CycleGraph> graphs;
    bool use_graphs = false;
    int64_t graph_replays = 0;

    ~BlockLanczos() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    }
    // steps [k, m): replayed from a captured graph when graphs are on, else launched one by one
    void cycle(int k, int64_t& steps) {
        steps += m - k;
        if (use_graphs) {
            for (auto& g : graphs)
                if (g.k == k && g.base == V.p) {
                    MOMED_CUDA_TRY(cudaGraphLaunch(g.exec, st));
                    note_launches(g.kernels);
                    ++graph_replays;
                    return;
                }
            // the graph's kernels: those its launchers note at once (the maps) plus those this
            // solver counts in `launches` (noted when the solve ends); other threads' launches
            // (serving slots) do not enter
            const int64_t l0 = launches_this_thread(), own0 = launches;
            cudaGraph_t graph = nullptr;
            MOMED_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            bool ok = true;
            try {
                for (int j = k; j < m; ++j) step(j);
            } catch (const Error&) {
                ok = false;
            }
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            cudaGraphExec_t exec = nullptr;
            if (ok && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                cudaGraphDestroy(graph);
                graphs.push_back({k, V.p, exec, (launches_this_thread() - l0) + (launches - own0)});
                MOMED_CUDA_TRY(cudaGraphLaunch(exec, st));
                ++graph_replays;
                return;
            }
            // capture refused: clear the error state and run this solve without graphs
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            use_graphs = false;
        }
        for (int j = k; j < m; ++j) step(j);
    }

    BlockLanczos(momed_handle* hh, int mm, const std::vector<double>& u) : h(hh), N(hh->n), m(mm), st(hh->stream) {
        {
            const char* e = std::getenv("MOMED_GRAPHS");
            use_graphs = !(e && e[0] == '0') && !hh->prof;   // per-launch timing needs eager launches
        }
        {   // kernel attributes are set before any capture
            constexpr size_t smem_max = (size_t)kMaxCols * NB * sizeof(double2);
            if (smem_max > 48 * 1024)
                MOMED_CUDA_TRY(cudaFuncSetAttribute(k_bupdate<VT, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)smem_max));
        }
        grid = std::max(1, std::min<int>((int)((N + rows_tile<NB>() - 1) / rows_tile<NB>()), sms() * 4));   // max row blocks
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
        // one full wave of resident CTAs over all column groups (measured: 1.5 waves left the
        // second half-wave's SMs idle at the end of every projection)
        static std::atomic<int> per_sm_cache{0};
        int per_sm = per_sm_cache.load(std::memory_order_relaxed);
        if (per_sm == 0) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bproj<VT, VT, NB>, kT, 0);
            if (per_sm <= 0) per_sm = 1;
            per_sm_cache.store(per_sm, std::memory_order_relaxed);
        }
        const int groups = std::max(1, (ncols + 7) / 8);
        int rb = std::max(1, per_sm * sms() / groups);
        rb = (int)std::min<int64_t>(rb, (N + rows_tile<NB>() - 1) / rows_tile<NB>());
        rb = std::max(1, std::min(rb, grid));
        k_bproj<VT, VT, NB><<<bproj_grid(rb, ncols), kT, 0, st>>>(V.p, N, ncols, w, partial.p, act);
        k_breduce<NB><<<breduce_grid(ncols + 1, NB), 256, 0, st>>>(partial.p, rb, ncols + 1, out, act);
        launches += 2;
    }
    void update(int ncols, const double2* coef, VT* w, const int* active, const int* act) {
        size_t smem = (size_t)ncols * NB * sizeof(double2);
        // one wave of resident CTAs (their count depends on the coefficients' shared memory); the
        // shared-memory attribute (process-wide, always the largest size) is set by the constructor
        static std::atomic<int> per_sm_cache[kMaxCols + 1];   // zero before first use (static storage)
        const int nc = std::min(std::max(ncols, 0), kMaxCols);
        int per_sm = per_sm_cache[nc].load(std::memory_order_relaxed);
        if (per_sm == 0) {
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_bupdate<VT, NB>, kT, smem);
            per_sm = std::max(b, 1);
            per_sm_cache[nc].store(per_sm, std::memory_order_relaxed);
        }
        const int g = std::max(1, std::min(ugrid, per_sm * sms()));
        k_bupdate<VT, NB><<<g, kT, smem, st>>>(V.p, N, ncols, coef, w, npart.p, active, act);
        ++launches;
        last_ugrid = g;
    }
    // column k0 made orthogonal to columns [0, k0) (two classical Gram-Schmidt passes), then normalised
    void orth_start(int k0) {
        VT* v = col(k0);
        for (int pass = 0; pass < 2 && k0 > 0; ++pass) {
            proj(k0, v, coefA.p, nullptr);
            update(k0, coefA.p, v, nullptr, nullptr);
        }
        normalize(v);
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
        k_bdecide<NB><<<1, NB * 32, 0, st>>>(coefA.p, nc, npart.p, last_ugrid, flag.p, any.p, after.p, dgks);
        ++launches;
        proj(nc, w, coefB.p, any.p);
        update(nc, coefB.p, w, flag.p, any.p);
        k_bfinalize<NB><<<1, NB * 32, 0, st>>>(coefA.p, coefB.p, nc, npart.p, last_ugrid, flag.p, any.p, after.p, scal.p,
                                          alpha.p, beta.p, j, m);
        k_bscale<VT, NB><<<ugrid, kT, 0, st>>>(w, N, scal.p);
        launches += 2;
    }
    template <typename VOUT>
    void combine(const std::vector<double>& Uh, int nout, VOUT* out, int copy_col, int mm) {
        MOMED_CUDA_TRY(cudaMemcpyAsync(Ud.p, Uh.data(), Uh.size() * 8, cudaMemcpyHostToDevice, st));
        // FP32 accumulation when FP32 vectors are recombined into FP32 vectors; FP64 otherwise
        constexpr bool f32 = std::is_same<VT, float2>::value && std::is_same<VOUT, float2>::value;
        using ACC = typename std::conditional<f32, float, double>::type;
        constexpr int RPT = f32 ? 4 : 2;
        constexpr int TR = (kT / NB) * RPT;
        // (one pass of 16 outputs and 2 rows per thread for 9..16 outputs was slower: 1.61 against
        // 1.21 ms for the headline restart's 12)
        auto k = k_bcombine<VT, VOUT, ACC, NB, RPT, 8>;
        int g = (int)std::max<int64_t>(1, std::min<int64_t>((N + TR - 1) / TR, (int64_t)sms() * 8));
        k<<<g, kT, 0, st>>>(V.p, N, mm, Ud.p, nout, out, copy_col);
        MOMED_CUDA_TRY(cudaGetLastError());
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        ++launches;
    }
    // restart: the kept combinations (and column m) go to V2, which then becomes the basis
    void recombine(const std::vector<double>& Uh, int keep) {
        V2.resize((size_t)(m + 1) * N * NB);
        combine<VT>(Uh, keep, V2.p, m, m);
        std::swap(V.p, V2.p);
        std::swap(V.n, V2.n);
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
        // The classical 1/2 (|w'| < 0.71 |w|) flags nearly every Lanczos step, because w = H v
        // carries alpha and beta along the two newest columns, and one flagged right-hand side
        // makes the whole block repeat the pass.  Measured on B200: with FP64 bases, or few
        // wanted pairs (nev <= m/5), 0.1 runs the same maps and gives the same eigenvalues as
        // 1/2 (3x9, 32 U0, nev 4: 16% faster; 0.01 the same); an FP32 basis with nev 12 in m 36
        // needed 1.65x the maps at 0.1, so FP32 with more wanted pairs keeps 1/2.
        dgks = (std::is_same<VT, float2>::value && 5 * nev > m) ? 0.5 : 0.1;
        // graphs captured by an earlier run of this object carry that run's dgks: capture anew
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
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
            if (restarts == 0) {
                for (int j = k; j < m; ++j) { step(j); ++steps; }
            } else {
                cycle(k, steps);
            }
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
            // Few wanted pairs (nev <= m/5) keep a third of the spare dimension beyond nev: measured
            // on B200 at m 30, nev 4, 12 kept beat 10, 15, 20 and (3m + 2 nconv)/5 by 5-13%.  More
            // wanted pairs keep (3m + 2 nconv)/5: at m 36, nev 12 a third of the spare dimension
            // (20 kept) needed 1.7x the maps, and at nev 15-20 it was 0-3% slower.
            int keep = 5 * nev <= m ? nev + (m - nev) / 3 : (3 * m + 2 * minconv) / 5;
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
            recombine(Uh, keep);
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

// out[n][r] = sum_{i<k} wt[r][i] (W[i][n][r] - th[r][i] X[i][n][r])  (start of the refinement)
template <typename VT, int NB>
__global__ void k_bresid_sum(const double2* __restrict__ W, const double2* __restrict__ X, int64_t N, int k,
                             const double* __restrict__ th, const double* __restrict__ wt, VT* __restrict__ out) {
    const int64_t total = N * NB;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % NB);
        double sx = 0.0, sy = 0.0;
        for (int i = 0; i < k; ++i) {
            const double c = wt[r * k + i];
            if (c == 0.0) continue;
            const double t = th[r * k + i];
            const double2 w = W[(int64_t)i * total + e], x = X[(int64_t)i * total + e];
            sx += c * (w.x - t * x.x);
            sy += c * (w.y - t * x.y);
        }
        out[e] = fr2<VT>(make_double2(sx, sy));
    }
}

// out[e] = (VT) X[e] over a flat range
template <typename VT>
__global__ void k_bto(const double2* __restrict__ X, int64_t total, VT* __restrict__ out) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = fr2<VT>(X[e]);
}

// out[i][n][r] = sum_{a<kx} Y[i][a][r] X[a][n][r] + sum_{b<kz} Y[i][kx+b][r] Z[b][n][r]
//               + sum_{j<p} Y[i][kx+kz+j][r] Q[j][n][r]
// (Y complex, [(i * (kx + kz + p) + a) * NB + r]; FP64 sources X and Z, FP32 source Q; FP64 out).
// A thread owns RPT rows of one right-hand side, so each coefficient load serves RPT rows.
template <int NB>
__global__ void __launch_bounds__(kT, 2)
k_bcombine_xq(const double2* __restrict__ X, int kx, const double2* __restrict__ Z, int kz,
              const float2* __restrict__ Q, int p, int64_t N, const double2* __restrict__ Y, int nout,
              double2* __restrict__ out) {
    constexpr int OC = 8, RPT = 2;
    constexpr int TPR = kT / NB;        // row slots per block pass
    const int d = kx + kz + p;
    const int64_t stride = N * NB;
    const int r = threadIdx.x % NB, slot = threadIdx.x / NB;
    for (int64_t t0 = (int64_t)blockIdx.x * TPR * RPT; t0 < N; t0 += (int64_t)gridDim.x * TPR * RPT) {
        int64_t off[RPT];
        bool ok[RPT];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int64_t row = t0 + slot + (int64_t)j * TPR;
            ok[j] = row < N;
            off[j] = (ok[j] ? row : 0) * NB + r;
        }
        for (int c0 = 0; c0 < nout; c0 += OC) {
            double ax[RPT][OC], ay[RPT][OC];
#pragma unroll
            for (int j = 0; j < RPT; ++j)
#pragma unroll
                for (int k = 0; k < OC; ++k) { ax[j][k] = 0.0; ay[j][k] = 0.0; }
            {
                // the FP32 extension Q in FP32 arithmetic (its values carry FP32 rounding already;
                // the products add an error of the same order), summed into the FP64 sums after
                float fx[RPT][OC], fy[RPT][OC];
#pragma unroll
                for (int j = 0; j < RPT; ++j)
#pragma unroll
                    for (int k = 0; k < OC; ++k) { fx[j][k] = 0.f; fy[j][k] = 0.f; }
                for (int a = kx + kz; a < d; ++a) {
                    float2 y[OC];
#pragma unroll
                    for (int k = 0; k < OC; ++k) {
                        const double2 yd = (c0 + k < nout) ? __ldg(Y + ((int64_t)(c0 + k) * d + a) * NB + r)
                                                           : make_double2(0.0, 0.0);
                        y[k] = make_float2((float)yd.x, (float)yd.y);
                    }
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        const float2 v = Q[(int64_t)(a - kx - kz) * stride + off[j]];
#pragma unroll
                        for (int k = 0; k < OC; ++k) {
                            fx[j][k] += y[k].x * v.x - y[k].y * v.y;
                            fy[j][k] += y[k].x * v.y + y[k].y * v.x;
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < RPT; ++j)
#pragma unroll
                    for (int k = 0; k < OC; ++k) { ax[j][k] = (double)fx[j][k]; ay[j][k] = (double)fy[j][k]; }
            }
            for (int a = 0; a < kx + kz; ++a) {            // the FP64 anchors X (and Z)
                double2 y[OC];
#pragma unroll
                for (int k = 0; k < OC; ++k)
                    y[k] = (c0 + k < nout) ? __ldg(Y + ((int64_t)(c0 + k) * d + a) * NB + r) : make_double2(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const double2 v = a < kx ? X[(int64_t)a * stride + off[j]] : Z[(int64_t)(a - kx) * stride + off[j]];
#pragma unroll
                    for (int k = 0; k < OC; ++k) {
                        ax[j][k] += y[k].x * v.x - y[k].y * v.y;
                        ay[j][k] += y[k].x * v.y + y[k].y * v.x;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                if (!ok[j]) continue;
#pragma unroll
                for (int k = 0; k < OC; ++k)
                    if (c0 + k < nout) out[(int64_t)(c0 + k) * stride + off[j]] = make_double2(ax[j][k], ay[j][k]);
            }
        }
    }
}


// Inner products of ncols columns of V with up to kGramRhs right-hand-side blocks at once:
// partial[b][j][i][r] = block's sum over rows of conj(V_i[n][r]) R_j[n][r].  Grid: x = row blocks,
// y = groups of 8 columns (warp per column, as in k_bproj); every column packet read from HBM
// serves all right-hand sides, which the block's warps share through L1.
constexpr int kGramRhs = 4;
struct GramRhs {
    const double2* p[kGramRhs];
};
template <typename VT, int NB>
__global__ void __launch_bounds__(kT, 4)
k_bgram(const VT* __restrict__ V, int64_t N, int ncols, GramRhs R, int nr, double2* __restrict__ partial) {
    using P = Pack<VT, NB>;
    constexpr int E = P::E;
    constexpr int PR = NB / E;
    constexpr int RS = 32 / PR;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int rp = lane % PR, rs = lane / PR;
    const int i = blockIdx.y * 8 + wid;
    if (i >= ncols) return;                     // warp-uniform
    double ax[kGramRhs][E], ay[kGramRhs][E];
#pragma unroll
    for (int j = 0; j < kGramRhs; ++j)
#pragma unroll
        for (int q = 0; q < E; ++q) { ax[j][q] = 0.0; ay[j][q] = 0.0; }
    const int64_t per = (N + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(N, r0 + per);
    const typename P::T* col = reinterpret_cast<const typename P::T*>(V + (int64_t)i * N * NB);
#pragma unroll 2
    for (int64_t t = r0 + rs; t < r1; t += RS) {
        double2 v[E];
        P::get(col[t * PR + rp], v);
#pragma unroll
        for (int j = 0; j < kGramRhs; ++j) {
            if (j < nr) {
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const double2 w = __ldg(R.p[j] + t * NB + rp * E + q);
                    ax[j][q] += v[q].x * w.x + v[q].y * w.y;
                    ay[j][q] += v[q].x * w.y - v[q].y * w.x;
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kGramRhs; ++j) {
#pragma unroll
        for (int q = 0; q < E; ++q) {
            double sx = ax[j][q], sy = ay[j][q];
#pragma unroll
            for (int o = PR; o < 32; o <<= 1) {
                sx += __shfl_xor_sync(0xffffffffu, sx, o);
                sy += __shfl_xor_sync(0xffffffffu, sy, o);
            }
            if (j < nr && rs == 0)
                partial[(((int64_t)blockIdx.x * kGramRhs + j) * ncols + i) * NB + rp * E + q] = make_double2(sx, sy);
        }
    }
}

// Row blocks of k_bgram: one wave of the CTAs that are resident at once over the ncols / 8
// column groups (measured: a grid of 0.67 or 3 waves left the SMs a third idle or ran a partial
// last wave), at least one row tile each, at most cap.
constexpr int kGramBlocksPerSm = 8;
template <int NB>
int gram_rowblocks_t(int64_t N, int ncols, bool fp32, int cap) {
    static std::atomic<int> per_sm[2];   // zero before first use (static storage)
    int ps = per_sm[fp32 ? 1 : 0].load(std::memory_order_relaxed);
    if (ps == 0) {
        if (fp32) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, k_bgram<float2, NB>, kT, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, k_bgram<double2, NB>, kT, 0);
        if (ps <= 0) ps = 1;
        per_sm[fp32 ? 1 : 0].store(ps, std::memory_order_relaxed);
    }
    int sm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    if (sm <= 0) sm = 148;
    const int groups = std::max(1, (ncols + 7) / 8);
    int rb = std::max(1, ps * sm / groups);
    rb = (int)std::min<int64_t>(rb, (N + rows_tile<NB>() - 1) / rows_tile<NB>());
    return std::max(1, std::min(rb, cap));
}

// out[e] = sum over blocks b < grid of partial[b * bstride + e] for e < count, one warp per
// element (fixed order)
__global__ void k_bsum_blocks(const double2* __restrict__ partial, int grid, int64_t bstride, int64_t count,
                              double2* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= count) return;
    double sx = 0.0, sy = 0.0;
    for (int b = lane; b < grid; b += 32) {
        const double2 v = partial[(int64_t)b * bstride + e];
        sx += v.x;
        sy += v.y;
    }
    sx = wsum(sx);
    sy = wsum(sy);
    if (lane == 0) out[e] = make_double2(sx, sy);
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
    const double u_handle = h->u;
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
        const int grid = std::max(1, std::min<int>((int)((N + rows_tile<NB>() - 1) / rows_tile<NB>()), sms() * 2));
        DevBuf<double2> part, red;
        part.resize((size_t)grid * (kMaxCols + 1) * NB);
        red.resize((size_t)(kMaxCols + 1) * NB);
        std::vector<std::vector<std::complex<double>>> G(NB, std::vector<std::complex<double>>((size_t)k1 * k1)),
            S(NB, std::vector<std::complex<double>>((size_t)k1 * k1));
        std::vector<double2> hr((size_t)(k1 + 1) * NB);
        for (int pass = 0; pass < 2; ++pass) {
            for (int i = 0; i < k1; ++i) {
                const double2* rhs = (pass == 0 ? Wb.p : Xb.p) + (size_t)i * stride;
                k_bproj<double2, double2, NB><<<bproj_grid(grid, k1), kT, 0, st>>>(Xb.p, N, k1, rhs, part.p, nullptr);
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
    // Mixed precision, parameters that missed the target: anchored refinement.  The FP64 Ritz
    // vectors X (with W = H X from the FP64 map) anchor a subspace that an FP32 Lanczos extends,
    // starting from their residuals.  Rayleigh-Ritz on [X, Q] takes X^H H X, X^H X, X^H H Q =
    // W^H Q and X^H Q from FP64 data and only Q^H H Q from the FP32 recurrence; an error e there
    // moves an eigenvalue by about |y_Q|^2 e, where y_Q (the correction's weight) is of the size
    // of the residual over the gap.  W is recomputed with the FP64 map each cycle, so the
    // residuals and the acceptance test are exact.  Parameters still failing after the cycles
    // go on to the FP64 block Lanczos below.
    if (mixed && m - k1 >= 4) {
        auto failing = [&]() {
            int c = 0;
            for (int q = 0; q < nu; ++q) c += (!okv[q] && !broken[q]) ? 1 : 0;
            return c;
        };
        if (failing() > 0) {
            const int p = m - k1, d = k1 + p;
            const int d2 = 2 * k1 + p + 1;     // sources of W': W, X, Q and the next Lanczos vector
            BlockLanczos<float2, NB> LR(h, m, uv);
            LR.dgks = 5 * nev > m ? 0.5 : 0.1;   // the rule of BlockLanczos::run for an FP32 basis
            DevBuf<double> thd, wtd;
            thd.resize((size_t)NB * k1);
            wtd.resize((size_t)NB * k1);
            DevBuf<double2> Yd, Y2d, W2;
            Yd.resize((size_t)k1 * d * NB);
            Y2d.resize((size_t)k1 * d2 * NB);
            W2.resize((size_t)k1 * stride);
            // Gram partials [row block][kGramRhs][columns][NB] and the summed blocks [2 k1][columns][NB]
            DevBuf<double2> gpart, gx, gq;
            // Gram row blocks: one wave of resident CTAs over all column groups (occupancy of
            // k_bgram), up to kGramBlocksPerSm per SM; the partial buffer holds that many
            const int gram_cap = kGramBlocksPerSm * sms();
            gpart.resize((size_t)gram_cap * kGramRhs * std::max(k1, m - k1) * NB);
            const size_t gx_n = (size_t)2 * k1 * k1 * NB, gq_n = (size_t)2 * k1 * (m - k1) * NB;
            gx.resize(gx_n);
            gq.resize(gq_n);
            std::vector<int> failed(NB, 0);
            std::vector<std::vector<double>> last_t(NB);   // full Ritz spectrum of the last cycle
            const int rg = std::max(1, std::min<int>((int)((stride + 255) / 256), 512));
            DevBuf<double> part;
            part.resize((size_t)rg * k1 * NB);
            // residual norms ||W_i - th_i X_i|| of every (i, q) into rs
            auto residuals = [&]() {
                std::vector<double> thn((size_t)NB * k1, 0.0);
                for (int q = 0; q < nu; ++q)
                    for (int i = 0; i < k1; ++i) thn[(size_t)q * k1 + i] = th[q][i];
                MOMED_CUDA_TRY(cudaMemcpyAsync(thd.p, thn.data(), thn.size() * 8, cudaMemcpyHostToDevice, st));
                k_bresid<NB><<<rg, 256, 0, st>>>(Wb.p, Xb.p, N, k1, thd.p, part.p);
                note_launches(1);
                MOMED_CUDA_TRY(cudaGetLastError());
                std::vector<double> hp((size_t)rg * k1 * NB);
                MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 8, cudaMemcpyDeviceToHost, st));
                MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                for (int q = 0; q < nu; ++q)
                    for (int i = 0; i < k1; ++i) {
                        double s2 = 0.0;
                        for (int b = 0; b < rg; ++b) s2 += hp[((size_t)b * k1 + i) * NB + q];
                        rs[q][i] = std::sqrt(s2);
                    }
            };
            // acceptance of parameter q from its Ritz spectrum t and rs; margin < 1 asks for more
            auto accept = [&](int q, const std::vector<double>& t, double margin) {
                int conv = 0;
                bool ok = true;
                for (int i = 0; i < nev; ++i) {
                    double gap = 1e300;
                    for (int j = 0; j < (int)t.size(); ++j)
                        if (j != i && std::fabs(t[j] - t[i]) > 1e-9 * std::max(1.0, std::fabs(t[i])))
                            gap = std::min(gap, std::fabs(t[j] - t[i]));
                    const double est = rs[q][i] * rs[q][i] / std::max(gap, 1e-300);
                    const bool good = rs[q][i] <= margin * tol ||
                                      est <= margin * kEigTarget * std::max(1.0, std::fabs(t[i]));
                    if (good && conv == i) ++conv;
                    ok = ok && good;
                }
                convv[q] = conv;
                okv[q] = ok ? 1 : 0;
            };
            int cycles = 0;
            for (int cyc = 0; cyc < kRefineCycles && failing() > 0; ++cyc) {
                ++cycles;
                // anchors and start vector (weighted residuals of the pairs not yet accepted)
                k_bto<float2><<<eg, 256, 0, st>>>(Xb.p, (int64_t)k1 * stride, LR.col(0));
                std::vector<double> thh((size_t)NB * k1, 0.0), wth((size_t)NB * k1, 0.0);
                for (int q = 0; q < nu; ++q) {
                    for (int i = 0; i < k1; ++i) thh[(size_t)q * k1 + i] = th[q][i];
                    int used = 0;
                    for (int i = convv[q]; i < nev; ++i)
                        if (rs[q][i] > 0.0) { wth[(size_t)q * k1 + i] = std::sqrt(i + 1.0) / rs[q][i]; ++used; }
                    if (!used)
                        for (int i = 0; i < nev; ++i)
                            if (rs[q][i] > 0.0) wth[(size_t)q * k1 + i] = std::sqrt(i + 1.0) / rs[q][i];
                }
                MOMED_CUDA_TRY(cudaMemcpyAsync(thd.p, thh.data(), thh.size() * 8, cudaMemcpyHostToDevice, st));
                MOMED_CUDA_TRY(cudaMemcpyAsync(wtd.p, wth.data(), wth.size() * 8, cudaMemcpyHostToDevice, st));
                k_bresid_sum<float2, NB><<<eg, 256, 0, st>>>(Wb.p, Xb.p, N, k1, thd.p, wtd.p, LR.col(k1));
                note_launches(2);
                MOMED_CUDA_TRY(cudaGetLastError());
                LR.orth_start(k1);
                for (int j = k1; j < m; ++j) LR.step(j);
                matvecs += (int64_t)p * nu;
                std::vector<double> ha((size_t)NB * m), hb((size_t)NB * m);
                MOMED_CUDA_TRY(cudaMemcpyAsync(ha.data(), LR.alpha.p, ha.size() * 8, cudaMemcpyDeviceToHost, st));
                MOMED_CUDA_TRY(cudaMemcpyAsync(hb.data(), LR.beta.p, hb.size() * 8, cudaMemcpyDeviceToHost, st));
                // FP64 Gram blocks: b_a^H H b_i and b_a^H b_i for the anchors i against [X, Q]
                std::vector<std::vector<std::complex<double>>> G(NB, std::vector<std::complex<double>>((size_t)d * d)),
                    S(NB, std::vector<std::complex<double>>((size_t)d * d));
                // FP64 Gram blocks: b_a^H H b_i and b_a^H b_i for the anchors i against [X, Q]; the
                // 2 k1 right-hand sides (W_i, then X_i) go kGramRhs at a time
                const int nrhs = 2 * k1;
                auto gram = [&](const void* cols, bool fp32, int ncols, int g0, int nr, double2* out) {
                    const int rb = gram_rowblocks_t<NB>(N, ncols, fp32, gram_cap);
                    GramRhs R{};
                    for (int j = 0; j < nr; ++j)
                        R.p[j] = (g0 + j < k1 ? Wb.p + (size_t)(g0 + j) * stride : Xb.p + (size_t)(g0 + j - k1) * stride);
                    for (int j = nr; j < kGramRhs; ++j) R.p[j] = R.p[0];
                    if (fp32)
                        k_bgram<float2, NB><<<bproj_grid(rb, ncols), kT, 0, st>>>(
                            reinterpret_cast<const float2*>(cols), N, ncols, R, nr, gpart.p);
                    else
                        k_bgram<double2, NB><<<bproj_grid(rb, ncols), kT, 0, st>>>(
                            reinterpret_cast<const double2*>(cols), N, ncols, R, nr, gpart.p);
                    // the nr valid slabs lead each block's [kGramRhs][ncols][NB] partials
                    const int64_t bstride = (int64_t)kGramRhs * ncols * NB, count = (int64_t)nr * ncols * NB;
                    k_bsum_blocks<<<(unsigned)((count + 7) / 8), 256, 0, st>>>(gpart.p, rb, bstride, count, out);
                    note_launches(2);
                };
                for (int g0 = 0; g0 < nrhs; g0 += kGramRhs) {
                    const int nr = std::min(kGramRhs, nrhs - g0);
                    gram(Xb.p, false, k1, g0, nr, gx.p + (size_t)g0 * k1 * NB);          // x_a^H rhs
                    gram(LR.col(k1), true, p, g0, nr, gq.p + (size_t)g0 * p * NB);       // q_j^H rhs
                }
                std::vector<double2> hx((size_t)gx_n), hq((size_t)gq_n);
                MOMED_CUDA_TRY(cudaMemcpyAsync(hx.data(), gx.p, hx.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
                MOMED_CUDA_TRY(cudaMemcpyAsync(hq.data(), gq.p, hq.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
                MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                for (int jr = 0; jr < nrhs; ++jr) {
                    const int i = jr < k1 ? jr : jr - k1;
                    auto& M = jr < k1 ? G : S;
                    const double2* bx = hx.data() + (size_t)jr * k1 * NB;
                    const double2* bq = hq.data() + (size_t)jr * p * NB;
                    for (int q = 0; q < nu; ++q) {
                        for (int a = 0; a < k1; ++a)
                            M[q][(size_t)i * d + a] = std::complex<double>(bx[a * NB + q].x, bx[a * NB + q].y);
                        for (int j = 0; j < p; ++j) {
                            std::complex<double> v(bq[j * NB + q].x, bq[j * NB + q].y);
                            M[q][(size_t)i * d + k1 + j] = v;
                            M[q][(size_t)(k1 + j) * d + i] = std::conj(v);
                        }
                    }
                }
                std::vector<double2> Yh((size_t)k1 * d * NB, make_double2(0.0, 0.0));
                std::vector<double2> Y2h((size_t)k1 * d2 * NB, make_double2(0.0, 0.0));
                std::vector<std::vector<double>> tq(NB);
                std::vector<int> ok_rr(NB, 0);
                {
                    std::vector<std::future<void>> fs;
                    for (int q = 0; q < nu; ++q) {
                        if (broken[q] || failed[q]) continue;
                        fs.push_back(std::async(std::launch::async, [&, q]() {
                            double tmax = 0.0;
                            for (int i = 0; i < k1; ++i) tmax = std::max(tmax, std::fabs(th[q][i]));
                            for (int j = 0; j < p; ++j) {
                                const double a = ha[(size_t)q * m + k1 + j];
                                G[q][(size_t)(k1 + j) * d + k1 + j] = a;
                                S[q][(size_t)(k1 + j) * d + k1 + j] = 1.0;
                                tmax = std::max(tmax, std::fabs(a));
                                if (j + 1 < p) {
                                    const double b = hb[(size_t)q * m + k1 + j];
                                    G[q][(size_t)(k1 + j) * d + k1 + j + 1] = b;
                                    G[q][(size_t)(k1 + j + 1) * d + k1 + j] = b;
                                }
                            }
                            for (int j = 0; j + 1 < p; ++j)
                                if (hb[(size_t)q * m + k1 + j] <= 1e-12 * std::max(tmax, 1.0)) return;   // invariant
                            std::vector<double> t;
                            std::vector<std::complex<double>> Y;
                            if (!gen_herm_eig(d, G[q], S[q], t, Y)) return;
                            for (int i = 0; i < k1; ++i)
                                for (int a = 0; a < d; ++a) {
                                    const auto y = Y[(size_t)i * d + a];
                                    Yh[((size_t)i * d + a) * NB + q] = make_double2(y.real(), y.imag());
                                }
                            // W' = H X' = W Y_X + X (C Y_Q) + Q (T Y_Q) + q_p beta_last (Y_Q)_last, with
                            // C = X^H H Q exact (from W) and T the FP32 recurrence
                            auto put2 = [&](int i, int a, std::complex<double> v) {
                                Y2h[((size_t)i * d2 + a) * NB + q] = make_double2(v.real(), v.imag());
                            };
                            const double blast = hb[(size_t)q * m + m - 1];
                            for (int i = 0; i < k1; ++i) {
                                const std::complex<double>* yq = &Y[(size_t)i * d + k1];
                                for (int a = 0; a < k1; ++a) put2(i, a, Y[(size_t)i * d + a]);
                                for (int b = 0; b < k1; ++b) {
                                    std::complex<double> c = 0.0;
                                    for (int j = 0; j < p; ++j) c += G[q][(size_t)(k1 + j) * d + b] * yq[j];
                                    put2(i, k1 + b, c);
                                }
                                for (int l = 0; l < p; ++l) {
                                    std::complex<double> c = ha[(size_t)q * m + k1 + l] * yq[l];
                                    if (l > 0) c += hb[(size_t)q * m + k1 + l - 1] * yq[l - 1];
                                    if (l + 1 < p) c += hb[(size_t)q * m + k1 + l] * yq[l + 1];
                                    put2(i, 2 * k1 + l, c);
                                }
                                put2(i, 2 * k1 + p, blast * yq[p - 1]);
                            }
                            tq[q] = t;
                            ok_rr[q] = 1;
                        }));
                    }
                    for (auto& f : fs) f.get();
                }
                for (int q = 0; q < NB; ++q) {
                    if (ok_rr[q]) continue;
                    if (q < nu && !okv[q]) failed[q] = 1;     // left to the FP64 block Lanczos
                    for (int i = 0; i < k1; ++i) {
                        Yh[((size_t)i * d + i) * NB + q] = make_double2(1.0, 0.0);
                        Y2h[((size_t)i * d2 + i) * NB + q] = make_double2(1.0, 0.0);
                    }
                }
                MOMED_CUDA_TRY(cudaMemcpyAsync(Yd.p, Yh.data(), Yh.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
                MOMED_CUDA_TRY(cudaMemcpyAsync(Y2d.p, Y2h.data(), Y2h.size() * sizeof(double2), cudaMemcpyHostToDevice,
                                               st));
                // X' = [X Q] Y and W' from the Lanczos relation (both read the old X and W)
                const int xg = std::max(1, std::min<int>((int)((N + 2 * (kT / NB) - 1) / (2 * (kT / NB))), sms() * 8));
                k_bcombine_xq<NB><<<xg, kT, 0, st>>>(Xb.p, k1, nullptr, 0, LR.col(k1), p, N, Yd.p, k1, Sb.p);
                k_bcombine_xq<NB><<<xg, kT, 0, st>>>(Wb.p, k1, Xb.p, k1, LR.col(k1), p + 1, N, Y2d.p, k1, W2.p);
                note_launches(2);
                MOMED_CUDA_TRY(cudaGetLastError());
                std::swap(Xb.p, Sb.p);
                std::swap(Wb.p, W2.p);
                for (int q = 0; q < nu; ++q)
                    if (ok_rr[q]) {
                        for (int i = 0; i < k1; ++i) th[q][i] = tq[q][i];
                        last_t[q] = tq[q];
                    }
                // residuals from W' (accurate to the FP32 error times |y_Q|) and acceptance with
                // a margin; the exact FP64 check follows the loop
                residuals();
                for (int q = 0; q < nu; ++q)
                    if (!okv[q] && !broken[q] && ok_rr[q]) accept(q, tq[q], 0.5);
                note_launches(LR.launches);
                LR.launches = 0;
            }
            if (cycles > 0) {
                // exact W = H X with the FP64 map for the nev wanted vectors (the acceptance reads
                // their residuals; the other anchors enter only through the Ritz values' gaps and
                // keep W' from the Lanczos relation), exact residuals, final acceptance
                for (int i = 0; i < nev; ++i)
                    BlockMv<double2>::run(h, Xb.p + (size_t)i * stride, Wb.p + (size_t)i * stride, ud64.p, NB);
                matvecs += (int64_t)nev * nu;
                matvecs64 += (int64_t)nev * nu;
                residuals();
                for (int q = 0; q < nu; ++q)
                    if (!broken[q] && !last_t[q].empty()) accept(q, last_t[q], 1.0);
            }
        }
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
            // (at its u: the handle's u, host and device, is put back below)
            double uq = uv[q];
            float uf = (float)uq;
            h->u = uq;
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
                                           o->vecs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }
    // the handle's own u (momed_set_param) again on the device
    h->u = u_handle;
    const float u32 = (float)u_handle;
    MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &u_handle, sizeof(double), cudaMemcpyHostToDevice, st));
    MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &u32, sizeof(float), cudaMemcpyHostToDevice, st));
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
    if (!h->sparse.built) ensure_hit_cache(h);
    // without a second operator (momed_set_scatter) every parameter solves H = A
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
