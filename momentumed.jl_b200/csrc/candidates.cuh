// Candidate-term machinery shared by the matrix-free maps (matvec.cu) and the device build of
// the sparse matrix (sparse.cu): for a row state s, the term groups whose creation mask lies in
// s are found by table lookup on its occupied orbitals and orbital pairs, their terms are
// flattened and dealt to the 32 lanes of the row's warp, and each lane evaluates one term
// (mask test, fermionic sign, index of the target state).
#pragma once
#include <algorithm>

#include "index.cuh"

namespace momed {

namespace {

constexpr int kWarps = 8;          // warps per block (256 threads)
constexpr unsigned kFull = 0xffffffffu;

template <typename R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };

struct WarpScratch {
    uint64_t out[32];
    int32_t start[32];
    int32_t pref[33];
};

__device__ __forceinline__ double2 load_amp(const double2* p, int t) { return __ldg(p + t); }
__device__ __forceinline__ float2 load_amp(const float2* p, int t) { return __ldg(p + t); }

template <typename R> __device__ __forceinline__ const typename Cx<R>::T* amp_a(const OpView& ov);
template <> __device__ __forceinline__ const double2* amp_a<double>(const OpView& ov) { return ov.t_amp; }
template <> __device__ __forceinline__ const float2* amp_a<float>(const OpView& ov) { return ov.t_amp32; }
template <typename R> __device__ __forceinline__ const typename Cx<R>::T* amp_b(const OpView& ov);
template <> __device__ __forceinline__ const double2* amp_b<double>(const OpView& ov) { return ov.t_ampb; }
template <> __device__ __forceinline__ const float2* amp_b<float>(const OpView& ov) { return ov.t_ampb32; }

struct SharedTables {
    uint32_t binom[33 * 33];
    uint32_t base_hi[34];
    uint32_t base_lo[34];
};

__device__ __forceinline__ void stage_tables(SharedTables& sh, const IndexView& iv) {
    for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) sh.binom[i] = __ldg(iv.binom + i);
    if (threadIdx.x < 34) {
        sh.base_hi[threadIdx.x] = iv.hi.base[threadIdx.x];
        sh.base_lo[threadIdx.x] = iv.lo.base[threadIdx.x];
    }
    __syncthreads();
}

// Position of the l-th (0-based) set bit of s, for l = lane and l = lane + 32.
__device__ __forceinline__ void occupied_positions(uint64_t s, int lane, int& pos0, int& pos1) {
    uint32_t lo32 = (uint32_t)s, hi32 = (uint32_t)(s >> 32);
    int clo = __popc(lo32);
    pos0 = lane < clo ? (int)__fns(lo32, 0, lane + 1) : 32 + (int)__fns(hi32, 0, lane - clo + 1);
    int l1 = lane + 32;
    pos1 = l1 < clo ? (int)__fns(lo32, 0, l1 + 1) : 32 + (int)__fns(hi32, 0, l1 - clo + 1);
}

__device__ __forceinline__ int pos_of(int l, int pos0, int pos1) {
    int a = __shfl_sync(kFull, pos0, l & 31);
    int b = __shfl_sync(kFull, pos1, l & 31);
    return l < 32 ? a : b;
}

// p-th pair (u < v) in the order (0,1), (0,2), (1,2), (0,3), ...: v(v-1)/2 <= p
__device__ __forceinline__ void pair_of(int p, int& u, int& v) {
    int w = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)p)) * 0.5f);
    while (w * (w - 1) / 2 > p) --w;
    while ((w + 1) * w / 2 <= p) ++w;
    v = w;
    u = p - w * (w - 1) / 2;
}

// Visit every candidate group of state s: calls f(g) once per lane per batch of 32 groups
// (g = -1 for idle lanes); f must be warp-collective.
template <typename F>
__device__ __forceinline__ void for_each_group_batch(uint64_t s, const OpView& ov, F&& f) {
    const int lane = threadIdx.x & 31;
    int pos0, pos1;
    occupied_positions(s, lane, pos0, pos1);
    const int ne = __popcll(s);
    for (int b0 = 0; b0 < ne; b0 += 32) {                       // one-body groups
        int l = b0 + lane;
        int g = (l < ne) ? __ldg(ov.single + (b0 == 0 ? pos0 : pos1)) : -1;
        f(g);
    }
    const int np = ne * (ne - 1) / 2;
    for (int b0 = 0; b0 < np; b0 += 32) {                       // two-body groups
        int p = b0 + lane;
        int u = 0, v = 1;
        if (p < np) pair_of(p, u, v);
        int a = pos_of(u, pos0, pos1);
        int b = pos_of(v, pos0, pos1);
        int g = (p < np) ? __ldg(ov.pair + a * 64 + b) : -1;
        f(g);
    }
    for (int b0 = 0; b0 < ov.ngeneric; b0 += 32) {             // other groups: direct test
        int q = b0 + lane;
        int g = -1;
        if (q < ov.ngeneric) {
            g = __ldg(ov.generic + q);
            uint64_t om = __ldg(ov.g_out + g);
            if ((s & om) != om) g = -1;
        }
        f(g);
    }
}

// Compact the batch's groups into warp scratch; returns the flattened term count.
__device__ __forceinline__ int stage_batch(int g, const OpView& ov, WarpScratch& ws) {
    const int lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(kFull, g >= 0);
    if (m == 0) return 0;
    int slot = __popc(m & ((1u << lane) - 1u));
    int sz = 0;
    if (g >= 0) {
        int st = __ldg(ov.g_start + g);
        sz = __ldg(ov.g_start + g + 1) - st;
        ws.out[slot] = __ldg(ov.g_out + g);
        ws.start[slot] = st;
    }
    int incl = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (g >= 0) ws.pref[slot + 1] = incl;
    if (lane == 0) ws.pref[0] = 0;
    int total = __shfl_sync(kFull, incl, 31);
    __syncwarp();
    return total;
}

// Evaluate the term at flattened position f of the staged batch: returns j (or -1) and the sign.
__device__ __forceinline__ int64_t eval_term(int f, int& gi, uint64_t s, int64_t row, const OpView& ov,
                                             const IndexView& iv, const WarpScratch& ws, const SharedTables& sh,
                                             int& t, bool& neg) {
    while (ws.pref[gi + 1] <= f) ++gi;
    t = ws.start[gi] + (f - ws.pref[gi]);
    uint64_t om = ws.out[gi];
    uint64_t tin = __ldg(ov.t_in + t);
    uint64_t mid = s & ~om;
    neg = false;
    if ((mid & tin) != 0) return -1;
    if (tin == om) return row;                                    // diagonal term
    neg = (__popcll(mid & __ldg(ov.t_pm + t)) & 1) != 0;
    return lookup_index(iv, mid | tin, sh.base_hi, sh.base_lo, sh.binom);
}

template <typename K>
int persistent_grid(K kernel, int64_t rows) {
    static const int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWarps * 32, 0);
    if (per_sm <= 0) per_sm = 1;
    int64_t need = (rows + kWarps - 1) / kWarps;
    return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * per_sm));
}

}  // namespace

}  // namespace momed
