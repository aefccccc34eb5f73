// Construction and verification of the basis lookup tables (see index.cuh).
#include <algorithm>
#include <climits>

#include "index.cuh"

namespace momed {

namespace {

__global__ void k_or_reduce(const uint64_t* __restrict__ b, int64_t n, unsigned long long* out) {
    uint64_t acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc |= b[i];
    for (int o = 16; o > 0; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicOr(out, (unsigned long long)acc);
}

// min/max popcount of the low L bits and of the remaining high bits, for one L
__global__ void k_popc_range(const uint64_t* __restrict__ b, int64_t n, int L, int* out /* lo_min, lo_max, hi_min, hi_max */) {
    int lmin = 64, lmax = 0, hmin = 64, hmax = 0;
    uint64_t m = (L >= 64) ? ~0ull : ((1ull << L) - 1ull);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t s = b[i];
        int lo = __popcll(s & m), hi = __popcll(s & ~m);
        lmin = min(lmin, lo); lmax = max(lmax, lo);
        hmin = min(hmin, hi); hmax = max(hmax, hi);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lmin = min(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        hmin = min(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
        hmax = max(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out + 0, lmin); atomicMax(out + 1, lmax);
        atomicMin(out + 2, hmin); atomicMax(out + 3, hmax);
    }
}

struct Tables {
    PartDesc hi, lo;
    const uint32_t* binom;
};

__device__ __forceinline__ uint32_t slot_of(uint64_t s, const PartDesc& d, const uint32_t* binom) {
    return part_slot(s, d, d.base, binom);
}

__global__ void k_build_off_hi(const uint64_t* __restrict__ b, int64_t n, Tables t, uint32_t* off_hi) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t hi = t.hi.width ? (b[i] >> t.hi.shift) : 0ull;
        uint64_t prev = (i > 0 && t.hi.width) ? (b[i - 1] >> t.hi.shift) : ~0ull;
        if (i == 0 || hi != prev) off_hi[slot_of(b[i], t.hi, t.binom)] = (uint32_t)i;
    }
}

__global__ void k_build_rank_lo(const uint64_t* __restrict__ b, int64_t n, Tables t, const uint32_t* off_hi,
                                uint32_t* rank_lo) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t o = off_hi[slot_of(b[i], t.hi, t.binom)];
        rank_lo[slot_of(b[i], t.lo, t.binom)] = (uint32_t)(i - (int64_t)o);
    }
}

__global__ void k_verify(const uint64_t* __restrict__ b, int64_t n, Tables t, const uint32_t* off_hi,
                         const uint32_t* rank_lo, unsigned long long* bad) {
    unsigned long long cnt = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && b[i] <= b[i - 1]) { ++cnt; continue; }     // must be strictly ascending
        int64_t j = (int64_t)off_hi[slot_of(b[i], t.hi, t.binom)] + (int64_t)rank_lo[slot_of(b[i], t.lo, t.binom)];
        if (j != i) ++cnt;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(bad, cnt);
}

__global__ void k_check_sorted(const uint64_t* __restrict__ b, int64_t n, unsigned long long* bad) {
    unsigned long long cnt = 0;
    for (int64_t i = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (b[i] <= b[i - 1]) ++cnt;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(bad, cnt);
}

uint64_t host_binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    uint64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
    return r;
}

// Fill a part descriptor for bits [shift, shift + width) with popcounts in [cmin, cmax];
// returns table entries (UINT64_MAX when the part cannot be tabulated).
uint64_t plan_part(PartDesc& d, int shift, int width, int cmin, int cmax) {
    d = PartDesc{};
    d.shift = shift;
    d.width = width;
    d.cmin = cmin;
    d.cmax = cmax;
    if (width == 0) { d.mode = PART_DIRECT; d.size = 1; return 1; }
    uint64_t direct = width <= 26 ? (1ull << width) : UINT64_MAX;
    uint64_t comb = UINT64_MAX;
    if (width <= 32 && cmin <= cmax) {
        comb = 0;
        for (int c = cmin; c <= cmax; ++c) comb += host_binom(width, c);
    }
    // combinadic costs a few instructions per set bit: take it only when it shrinks the table 2x
    if (comb != UINT64_MAX && (direct == UINT64_MAX || comb * 2 <= direct)) {
        d.mode = PART_COMBINADIC;
        uint64_t acc = 0;
        for (int c = cmin; c <= cmax; ++c) { d.base[c - cmin] = (uint32_t)acc; acc += host_binom(width, c); }
        d.size = (uint32_t)comb;
        return comb;
    }
    if (direct == UINT64_MAX) return UINT64_MAX;
    d.mode = PART_DIRECT;
    d.size = (uint32_t)direct;
    return direct;
}

int grid_for(int64_t n, int threads = 256) {
    int64_t blocks = (n + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, 148 * 16));
}

}  // namespace

// Table size cap: 2^26 entries per table (256 MiB as uint32).
static constexpr uint64_t kMaxTableEntries = 1ull << 26;

void build_index(momed_handle* h) {
    Index& ix = h->index;
    ix.mode = INDEX_SEARCH;
    ix.misses_checked = -1;
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    if (n == 0) return;
    MOMED_REQUIRE(n < (int64_t)kInvalid, MOMED_EINVAL, "basis larger than 2^32-1 states");

    h->counters.resize(16);
    unsigned long long* dc = h->counters.p;
    MOMED_CUDA_TRY(cudaMemsetAsync(dc, 0, 16 * sizeof(unsigned long long), st));
    k_check_sorted<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, dc);
    k_or_reduce<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, dc + 1);
    unsigned long long hc[2];
    MOMED_CUDA_TRY(cudaMemcpyAsync(hc, dc, sizeof(hc), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    MOMED_REQUIRE(hc[0] == 0, MOMED_EINVAL, "basis must be sorted ascending without duplicates");
    uint64_t bits_or = hc[1] | h->op_mask_or;
    int nbits = bits_or ? 64 - __builtin_clzll(bits_or) : 1;

    // popcount ranges for every split point
    std::vector<int> ranges(4 * (nbits + 1));
    DevBuf<int> dr;
    dr.resize(4 * (nbits + 1));
    std::vector<int> init(4 * (nbits + 1));
    for (int L = 0; L <= nbits; ++L) { init[4 * L] = 64; init[4 * L + 1] = 0; init[4 * L + 2] = 64; init[4 * L + 3] = 0; }
    MOMED_CUDA_TRY(cudaMemcpyAsync(dr.p, init.data(), init.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    for (int L = 0; L <= nbits; ++L) k_popc_range<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, L, dr.p + 4 * L);
    MOMED_CUDA_TRY(cudaMemcpyAsync(ranges.data(), dr.p, ranges.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));

    // choose the split minimising table entries; widen popcount ranges by the largest
    // change a term can make so that every target of a hit maps into the tables
    int best_L = -1;
    uint64_t best = UINT64_MAX;
    PartDesc best_hi{}, best_lo{};
    for (int L = 0; L <= nbits; ++L) {
        PartDesc lo, hi;
        int lomin = ranges[4 * L], lomax = ranges[4 * L + 1], himin = ranges[4 * L + 2], himax = ranges[4 * L + 3];
        uint64_t slo = plan_part(lo, 0, L, lomin, lomax);
        uint64_t shi = plan_part(hi, L, nbits - L, himin, himax);
        if (slo == UINT64_MAX || shi == UINT64_MAX) continue;
        if (slo > kMaxTableEntries || shi > kMaxTableEntries) continue;
        uint64_t tot = slo + shi;
        if (tot < best) { best = tot; best_L = L; best_hi = hi; best_lo = lo; }
    }
    ix.hi = best_hi;
    ix.lo = best_lo;
    if (best_L < 0) return;   // search mode

    ix.off_hi.resize(ix.hi.size);
    ix.rank_lo.resize(ix.lo.size);
    MOMED_CUDA_TRY(cudaMemsetAsync(ix.off_hi.p, 0xFF, (size_t)ix.hi.size * 4, st));
    MOMED_CUDA_TRY(cudaMemsetAsync(ix.rank_lo.p, 0xFF, (size_t)ix.lo.size * 4, st));
    Tables t{ix.hi, ix.lo, h->binom.p};
    k_build_off_hi<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, t, ix.off_hi.p);
    k_build_rank_lo<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, t, ix.off_hi.p, ix.rank_lo.p);
    MOMED_CUDA_TRY(cudaMemsetAsync(dc + 2, 0, sizeof(unsigned long long), st));
    k_verify<<<grid_for(n), 256, 0, st>>>(h->basis.p, n, t, ix.off_hi.p, ix.rank_lo.p, dc + 2);
    unsigned long long bad = 0;
    MOMED_CUDA_TRY(cudaMemcpyAsync(&bad, dc + 2, sizeof(bad), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad == 0) {
        ix.mode = INDEX_CHECKED;   // promoted to RANKED once an operator validates without misses
    } else {
        ix.off_hi.release();
        ix.rank_lo.release();
        ix.mode = INDEX_SEARCH;
    }
}

IndexView index_view(const momed_handle* h) {
    IndexView v{};
    v.basis = h->basis.p;
    v.n = h->n;
    v.off_hi = h->index.off_hi.p;
    v.rank_lo = h->index.rank_lo.p;
    v.hi = h->index.hi;
    v.lo = h->index.lo;
    v.mode = h->index.mode;
    v.binom = h->binom.p;
    return v;
}

}  // namespace momed
