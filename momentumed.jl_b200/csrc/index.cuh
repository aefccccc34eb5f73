// Device-side basis index lookup: target state -> row index in the sorted basis.
//
// The reference searches the sorted basis per hit (device_binary_search,
// gpu_interface.jl:98-113; CPU searchsortedfirst + index_fit,
// hilbert_subspace.jl:67-72), about log2(N) dependent loads.  Here the
// lookup is two independent table reads:
//
//     index(t) = off_hi[slot(t >> L)] + rank_lo[slot(t & (2^L - 1))]
//
// valid whenever every low pattern has the same rank inside every high group
// in which it occurs.  That holds for every sector ED_momentum_subspaces
// produces (all states with fixed per-component counts and total momentum),
// and build_index verifies it on the actual basis before enabling it; other
// bases fall back to the branch-free binary search.  A target that is not in
// the basis (a term that leaves the sector, dropped by the reference through
// index_fit / j == 0) is detected in the checked mode by comparing keys.
#pragma once
#include "momed_internal.cuh"

namespace momed {

__device__ __forceinline__ uint32_t part_slot(uint64_t state, const PartDesc& d, const uint32_t* __restrict__ base,
                                              const uint32_t* __restrict__ binom) {
    if (d.width == 0) return 0u;
    uint64_t p = (state >> d.shift) & ((1ull << d.width) - 1ull);
    if (d.mode == PART_DIRECT) return (uint32_t)p;
    int c = __popcll(p);
    if (c < d.cmin || c > d.cmax) return kInvalid;
    uint32_t r = base[c - d.cmin];
    int k = 1;
    while (p) {
        int pos = __ffsll((long long)p) - 1;
        r += binom[pos * 33 + k];
        ++k;
        p &= p - 1ull;
    }
    return r;
}

// Branch-free lower bound on a sorted unique array; -1 when v is absent.
__device__ __forceinline__ int64_t search_basis(const uint64_t* __restrict__ b, int64_t n, uint64_t v) {
    if (n <= 0) return -1;
    int64_t base = 0, len = n;
    while (len > 1) {
        int64_t half = len >> 1;
        base = (__ldg(b + base + half) <= v) ? base + half : base;
        len -= half;
    }
    return (__ldg(b + base) == v) ? base : -1;
}

// base_hi / base_lo / binom are the caller's (shared-memory) copies of the tables
__device__ __forceinline__ int64_t lookup_index(const IndexView& iv, uint64_t t, const uint32_t* base_hi,
                                                const uint32_t* base_lo, const uint32_t* binom) {
    if (iv.mode == INDEX_SEARCH) return search_basis(iv.basis, iv.n, t);
    uint32_t sh = part_slot(t, iv.hi, base_hi, binom);
    uint32_t sl = part_slot(t, iv.lo, base_lo, binom);
    if (iv.mode == INDEX_RANKED) return (int64_t)__ldg(iv.off_hi + sh) + (int64_t)__ldg(iv.rank_lo + sl);
    if (sh == kInvalid || sl == kInvalid || sh >= iv.hi.size || sl >= iv.lo.size) return -1;
    uint32_t o = __ldg(iv.off_hi + sh), r = __ldg(iv.rank_lo + sl);
    if (o == kInvalid || r == kInvalid) return -1;
    int64_t j = (int64_t)o + (int64_t)r;
    if (j >= iv.n || __ldg(iv.basis + j) != t) return -1;
    return j;
}

}  // namespace momed
