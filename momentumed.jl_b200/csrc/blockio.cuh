// Lane layout of the block kernels: NB right-hand sides interleaved per row as x[row * NB + r].
// A hit's NB values are read by LPH = NB / RPL lanes, RPL values per lane (16-byte loads), so a
// warp iteration covers HPI = 32 / LPH hits.  The values a lane holds are chosen so that every
// load instruction of the LPH lanes reads one contiguous run of the row: lane kk's load i covers
// values i * NB / L + P * kk .. + P - 1 (P values per load, L loads per lane), i.e. for c64 at
// NB = 32 the 8 lanes read bytes 0..127 of the row with the first float4 load and 128..255 with
// the second, one full 128-byte line per load instead of two half-read lines.
#pragma once
#include <type_traits>

#include "candidates.cuh"

namespace momed {

namespace {

template <typename R> struct BlkMax;
template <> struct BlkMax<float> { static constexpr int RPL = 4; };
template <> struct BlkMax<double> { static constexpr int RPL = 2; };
template <typename R, int NB> struct Blk {
    static constexpr int RPL = NB < BlkMax<R>::RPL ? NB : BlkMax<R>::RPL;
};
// c128 below 32 right-hand sides: one 16-byte value per lane keeps the register count (and so the
// occupancy) of the candidate stage; two per lane measured slower there
template <int NB> struct Blk<double, NB> {
    static constexpr int RPL = NB == 32 ? 2 : 1;
};

template <typename R, int NB> struct BlkIO {
    static constexpr int RPL = Blk<R, NB>::RPL;
    static constexpr int LPH = NB / RPL;                                           // lanes per hit
    static constexpr int HPI = 32 / LPH;                                           // hits per warp iteration
    static constexpr int P = (std::is_same<R, float>::value && RPL >= 2) ? 2 : 1;  // values per load
    static constexpr int L = RPL / P;                                              // loads per lane
    // right-hand side of a lane's q-th value (kk = lane % LPH)
    __device__ static __forceinline__ int rhs(int kk, int q) { return (q / P) * (NB / L) + P * kk + (q % P); }
};

// The RPL values of lane kk in the row that starts at p (p 16-byte aligned).
template <typename R, int NB>
__device__ __forceinline__ void load_lane(const typename Cx<R>::T* __restrict__ p, int kk, typename Cx<R>::T* v) {
    using IO = BlkIO<R, NB>;
    if constexpr (IO::P == 2) {
#pragma unroll
        for (int i = 0; i < IO::L; ++i) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(p + i * (NB / IO::L) + 2 * kk));
            v[2 * i] = make_float2(a.x, a.y);
            v[2 * i + 1] = make_float2(a.z, a.w);
        }
    } else {
#pragma unroll
        for (int q = 0; q < IO::RPL; ++q) v[q] = __ldg(p + IO::rhs(kk, q));
    }
}

template <typename R, int NB>
__device__ __forceinline__ void store_lane(typename Cx<R>::T* __restrict__ p, int kk, const typename Cx<R>::T* v) {
    using IO = BlkIO<R, NB>;
    if constexpr (IO::P == 2) {
#pragma unroll
        for (int i = 0; i < IO::L; ++i)
            *reinterpret_cast<float4*>(p + i * (NB / IO::L) + 2 * kk) =
                make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
    } else {
#pragma unroll
        for (int q = 0; q < IO::RPL; ++q) p[IO::rhs(kk, q)] = v[q];
    }
}

}  // namespace

}  // namespace momed
