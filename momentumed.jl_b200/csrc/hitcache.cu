// Hit cache of the matrix-free map: for one sector basis and one term list, the (target row,
// term slot, sign) of every off-diagonal (row, term) hit and each row's diagonal sums, found
// once by the candidate machinery and reused by every later map of the solve.
//
// The map of ka_linearmap_kernel! (MomentumED/src/method/gpu_interface.jl:128-163) evaluates
// every term of every row at every application: mask test, fermionic sign, index of the target
// (binary search there, two table reads here).  Within an eigensolve those results are the
// same at every application, and for every right-hand side of a block; only the amplitudes
// (A + u B per right-hand side) and x change.  On the headline sector the candidate stage is
// ~80% of the block map's instructions.  The cache keeps what the candidate stage computes and
// nothing the amplitudes determine:
//
//   row_ptr[n+1] (int64)   start of each row's hits
//   seg[n] (int2)          ends of the row's B-only and A-only runs, relative to row_ptr[row]:
//                          hits are stored B-only | A-only | A-and-B, each run in candidate order
//   hit[nnz] (uint2)       {target row, term slot | sign << 31}
//   diag[2n]               the row's diagonal terms summed, A part and B part (FP64, and c64)
//
// 8 bytes per hit, against 20-44 for a stored matrix entry; the values are still formed from the
// term list at every application, so a new u needs no rebuild.  A map over the cache reads the
// hit stream (coalesced), the amplitude of each hit's term slot (the term list stays in L1/L2)
// and gathers x.  The cache is built when it fits a quarter of the free HBM (MOMED_HITCACHE=0
// turns it off, =1 builds it whatever its size); sectors whose hits do not fit (the 35M-state
// 4x9 sectors: ~170 GB) get the slot mode instead: per hit only its term slot (uint16, 2 bytes;
// 43 GB for a 4x9 Ne = 12 sector), from which the single-vector map forms the target exactly as
// the candidate map does (mask arithmetic, sign, two table reads) without the candidate stage;
// the block maps read full caches only.  It is dropped with the basis, the operator or the
// amplitudes (a twisted-boundary update) it was built from.
#include <chrono>
#include <cstdlib>
#include <string>

#include "blockio.cuh"

namespace momed {

namespace {

// 0: B part only, 1: A part only (every hit of an operator without a B part), 2: both
__device__ __forceinline__ int hit_kind(const OpView& ov, int t) {
    if (!ov.t_ampb) return 1;
    const double2 a = __ldg(ov.t_amp + t), b = __ldg(ov.t_ampb + t);
    const bool za = a.x == 0.0 && a.y == 0.0, zb = b.x == 0.0 && b.y == 0.0;
    return za ? 0 : (zb ? 1 : 2);
}

__global__ void __launch_bounds__(kWarps * 32)
k_hc_count(IndexView iv, OpView ov, int32_t* __restrict__ counts, int64_t rows) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpScratch& ws = s_ws[wid];
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        int c0 = 0, c1 = 0, c2 = 0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                if (f < total) {
                    int t;
                    bool neg;
                    const int64_t j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                    if (j >= 0 && j != row) {
                        const int k = hit_kind(ov, t);
                        c0 += k == 0;
                        c1 += k == 1;
                        c2 += k == 2;
                    }
                }
            }
            __syncwarp();
        });
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            c0 += __shfl_xor_sync(kFull, c0, o);
            c1 += __shfl_xor_sync(kFull, c1, o);
            c2 += __shfl_xor_sync(kFull, c2, o);
        }
        if (lane == 0) {
            counts[3 * row] = c0;
            counts[3 * row + 1] = c1;
            counts[3 * row + 2] = c2;
        }
    }
}

// bad[0]: hits that fell outside their run (count and fill passes disagree); such hits are not
// written.  The diagonal sums are formed lane by lane and reduced by the same butterfly as the
// candidate block map's, so the FP64 diagonal is that map's to the bit.
__global__ void __launch_bounds__(kWarps * 32)
k_hc_fill(IndexView iv, OpView ov, const int64_t* __restrict__ row_ptr, const int2* __restrict__ seg,
          uint2* __restrict__ hit, double2* __restrict__ dg64, float2* __restrict__ dg32, int64_t rows,
          unsigned long long* bad) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    WarpScratch& ws = s_ws[wid];
    unsigned long long nbad = 0;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        const int64_t base = row_ptr[row], end = row_ptr[row + 1];
        const int2 sg = seg[row];
        const int64_t e0 = base + sg.x, e1 = base + sg.y;
        int64_t p0 = base, p1 = e0, p2 = e1;   // warp-uniform: next free position of each run
        double dar = 0.0, dai = 0.0, dbr = 0.0, dbi = 0.0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                int64_t j = -1;
                int t = 0;
                bool neg = false;
                if (f < total) j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                if (j == row) {              // diagonal term (sign +)
                    const double2 a = __ldg(ov.t_amp + t);
                    dar += a.x;
                    dai += a.y;
                    if (ov.t_ampb) {
                        const double2 b = __ldg(ov.t_ampb + t);
                        dbr += b.x;
                        dbi += b.y;
                    }
                }
                const bool off = j >= 0 && j != row;
                const int k = off ? hit_kind(ov, t) : -1;
                const unsigned m0 = __ballot_sync(kFull, k == 0);
                const unsigned m1 = __ballot_sync(kFull, k == 1);
                const unsigned m2 = __ballot_sync(kFull, k == 2);
                if (off) {
                    const unsigned mk = k == 0 ? m0 : (k == 1 ? m1 : m2);
                    const int64_t pos = (k == 0 ? p0 : (k == 1 ? p1 : p2)) + __popc(mk & lt);
                    const int64_t lim = k == 0 ? e0 : (k == 1 ? e1 : end);
                    if (pos < lim) hit[pos] = make_uint2((uint32_t)j, (uint32_t)t | (neg ? 0x80000000u : 0u));
                    else ++nbad;
                }
                p0 += __popc(m0);
                p1 += __popc(m1);
                p2 += __popc(m2);
            }
            __syncwarp();
        });
        if (lane == 0 && (p0 != e0 || p1 != e1 || p2 != end)) ++nbad;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dar += __shfl_xor_sync(kFull, dar, o);
            dai += __shfl_xor_sync(kFull, dai, o);
            dbr += __shfl_xor_sync(kFull, dbr, o);
            dbi += __shfl_xor_sync(kFull, dbi, o);
        }
        if (lane == 0) {
            dg64[2 * row] = make_double2(dar, dai);
            dg64[2 * row + 1] = make_double2(dbr, dbi);
            dg32[2 * row] = make_float2((float)dar, (float)dai);
            dg32[2 * row + 1] = make_float2((float)dbr, (float)dbi);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nbad += __shfl_xor_sync(kFull, nbad, o);
    if (lane == 0 && nbad) atomicAdd(bad, nbad);
}

// Slot mode: the term slot of every off-diagonal hit in candidate order (one run per row), and
// the diagonal sums as k_hc_fill forms them.
__global__ void __launch_bounds__(kWarps * 32)
k_hc_fill_slots(IndexView iv, OpView ov, const int64_t* __restrict__ row_ptr, uint16_t* __restrict__ slot,
                double2* __restrict__ dg64, float2* __restrict__ dg32, int64_t rows, unsigned long long* bad) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    WarpScratch& ws = s_ws[wid];
    unsigned long long nbad = 0;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        const int64_t base = row_ptr[row], end = row_ptr[row + 1];
        int64_t p = base;                  // warp-uniform
        double dar = 0.0, dai = 0.0, dbr = 0.0, dbi = 0.0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                int64_t j = -1;
                int t = 0;
                bool neg = false;
                if (f < total) j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                if (j == row) {
                    const double2 a = __ldg(ov.t_amp + t);
                    dar += a.x;
                    dai += a.y;
                    if (ov.t_ampb) {
                        const double2 b = __ldg(ov.t_ampb + t);
                        dbr += b.x;
                        dbi += b.y;
                    }
                }
                const bool off = j >= 0 && j != row;
                const unsigned m = __ballot_sync(kFull, off);
                if (off) {
                    const int64_t pos = p + __popc(m & lt);
                    if (pos < end) slot[pos] = (uint16_t)t;
                    else ++nbad;
                }
                p += __popc(m);
            }
            __syncwarp();
        });
        if (lane == 0 && p != end) ++nbad;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dar += __shfl_xor_sync(kFull, dar, o);
            dai += __shfl_xor_sync(kFull, dai, o);
            dbr += __shfl_xor_sync(kFull, dbr, o);
            dbi += __shfl_xor_sync(kFull, dbi, o);
        }
        if (lane == 0) {
            dg64[2 * row] = make_double2(dar, dai);
            dg64[2 * row + 1] = make_double2(dbr, dbi);
            dg32[2 * row] = make_float2((float)dar, (float)dai);
            dg32[2 * row + 1] = make_float2((float)dbr, (float)dbi);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nbad += __shfl_xor_sync(kFull, nbad, o);
    if (lane == 0 && nbad) atomicAdd(bad, nbad);
}

template <typename R> __device__ __forceinline__ const typename Cx<R>::T* hc_diag(const HitCacheView& v);
template <> __device__ __forceinline__ const double2* hc_diag<double>(const HitCacheView& v) { return v.dg64; }
template <> __device__ __forceinline__ const float2* hc_diag<float>(const HitCacheView& v) { return v.dg32; }

// hit records are read once per map: not allocated in L1, which stays with the x gathers and the
// amplitude table (ld.global.nc.L1::no_allocate; 1-2% faster maps than cached loads)
__device__ __forceinline__ uint2 ld_hit(const uint2* p) {
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}





template <typename C2>
__device__ __forceinline__ C2 signed_amp(const C2* __restrict__ amp, uint32_t tw) {
    C2 a = __ldg(amp + (tw & 0x7fffffffu));
    if (tw >> 31) { a.x = -a.x; a.y = -a.y; }
    return a;
}

// y = H x over the cache, one right-hand side: a warp per row, lanes stride over its hits four
// at a time (hit records coalesced, amplitude and x gathers in flight together); the value of a
// hit is sign * (A + u B) of its term slot, as the candidate map forms it.
// comb[t] = A[t] + u B[t], formed as the candidate map forms a hit's value (same rounding)
template <typename R>
__global__ void k_hc_combine(const typename Cx<R>::T* __restrict__ A, const typename Cx<R>::T* __restrict__ B,
                             const R* __restrict__ u_ptr, typename Cx<R>::T* __restrict__ comb, int64_t n) {
    const R u = *u_ptr;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        typename Cx<R>::T a = A[t];
        const typename Cx<R>::T b = B[t];
        a.x += u * b.x;
        a.y += u * b.y;
        comb[t] = a;
    }
}

// amp: the term amplitudes at the map's u (A, or A + u B from k_hc_combine); the diagonal sums
// keep their A and B parts and take u here.
template <typename R, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_matvec_hc(HitCacheView hv, const typename Cx<R>::T* __restrict__ amp, const typename Cx<R>::T* __restrict__ x,
            typename Cx<R>::T* __restrict__ y, const R* __restrict__ u_ptr, int64_t rows) {
    using C2 = typename Cx<R>::T;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const R u = HAS_B ? *u_ptr : R(0);
    const C2* __restrict__ dg = hc_diag<R>(hv);
    auto val = [&](uint32_t tw) { return signed_amp(amp, tw); };
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const int64_t b = __ldg(hv.row_ptr + row), e = __ldg(hv.row_ptr + row + 1);
        R ar = 0, ai = 0;
        int64_t p = b + lane;
        for (; p + 96 < e; p += 128) {
            uint2 h[4];
            C2 v[4], xv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) h[q] = ld_hit(hv.hit + p + 32 * q);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                v[q] = val(h[q].y);
                xv[q] = __ldg(x + h[q].x);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ar += v[q].x * xv[q].x - v[q].y * xv[q].y;
                ai += v[q].x * xv[q].y + v[q].y * xv[q].x;
            }
        }
        for (; p < e; p += 32) {
            const uint2 h = ld_hit(hv.hit + p);
            const C2 v = val(h.y), xv = __ldg(x + h.x);
            ar += v.x * xv.x - v.y * xv.y;
            ai += v.x * xv.y + v.y * xv.x;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ar += __shfl_xor_sync(kFull, ar, o);
            ai += __shfl_xor_sync(kFull, ai, o);
        }
        if (lane == 0) {
            const C2 da = __ldg(dg + 2 * row);
            R cx = da.x, cy = da.y;
            if (HAS_B) {
                const C2 db = __ldg(dg + 2 * row + 1);
                cx += u * db.x;
                cy += u * db.y;
            }
            const C2 xd = __ldg(x + row);
            C2 o;
            o.x = ar + cx * xd.x - cy * xd.y;
            o.y = ai + cx * xd.y + cy * xd.x;
            y[row] = o;
        }
    }
}

// y = H x in slot mode, one right-hand side: a warp per row, lanes stride over its hit slots four
// at a time; each slot's target is formed as the candidate map forms it (the term's out and in
// masks on the row state, the sign from its parity mask, two index-table reads), its value from
// the A (+ u B) table, so only the candidate stage (groups, mask tests of the misses) is saved.
template <typename R, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_matvec_slots(IndexView iv, HitCacheView hv, OpView ov, const typename Cx<R>::T* __restrict__ amp,
               const typename Cx<R>::T* __restrict__ x, typename Cx<R>::T* __restrict__ y,
               const R* __restrict__ u_ptr, int64_t rows) {
    using C2 = typename Cx<R>::T;
    __shared__ SharedTables sh;
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const R u = HAS_B ? *u_ptr : R(0);
    const C2* __restrict__ dg = hc_diag<R>(hv);
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        const int64_t b = __ldg(hv.row_ptr + row), e = __ldg(hv.row_ptr + row + 1);
        R ar = 0, ai = 0;
        auto hit = [&](int t) {
            const uint64_t mid = s & ~__ldg(ov.t_out + t);
            const int64_t j = lookup_index(iv, mid | __ldg(ov.t_in + t), sh.base_hi, sh.base_lo, sh.binom);
            C2 v = __ldg(amp + t);
            if (__popcll(mid & __ldg(ov.t_pm + t)) & 1) { v.x = -v.x; v.y = -v.y; }
            const C2 xv = __ldg(x + j);
            ar += v.x * xv.x - v.y * xv.y;
            ai += v.x * xv.y + v.y * xv.x;
        };
        int64_t p = b + lane;
        for (; p + 96 < e; p += 128) {
            int t[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) t[q] = __ldg(hv.slot + p + 32 * q);
#pragma unroll
            for (int q = 0; q < 4; ++q) hit(t[q]);
        }
        for (; p < e; p += 32) hit(__ldg(hv.slot + p));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ar += __shfl_xor_sync(kFull, ar, o);
            ai += __shfl_xor_sync(kFull, ai, o);
        }
        if (lane == 0) {
            const C2 da = __ldg(dg + 2 * row);
            R cx = da.x, cy = da.y;
            if (HAS_B) {
                const C2 db = __ldg(dg + 2 * row + 1);
                cx += u * db.x;
                cy += u * db.y;
            }
            const C2 xd = __ldg(x + row);
            C2 o;
            o.x = ar + cx * xd.x - cy * xd.y;
            o.y = ai + cx * xd.y + cy * xd.x;
            y[row] = o;
        }
    }
}

// Block map over the cache: NB right-hand sides, operator A + u[r] B for right-hand side r.
// The three runs of a row are read with their kind fixed at compile time: B-only hits
// accumulate into a sum scaled by u once per row, A-only hits into the A sum, and hits with
// both parts form A + u B per right-hand side (the candidate map's three hit rings).
// Each lane group loads its own hit record and amplitude, two hits in flight per lane.  Loading
// 32 records per warp at once (the next 32 in flight) and handing them out by shuffles was
// measured slower (0.84 against 0.70 ms per launch on the headline sector: more registers, the
// shuffles on the issue path).
// The hit records of a lane group's next two hits are loaded before the current two are
// consumed (their stream comes from HBM; the x rows, from L2, then wait on one latency only;
// 1% faster maps).  Fitting its registers to 5 or 6 resident CTAs per SM (48 or 40 registers)
// spilled 156-232 bytes and ran 1.14-1.16 ms per launch against 0.70 ms at 63 registers; four
// hits in flight per lane group (72 registers, 3 CTAs per SM) ran 0.76 ms.
template <typename R, int NB, bool HAS_B>
__device__ __forceinline__ void block_hc_body(const HitCacheView& hv, const OpView& ov,
                                              const typename Cx<R>::T* __restrict__ x,
                                              typename Cx<R>::T* __restrict__ y, const R* __restrict__ u,
                                              int64_t rows) {
    using C2 = typename Cx<R>::T;
    using IO = BlkIO<R, NB>;
    constexpr int RPL = IO::RPL, LPH = IO::LPH, HPI = IO::HPI;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hslot = lane / LPH, kk = lane % LPH;
    auto urq = [&](int q) { return HAS_B ? __ldg(u + IO::rhs(kk, q)) : R(0); };
    const C2* __restrict__ A = amp_a<R>(ov);
    const C2* __restrict__ B = amp_b<R>(ov);
    const C2* __restrict__ dg = hc_diag<R>(hv);

    // KIND 0: accb += c x (c = B); 1: acc += c x (c = A); 2: acc += (A + u B) x
    auto run = [&](auto kind_tag, int64_t beg, int64_t end, C2* acc, C2* accb) {
        constexpr int KIND = decltype(kind_tag)::value;
        auto fma = [&](uint32_t j, C2 c, C2 cb) {
            C2 xv[RPL];
            load_lane<R, NB>(x + (int64_t)j * NB, kk, xv);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                R cx = c.x, cy = c.y;
                if constexpr (KIND == 2) {
                    cx += urq(q) * cb.x;
                    cy += urq(q) * cb.y;
                }
                C2* a = KIND == 0 ? accb : acc;
                a[q].x += cx * xv[q].x - cy * xv[q].y;
                a[q].y += cx * xv[q].y + cy * xv[q].x;
            }
        };
        // the hit with record h: target and signed amplitude(s) of its kind
        auto use = [&](uint2 h) {
            C2 c, cb;
            if constexpr (KIND == 0) c = signed_amp(B, h.y);
            else c = signed_amp(A, h.y);
            if constexpr (KIND == 2) cb = signed_amp(B, h.y);
            fma(h.x, c, cb);
        };
        // two hits of a lane group per step, the next two hit records loaded before these are used
        int64_t p = beg + hslot;
        if (p + HPI < end) {
            uint2 h0 = ld_hit(hv.hit + p), h1 = ld_hit(hv.hit + p + HPI);
            for (;;) {
                const int64_t pn = p + 2 * HPI;
                const bool more = pn + HPI < end;
                uint2 n0 = h0, n1 = h1;
                if (more) {
                    n0 = ld_hit(hv.hit + pn);
                    n1 = ld_hit(hv.hit + pn + HPI);
                }
                use(h0);
                use(h1);
                p = pn;
                if (!more) break;
                h0 = n0;
                h1 = n1;
            }
        }
        if (p < end) use(ld_hit(hv.hit + p));
    };

    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const int64_t b0 = __ldg(hv.row_ptr + row), e2 = __ldg(hv.row_ptr + row + 1);
        const int2 sg = __ldg(hv.seg + row);
        const int64_t e0 = b0 + sg.x, e1 = b0 + sg.y;
        C2 acc[RPL], accb[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            acc[q].x = 0; acc[q].y = 0;
            accb[q].x = 0; accb[q].y = 0;
        }
        if (HAS_B) {
            run(std::integral_constant<int, 0>{}, b0, e0, acc, accb);
            // fold u * (B-only sum) here, not after the other runs: the B accumulators and the
            // u values are then dead in the A-only and A + uB runs and the kernel fits 48
            // registers (5 CTAs per SM for c64) instead of 63 (4)
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                const R uq = __ldg(u + IO::rhs(kk, q));
                acc[q].x = uq * accb[q].x;
                acc[q].y = uq * accb[q].y;
            }
            run(std::integral_constant<int, 1>{}, e0, e1, acc, accb);
            run(std::integral_constant<int, 2>{}, e1, e2, acc, accb);
        } else {
            // without u the operator is its A part: B-only hits contribute nothing
            run(std::integral_constant<int, 1>{}, e0, e2, acc, accb);
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
#pragma unroll
            for (int o = LPH; o < 32; o <<= 1) {
                acc[q].x += __shfl_xor_sync(kFull, acc[q].x, o);
                acc[q].y += __shfl_xor_sync(kFull, acc[q].y, o);
            }
        }
        if (hslot == 0) {
            const C2 da = __ldg(dg + 2 * row);
            C2 db;
            db.x = 0; db.y = 0;
            if (HAS_B) db = __ldg(dg + 2 * row + 1);
            C2 xd[RPL], o[RPL];
            load_lane<R, NB>(x + row * NB, kk, xd);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                const R cx = da.x + urq(q) * db.x, cy = da.y + urq(q) * db.y;
                o[q].x = acc[q].x + cx * xd[q].x - cy * xd[q].y;
                o[q].y = acc[q].y + cx * xd[q].y + cy * xd[q].x;
            }
            store_lane<R, NB>(y + row * NB, kk, o);
        }
    }
}

template <typename R, int NB, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_block_hc(HitCacheView hv, OpView ov, const typename Cx<R>::T* __restrict__ x, typename Cx<R>::T* __restrict__ y,
           const R* __restrict__ u, int64_t rows) {
    block_hc_body<R, NB, HAS_B>(hv, ov, x, y, u, rows);
}

template <typename K>
int hc_grid(K kernel, int64_t rows) { return persistent_grid(kernel, rows); }

template <typename R> const typename Cx<R>::T* amp_a_host(const OpView& ov);
template <> const double2* amp_a_host<double>(const OpView& ov) { return ov.t_amp; }
template <> const float2* amp_a_host<float>(const OpView& ov) { return ov.t_amp32; }
template <typename R> const typename Cx<R>::T* amp_b_host(const OpView& ov);
template <> const double2* amp_b_host<double>(const OpView& ov) { return ov.t_ampb; }
template <> const float2* amp_b_host<float>(const OpView& ov) { return ov.t_ampb32; }

}  // namespace

HitCacheView HitCache::view() const {
    HitCacheView v{};
    v.row_ptr = row_ptr.p;
    v.seg = seg.p;
    v.hit = hit.p;
    v.dg64 = dg64.p;
    v.dg32 = dg32.p;
    v.slot = slot.p;
    return v;
}

int64_t hit_cache_bytes(int64_t n, int64_t hits) {
    return (n + 1) * 8 + n * (8 + 32 + 16) + hits * 8;
}

int64_t slot_cache_bytes(int64_t n, int64_t hits) {
    return (n + 1) * 8 + n * (32 + 16) + hits * 2;
}

// The full cache when it fits a quarter of the free memory, else the slot mode when that fits
// 30% (term slots must fit 16 bits); MOMED_HITCACHE=0: none, =1: full whatever its size, =2:
// slot mode whatever its size.
int hit_cache_wanted(const momed_handle* h) {
    const char* e = std::getenv("MOMED_HITCACHE");
    if (e && e[0] == '0') return 0;
    if (!h->hit_cache_ok || h->hbm_budget > 0 || h->sparse.built || h->sparse_only || h->n <= 0 || !h->op_set)
        return 0;
    const bool slots_ok = h->op.nterms <= 65536;
    if (e && e[0] == '1') return 1;
    if (e && e[0] == '2') return slots_ok ? 2 : 0;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    if ((double)hit_cache_bytes(h->n, h->nnz) <= 0.25 * (double)free_b) return 1;
    if (slots_ok && (double)slot_cache_bytes(h->n, h->nnz) <= 0.30 * (double)free_b) return 2;
    return 0;
}

void build_hit_cache(momed_handle* h, int mode) {
    HitCache& hc = h->hcache;
    hc.release();
    MOMED_REQUIRE(mode == 1 || mode == 2, MOMED_EINVAL, "hit cache: unknown mode");
    MOMED_REQUIRE(mode == 1 || h->op.nterms <= 65536, MOMED_EINVAL, "hit cache: slot mode needs <= 65536 terms");
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    MOMED_REQUIRE(n > 0 && n < (int64_t)0x7fffffff, MOMED_EINVAL, "hit cache: basis size out of range");
    MOMED_REQUIRE(h->op.nterms < (int64_t)0x7fffffff, MOMED_EINVAL, "hit cache: too many terms");
    const IndexView iv = index_view(h);
    const OpView ov = h->op.view();

    DevBuf<int32_t> counts;
    counts.resize(3 * n);
    k_hc_count<<<hc_grid(k_hc_count, n), kWarps * 32, 0, st>>>(iv, ov, counts.p, n);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    std::vector<int32_t> c(3 * n);
    MOMED_CUDA_TRY(cudaMemcpyAsync(c.data(), counts.p, 3 * n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    counts.release();
    std::vector<int64_t> rp(n + 1);
    std::vector<int2> sg(n);
    rp[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int32_t a = c[3 * i], b = c[3 * i + 1], d = c[3 * i + 2];
        sg[i] = make_int2(a, a + b);
        rp[i + 1] = rp[i] + a + b + d;
    }
    const int64_t nnz = rp[n];
    const int64_t need = mode == 1 ? hit_cache_bytes(n, nnz) : slot_cache_bytes(n, nnz);
    size_t free_b = 0, total_b = 0;
    MOMED_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if ((double)need > 0.9 * (double)free_b)
        throw Error{MOMED_ENOMEM, "hit cache: needs " + std::to_string(need) + " bytes, " + std::to_string(free_b) +
                                     " free"};
    hc.row_ptr.resize(n + 1);
    hc.dg64.resize(2 * n);
    hc.dg32.resize(2 * n);
    MOMED_CUDA_TRY(cudaMemcpyAsync(hc.row_ptr.p, rp.data(), (n + 1) * 8, cudaMemcpyHostToDevice, st));
    h->counters.resize(16);
    MOMED_CUDA_TRY(cudaMemsetAsync(h->counters.p + 4, 0, sizeof(unsigned long long), st));
    if (mode == 1) {
        hc.seg.resize(n);
        hc.hit.resize(std::max<int64_t>(nnz, 1));
        MOMED_CUDA_TRY(cudaMemcpyAsync(hc.seg.p, sg.data(), n * sizeof(int2), cudaMemcpyHostToDevice, st));
        k_hc_fill<<<hc_grid(k_hc_fill, n), kWarps * 32, 0, st>>>(iv, ov, hc.row_ptr.p, hc.seg.p, hc.hit.p,
                                                                  hc.dg64.p, hc.dg32.p, n, h->counters.p + 4);
    } else {
        hc.slot.resize(std::max<int64_t>(nnz, 1));
        k_hc_fill_slots<<<hc_grid(k_hc_fill_slots, n), kWarps * 32, 0, st>>>(iv, ov, hc.row_ptr.p, hc.slot.p,
                                                                              hc.dg64.p, hc.dg32.p, n,
                                                                              h->counters.p + 4);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    unsigned long long bad = 0;
    MOMED_CUDA_TRY(cudaMemcpyAsync(&bad, h->counters.p + 4, sizeof(bad), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));   // also keeps rp / sg alive until their copies ran
    if (bad != 0) {
        hc.release();
        throw Error{MOMED_EINVAL, "hit cache: count and fill passes disagree on " + std::to_string(bad) + " hits"};
    }
    hc.nnz = nnz;
    hc.bytes = need;
    hc.mode = mode;
    hc.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    hc.built = true;
}

// The automatic build is an optimisation: when its allocations are refused (memory taken by
// another handle between the size check and the build) the solve goes on over the candidate map.
void ensure_hit_cache(momed_handle* h) {
    if (h->hcache.built) return;
    const int mode = hit_cache_wanted(h);
    if (!mode) return;
    try {
        build_hit_cache(h, mode);
    } catch (const Error& e) {
        if (e.code != MOMED_ENOMEM) throw;
        h->hcache.release();
    }
}

template <typename R> struct CombSlot;
template <> struct CombSlot<double> {
    static DevBuf<double2>& buf(HitCache& c) { return c.comb64; }
    static double& u(HitCache& c) { return c.comb_u64; }
    static bool& ok(HitCache& c) { return c.comb_ok64; }
};
template <> struct CombSlot<float> {
    static DevBuf<float2>& buf(HitCache& c) { return c.comb32; }
    static double& u(HitCache& c) { return c.comb_u32; }
    static bool& ok(HitCache& c) { return c.comb_ok32; }
};

// u is the handle's parameter on the device (h->u_dev / u_dev32): the combined amplitudes are
// formed again whenever the handle's u differs from the one they were formed at.
template <typename R>
static void matvec_hc_dispatch(momed_handle* h, const typename Cx<R>::T* x, typename Cx<R>::T* y, const R* u,
                               int64_t rows, cudaStream_t st) {
    using C2 = typename Cx<R>::T;
    if (rows <= 0) return;
    const HitCacheView hv = h->hcache.view();
    const OpView ov = h->op.view();
    const bool hb = (u != nullptr) && (std::is_same<R, double>::value ? ov.t_ampb != nullptr : ov.t_ampb32 != nullptr);
    const C2* amp = amp_a_host<R>(ov);
    MOMED_REQUIRE(h->hcache.built, MOMED_ESTATE, "hit cache: not built");
    if (hb) {
        HitCache& hc = h->hcache;
        auto& cb = CombSlot<R>::buf(hc);
        if (!CombSlot<R>::ok(hc) || CombSlot<R>::u(hc) != h->u) {
            const int64_t n = ov.nterms;
            cb.resize(std::max<int64_t>(n, 1));
            const int g = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184));
            k_hc_combine<R><<<g, 256, 0, st>>>(amp, amp_b_host<R>(ov), u, cb.p, n);
            MOMED_CUDA_TRY(cudaGetLastError());
            note_launches(1);
            CombSlot<R>::u(hc) = h->u;
            CombSlot<R>::ok(hc) = true;
        }
        amp = cb.p;
    }
    if (h->hcache.mode == 2) {
        const IndexView iv = index_view(h);
        auto gs = [&](auto k, const R* up) { k<<<hc_grid(k, rows), kWarps * 32, 0, st>>>(iv, hv, ov, amp, x, y, up, rows); };
        if (hb) gs(k_matvec_slots<R, true>, u);
        else gs(k_matvec_slots<R, false>, nullptr);
    } else {
        auto go = [&](auto k, const R* up) { k<<<hc_grid(k, rows), kWarps * 32, 0, st>>>(hv, amp, x, y, up, rows); };
        if (hb) go(k_matvec_hc<R, true>, u);
        else go(k_matvec_hc<R, false>, nullptr);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

void launch_matvec_hc_c128(momed_handle* h, const double2* x, double2* y, const double* u, int64_t rows,
                           cudaStream_t st) {
    matvec_hc_dispatch<double>(h, x, y, u, rows, st);
}

void launch_matvec_hc_c64(momed_handle* h, const float2* x, float2* y, const float* u, int64_t rows,
                          cudaStream_t st) {
    matvec_hc_dispatch<float>(h, x, y, u, rows, st);
}

template <typename R>
static void block_hc_dispatch(const momed_handle* h, const typename Cx<R>::T* x, typename Cx<R>::T* y, const R* u,
                              int32_t nb, int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    MOMED_REQUIRE(h->hcache.full(), MOMED_ESTATE, "hit cache: the block map needs a full cache");
    const HitCacheView hv = h->hcache.view();
    const OpView ov = h->op.view();
    const bool hb = (u != nullptr) && (std::is_same<R, double>::value ? ov.t_ampb != nullptr : ov.t_ampb32 != nullptr);
    auto go = [&](auto k, const R* up) { k<<<hc_grid(k, rows), kWarps * 32, 0, st>>>(hv, ov, x, y, up, rows); };
#define MOMED_BHC(NBV)                                                                        \
    case NBV:                                                                                 \
        if (hb) go(k_block_hc<R, NBV, true>, u);                                              \
        else go(k_block_hc<R, NBV, false>, nullptr);                                          \
        break;
    switch (nb) {
        MOMED_BHC(1)
        MOMED_BHC(2)
        MOMED_BHC(4)
        MOMED_BHC(8)
        MOMED_BHC(16)
        MOMED_BHC(32)
        default:
            throw Error{MOMED_EINVAL, "block width must be a power of two <= 32"};
    }
#undef MOMED_BHC
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

void launch_block_hc_c64(const momed_handle* h, const float2* x, float2* y, const float* u, int32_t nb, int64_t rows,
                         cudaStream_t st) {
    block_hc_dispatch<float>(h, x, y, u, nb, rows, st);
}
void launch_block_hc_c128(const momed_handle* h, const double2* x, double2* y, const double* u, int32_t nb,
                          int64_t rows, cudaStream_t st) {
    block_hc_dispatch<double>(h, x, y, u, nb, rows, st);
}

}  // namespace momed
