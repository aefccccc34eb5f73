// Kernel (b): matrix-free Hamiltonian map y = H x over the Hermitian-completed
// scatter list.
//
// Reference: ka_linearmap_kernel! (MomentumED/src/method/gpu_interface.jl:128-163)
// gives every row all N_scat terms and binary-searches each hit; it computes
// conj(H) x because it treats the row state as the term's input.  The CPU map
// (linear_map.jl:100-118, with mbs_out * scat from EDCore/src/multiplication.jl:55-69)
// computes H x, and that is what this kernel computes:
//
//   for row i with state s, for every term (amp, in, out, pm) with out within s:
//     mid = s & ~out;  skip if mid & in;  t = mid | in
//     sign = 1 - 2 (popcount(mid & pm) & 1);  j = index(t) (dropped if absent)
//     y[i] += sign * amp * x[j]
//
// Layout and schedule (B200):
//   - one warp per row, rows grid-strided so neighbouring warps work on
//     neighbouring (similar) states and their x gathers share L2 lines;
//   - terms are regrouped by `out`; a row only visits the groups whose `out`
//     it contains, found by table lookup on its occupied orbitals (one-body)
//     and orbital pairs (two-body): ~Ne + Ne(Ne-1)/2 lookups instead of N_scat
//     mask tests;
//   - the candidate terms of a batch of groups are flattened and dealt to the
//     32 lanes, so work stays balanced however uneven the groups are;
//   - the index of a target is two independent table reads (index.cuh);
//   - lanes accumulate privately and reduce with shuffles: no atomics.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "blockio.cuh"

namespace momed {

namespace {

template <typename R, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_matvec(IndexView iv, OpView ov, const typename Cx<R>::T* __restrict__ x, typename Cx<R>::T* __restrict__ y,
         const R* __restrict__ u_ptr, int64_t rows) {
    using C2 = typename Cx<R>::T;
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpScratch& ws = s_ws[wid];
    const R u = HAS_B ? *u_ptr : R(0);
    const C2* __restrict__ A = amp_a<R>(ov);
    const C2* __restrict__ B = amp_b<R>(ov);
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        R ar = 0, ai = 0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                if (f < total) {
                    int t;
                    bool neg;
                    int64_t j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                    if (j >= 0) {
                        C2 a = load_amp(A, t);
                        if (HAS_B) {
                            C2 b = load_amp(B, t);
                            a.x += u * b.x;
                            a.y += u * b.y;
                        }
                        C2 xv = x[j];
                        R pr = a.x * xv.x - a.y * xv.y;
                        R pi = a.x * xv.y + a.y * xv.x;
                        if (neg) { ar -= pr; ai -= pi; } else { ar += pr; ai += pi; }
                    }
                }
            }
            __syncwarp();
        });
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ar += __shfl_xor_sync(kFull, ar, o);
            ai += __shfl_xor_sync(kFull, ai, o);
        }
        if (lane == 0) {
            C2 out;
            out.x = ar;
            out.y = ai;
            y[row] = out;
        }
    }
}

// <bra| H |ket> without writing H ket: rows run over the bra space (row_states), targets are
// looked up in the ket space (iv; checked keys when the two spaces differ, so a target outside the
// ket space is dropped as index_fit drops it).  A lane folds conj(bra[row]) into its share of each
// row, a block writes one partial sum; the host adds the partials in block order.
template <bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_bracket(IndexView iv, OpView ov, const uint64_t* __restrict__ row_states, const double2* __restrict__ bra,
          const double2* __restrict__ ket, const double* __restrict__ u_ptr, int64_t rows,
          double2* __restrict__ partial) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    __shared__ double2 s_sum[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpScratch& ws = s_ws[wid];
    const double u = HAS_B ? *u_ptr : 0.0;
    double wr = 0.0, wi = 0.0;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(row_states + row);
        double ar = 0.0, ai = 0.0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                if (f < total) {
                    while (ws.pref[gi + 1] <= f) ++gi;
                    const int t = ws.start[gi] + (f - ws.pref[gi]);
                    const uint64_t om = ws.out[gi];
                    const uint64_t tin = __ldg(ov.t_in + t);
                    const uint64_t mid = s & ~om;
                    if ((mid & tin) == 0) {
                        const bool neg = (__popcll(mid & __ldg(ov.t_pm + t)) & 1) != 0;
                        const int64_t j = lookup_index(iv, mid | tin, sh.base_hi, sh.base_lo, sh.binom);
                        if (j >= 0) {
                            double2 a = __ldg(ov.t_amp + t);
                            if (HAS_B) {
                                const double2 b = __ldg(ov.t_ampb + t);
                                a.x += u * b.x;
                                a.y += u * b.y;
                            }
                            const double2 xv = __ldg(ket + j);
                            const double pr = a.x * xv.x - a.y * xv.y, pi = a.x * xv.y + a.y * xv.x;
                            if (neg) { ar -= pr; ai -= pi; } else { ar += pr; ai += pi; }
                        }
                    }
                }
            }
            __syncwarp();
        });
        const double2 bv = __ldg(bra + row);            // conj(bra) times this lane's share of the row
        wr += bv.x * ar + bv.y * ai;
        wi += bv.x * ai - bv.y * ar;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wr += __shfl_xor_sync(kFull, wr, o);
        wi += __shfl_xor_sync(kFull, wi, o);
    }
    if (lane == 0) s_sum[wid] = make_double2(wr, wi);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 acc = make_double2(0.0, 0.0);
        for (int w = 0; w < kWarps; ++w) { acc.x += s_sum[w].x; acc.y += s_sum[w].y; }
        partial[blockIdx.x] = acc;
    }
}

// Counts hits (targets found) and misses (targets outside the basis) without touching x.
__global__ void __launch_bounds__(kWarps * 32)
k_count(IndexView iv, OpView ov, unsigned long long* hits, unsigned long long* misses, int64_t rows) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpScratch& ws = s_ws[wid];
    unsigned long long nh = 0, nm = 0;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                if (f < total) {
                    int t;
                    bool neg;
                    // decide "mask-compatible" separately from "found"
                    while (ws.pref[gi + 1] <= f) ++gi;
                    t = ws.start[gi] + (f - ws.pref[gi]);
                    uint64_t om = ws.out[gi];
                    uint64_t tin = __ldg(ov.t_in + t);
                    uint64_t mid = s & ~om;
                    (void)neg;
                    if ((mid & tin) == 0) {
                        int64_t j = (tin == om) ? row : lookup_index(iv, mid | tin, sh.base_hi, sh.base_lo, sh.binom);
                        if (j >= 0) ++nh; else ++nm;
                    }
                }
            }
            __syncwarp();
        });
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nh += __shfl_xor_sync(kFull, nh, o);
        nm += __shfl_xor_sync(kFull, nm, o);
    }
    if (lane == 0) {
        if (nh) atomicAdd(hits, nh);
        if (nm) atomicAdd(misses, nm);
    }
}

// Block map: NB right-hand sides interleaved as x[row * NB + b], operator H_b = A + u[b] B.
// Candidate terms are evaluated once per row for all NB
// right-hand sides (one index lookup per hit); hits are compacted into three lists by amplitude
// kind (B only, A only, both), and each hit's NB values are read by LPH = NB / RPL lanes with RPL
// right-hand sides per lane (RPL = min(NB, 4) for c64; for c128 2 at NB = 32, else 1: 16-byte
// loads, laid out as blockio.cuh describes), so one warp iteration consumes HPI = 32 / LPH hits.
// B-only hits accumulate into a separate sum that is scaled by u once per row.
// Per-warp rings of found hits, one per amplitude kind.  A batch of 32 candidates yields about
// a dozen hits; they wait in the ring until 32 of a kind are pending, so the accumulation runs
// whole iterations and keeps several gathers in flight.
constexpr int kRing = 64;
template <typename R> struct HitRing {
    uint32_t j[3][kRing];
    typename Cx<R>::T c[3][kRing];
    typename Cx<R>::T cb[kRing];
};

// Accumulate the hits at ring positions start .. start + n - 1 (mod kRing) of amplitude kind KIND
// into acc: each hit's NB values are read by NB / RPL lanes.  N > 0 fixes n = N at compile time.
template <typename R, int NB, int KIND, int N>
__device__ __forceinline__ void consume_hits(const HitRing<R>& hl, int start, int n, int hslot, int kk,
                                             const typename Cx<R>::T* __restrict__ x, const R* ur,
                                             typename Cx<R>::T* acc) {
    using C2 = typename Cx<R>::T;
    constexpr int RPL = Blk<R, NB>::RPL;
    constexpr int HPI = 32 / (NB / RPL);
    auto one = [&](int k) {
        const int p = (start + k) & (kRing - 1);
        const C2 c = hl.c[KIND][p];
        C2 cb;
        if constexpr (KIND == 2) cb = hl.cb[p];
        C2 xv[RPL];
        load_lane<R, NB>(x + (int64_t)hl.j[KIND][p] * NB, kk, xv);
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            R cx = c.x, cy = c.y;
            if constexpr (KIND == 2) {
                cx += ur[q] * cb.x;
                cy += ur[q] * cb.y;
            }
            acc[q].x += cx * xv[q].x - cy * xv[q].y;
            acc[q].y += cx * xv[q].y + cy * xv[q].x;
        }
    };
    if constexpr (N > 0) {
#pragma unroll 2
        for (int i = 0; i < N / HPI; ++i) one(hslot + i * HPI);
    } else {
        for (int k = hslot; k < n; k += HPI) one(k);
    }
}

template <typename R, int NB, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32, (std::is_same<R, double>::value && NB == 32) ? 3 : 4)
k_block_matvec_v(IndexView iv, OpView ov, const typename Cx<R>::T* __restrict__ x, typename Cx<R>::T* __restrict__ y,
                 const R* __restrict__ u, int64_t rows, int rpw) {
    using C2 = typename Cx<R>::T;
    constexpr int RPL = Blk<R, NB>::RPL;
    constexpr int LPH = NB / RPL;      // lanes per hit
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    __shared__ HitRing<R> s_hits[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hslot = lane / LPH, kk = lane % LPH;
    WarpScratch& ws = s_ws[wid];
    HitRing<R>& hl = s_hits[wid];
    R ur[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) ur[q] = HAS_B ? u[BlkIO<R, NB>::rhs(kk, q)] : R(0);
    const C2* __restrict__ A = amp_a<R>(ov);
    const C2* __restrict__ B = amp_b<R>(ov);
    const unsigned lt = (1u << lane) - 1u;
    // a warp takes chunks of rpw consecutive rows (the autotuner's rows per warp)
    const int64_t nchunks = (rows + rpw - 1) / rpw;
    for (int64_t chunk = (int64_t)blockIdx.x * kWarps + wid; chunk < nchunks; chunk += (int64_t)gridDim.x * kWarps)
    for (int64_t row = chunk * rpw; row < rows && row < (chunk + 1) * rpw; ++row) {
        const uint64_t s = __ldg(iv.basis + row);
        C2 aa[RPL], ab[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) { aa[q].x = 0; aa[q].y = 0; ab[q].x = 0; ab[q].y = 0; }
        R dax = 0, day = 0, dbx = 0, dby = 0;
        int hd0 = 0, hd1 = 0, hd2 = 0, n0 = 0, n1 = 0, n2 = 0;   // ring heads and pending hits (warp-uniform)
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                int64_t j = -1;
                int t = 0;
                bool neg = false;
                if (f < total) j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                C2 a, b;
                a.x = 0; a.y = 0; b.x = 0; b.y = 0;
                if (j >= 0) {
                    a = load_amp(A, t);
                    if (HAS_B) b = load_amp(B, t);
                    if (neg) { a.x = -a.x; a.y = -a.y; b.x = -b.x; b.y = -b.y; }
                }
                if (j == row) {   // diagonal term (its sign is +): folded into a per-row sum
                    dax += a.x; day += a.y; dbx += b.x; dby += b.y;
                    j = -1;
                }
                const bool za = (a.x == R(0) && a.y == R(0)), zb = (b.x == R(0) && b.y == R(0));
                const int kind = !HAS_B ? 1 : (za ? 0 : (zb ? 1 : 2));
                const unsigned m0 = __ballot_sync(kFull, j >= 0 && kind == 0);
                const unsigned m1 = __ballot_sync(kFull, j >= 0 && kind == 1);
                const unsigned m2 = __ballot_sync(kFull, j >= 0 && kind == 2);
                if (j >= 0) {
                    const unsigned mk = kind == 0 ? m0 : (kind == 1 ? m1 : m2);
                    const int at = kind == 0 ? hd0 + n0 : (kind == 1 ? hd1 + n1 : hd2 + n2);
                    const int p = (at + __popc(mk & lt)) & (kRing - 1);
                    hl.j[kind][p] = (uint32_t)j;
                    hl.c[kind][p] = kind == 0 ? b : a;
                    if (kind == 2) hl.cb[p] = b;
                }
                n0 += __popc(m0);
                n1 += __popc(m1);
                n2 += __popc(m2);
                __syncwarp();
                if (HAS_B && n0 >= 32) {          // B only: accumulate, scale by u once per row
                    consume_hits<R, NB, 0, 32>(hl, hd0, 32, hslot, kk, x, ur, ab);
                    hd0 = (hd0 + 32) & (kRing - 1);
                    n0 -= 32;
                }
                if (n1 >= 32) {                   // A only
                    consume_hits<R, NB, 1, 32>(hl, hd1, 32, hslot, kk, x, ur, aa);
                    hd1 = (hd1 + 32) & (kRing - 1);
                    n1 -= 32;
                }
                if (HAS_B && n2 >= 32) {          // both: A + u B per right-hand side
                    consume_hits<R, NB, 2, 32>(hl, hd2, 32, hslot, kk, x, ur, aa);
                    hd2 = (hd2 + 32) & (kRing - 1);
                    n2 -= 32;
                }
                __syncwarp();
            }
        });
        if (HAS_B) consume_hits<R, NB, 0, 0>(hl, hd0, n0, hslot, kk, x, ur, ab);
        consume_hits<R, NB, 1, 0>(hl, hd1, n1, hslot, kk, x, ur, aa);
        if (HAS_B) consume_hits<R, NB, 2, 0>(hl, hd2, n2, hslot, kk, x, ur, aa);
        __syncwarp();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dax += __shfl_xor_sync(kFull, dax, o);
            day += __shfl_xor_sync(kFull, day, o);
            if (HAS_B) {
                dbx += __shfl_xor_sync(kFull, dbx, o);
                dby += __shfl_xor_sync(kFull, dby, o);
            }
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            aa[q].x += ur[q] * ab[q].x;
            aa[q].y += ur[q] * ab[q].y;
#pragma unroll
            for (int o = LPH; o < 32; o <<= 1) {
                aa[q].x += __shfl_xor_sync(kFull, aa[q].x, o);
                aa[q].y += __shfl_xor_sync(kFull, aa[q].y, o);
            }
        }
        if (hslot == 0) {
            C2 xd[RPL], o[RPL];
            load_lane<R, NB>(x + row * NB, kk, xd);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                R cx = dax + ur[q] * dbx, cy = day + ur[q] * dby;
                o[q].x = aa[q].x + cx * xd[q].x - cy * xd[q].y;
                o[q].y = aa[q].y + cx * xd[q].y + cy * xd[q].x;
            }
            store_lane<R, NB>(y + row * NB, kk, o);
        }
    }
}

}  // namespace

void launch_matvec_c128(const IndexView& iv, const OpView& ov, const double2* x, double2* y, const double* u_scale,
                        int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    if (u_scale && ov.t_ampb) {
        auto k = k_matvec<double, true>;
        k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(iv, ov, x, y, u_scale, rows);
    } else {
        auto k = k_matvec<double, false>;
        k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(iv, ov, x, y, nullptr, rows);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

void launch_matvec_c64(const IndexView& iv, const OpView& ov, const float2* x, float2* y, const float* u_scale,
                       int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    if (u_scale && ov.t_ampb32) {
        auto k = k_matvec<float, true>;
        k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(iv, ov, x, y, u_scale, rows);
    } else {
        auto k = k_matvec<float, false>;
        k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(iv, ov, x, y, nullptr, rows);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

int bracket_grid(int64_t rows) { return persistent_grid(k_bracket<false>, rows); }

void launch_bracket(const IndexView& iv, const OpView& ov, const uint64_t* row_states, const double2* bra,
                    const double2* ket, const double* u, int64_t rows, double2* partial, int grid, cudaStream_t st) {
    if (u && ov.t_ampb) k_bracket<true><<<grid, kWarps * 32, 0, st>>>(iv, ov, row_states, bra, ket, u, rows, partial);
    else k_bracket<false><<<grid, kWarps * 32, 0, st>>>(iv, ov, row_states, bra, ket, nullptr, rows, partial);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

void launch_count_hits(const IndexView& iv, const OpView& ov, unsigned long long* hits, unsigned long long* misses,
                       int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    k_count<<<persistent_grid(k_count, rows), kWarps * 32, 0, st>>>(iv, ov, hits, misses, rows);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

// ---------------------------------------------------------------------------------------
// Autotuner of the block map.  Two launch parameters are chosen by timing on the operator and
// basis at hand, once per (term list, orbitals used, size class of the sector, block width,
// precision): the persistent grid (resident CTAs per SM, or twice that for dynamic balance at
// the tail) and the rows per warp (1, 2 or 4 consecutive rows per work item: neighbouring
// basis states share most of their targets, so their x gathers meet in L1/L2).  Each candidate
// runs twice (the second timed with CUDA events on the launching stream); the fastest is cached
// for the process and reported by momed_block_tuning.  Tuning needs a stream outside capture;
// a launch inside a capture before its key is tuned uses the default (resident grid, 1 row).
struct TuneKey {
    int64_t nterms, size_class;
    int64_t groups;      // term groups and the per-row candidate bound: with nterms, the term list
    int nb, dbl, hb;
    bool operator<(const TuneKey& o) const {
        return std::tie(nterms, size_class, groups, nb, dbl, hb) <
               std::tie(o.nterms, o.size_class, o.groups, o.nb, o.dbl, o.hb);
    }
};
struct TuneChoice {
    int grid_mult = 0;   // 0: resident CTAs per SM - 1, 1: resident, 2: twice resident
    int rpw = 1;
    float ms = 0.f, ms_default = 0.f;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune;

bool autotune_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("MOMED_AUTOTUNE");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename K>
int tuned_grid(K kernel, int64_t rows, int rpw, int mult) {
    static const int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWarps * 32, 0);
    if (per_sm <= 0) per_sm = 1;
    const int64_t resident = (int64_t)sms * (mult == 0 ? std::max(1, per_sm - 1) : per_sm * mult);
    const int64_t need = ((rows + rpw - 1) / rpw + kWarps - 1) / kWarps;
    return (int)std::max<int64_t>(1, std::min<int64_t>(need, resident));
}

template <typename R, int NBV, bool HB>
void launch_block(const IndexView& iv, const OpView& ov, const typename Cx<R>::T* x, typename Cx<R>::T* y,
                  const R* u, int64_t rows, cudaStream_t st, const TuneKey& key) {
    auto k = k_block_matvec_v<R, NBV, HB>;
    TuneChoice ch;
    bool have = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) { ch = it->second; have = true; }
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (!have && autotune_enabled() && cs == cudaStreamCaptureStatusNone && rows >= 4096) {
        cudaEvent_t e0, e1;
        MOMED_CUDA_TRY(cudaEventCreate(&e0));
        MOMED_CUDA_TRY(cudaEventCreate(&e1));
        float best = 1e30f, dflt = 0.f;
        for (int mult = 0; mult <= 2; ++mult)
            for (int rpw : {1, 2, 4}) {
                const int g = tuned_grid(k, rows, rpw, mult);
                k<<<g, kWarps * 32, 0, st>>>(iv, ov, x, y, u, rows, rpw);
                MOMED_CUDA_TRY(cudaEventRecord(e0, st));
                k<<<g, kWarps * 32, 0, st>>>(iv, ov, x, y, u, rows, rpw);
                MOMED_CUDA_TRY(cudaEventRecord(e1, st));
                MOMED_CUDA_TRY(cudaEventSynchronize(e1));
                MOMED_CUDA_TRY(cudaGetLastError());
                note_launches(2);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (mult == 1 && rpw == 1) dflt = ms;
                if (ms < best) { best = ms; ch.grid_mult = mult; ch.rpw = rpw; }
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ch.ms = best;
        ch.ms_default = dflt;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune.emplace(key, ch);
    } else if (!have) {
        ch.grid_mult = 1;
        ch.rpw = 1;
    }
    k<<<tuned_grid(k, rows, ch.rpw, ch.grid_mult), kWarps * 32, 0, st>>>(iv, ov, x, y, u, rows, ch.rpw);
}

TuneKey tune_key(const OpView& ov, int64_t rows, int nb, bool dbl, bool hb) {
    TuneKey k;
    k.nterms = ov.nterms;
    int64_t c = 0;
    while ((rows >> c) > 1) ++c;                  // sectors within a factor 2 share a choice
    k.size_class = c;
    k.groups = (int64_t)ov.ngroups * 4096 + ov.max_groups_per_row;
    k.nb = nb;
    k.dbl = dbl ? 1 : 0;
    k.hb = hb ? 1 : 0;
    return k;
}

template <typename R>
static void block_dispatch(const IndexView& iv, const OpView& ov, const typename Cx<R>::T* x, typename Cx<R>::T* y,
                           const R* u, int32_t nb, int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    const bool hb = (u != nullptr) && (std::is_same<R, double>::value ? ov.t_ampb != nullptr : ov.t_ampb32 != nullptr);
    const TuneKey key = tune_key(ov, rows, nb, std::is_same<R, double>::value, hb);
#define MOMED_BLK(NBV)                                                                                   \
    case NBV:                                                                                            \
        if (hb) launch_block<R, NBV, true>(iv, ov, x, y, u, rows, st, key);                             \
        else launch_block<R, NBV, false>(iv, ov, x, y, u, rows, st, key);                               \
        break;
    switch (nb) {
        MOMED_BLK(1)
        MOMED_BLK(2)
        MOMED_BLK(4)
        MOMED_BLK(8)
        MOMED_BLK(16)
        MOMED_BLK(32)
        default:
            throw Error{MOMED_EINVAL, "block width must be a power of two <= 32"};
    }
#undef MOMED_BLK
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

bool block_tuning_lookup(const OpView& ov, int64_t rows, int nb, bool dbl, bool hb, int* grid_mult, int* rpw,
                         float* ms, float* ms_default) {
    const TuneKey key = tune_key(ov, rows, nb, dbl, hb);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    *grid_mult = it->second.grid_mult;
    *rpw = it->second.rpw;
    *ms = it->second.ms;
    *ms_default = it->second.ms_default;
    return true;
}

void launch_block_matvec_c64(const IndexView& iv, const OpView& ov, const float2* x, float2* y, const float* u,
                             int32_t nb, int64_t rows, cudaStream_t st) {
    block_dispatch<float>(iv, ov, x, y, u, nb, rows, st);
}
void launch_block_matvec_c128(const IndexView& iv, const OpView& ov, const double2* x, double2* y, const double* u,
                              int32_t nb, int64_t rows, cudaStream_t st) {
    block_dispatch<double>(iv, ov, x, y, u, nb, rows, st);
}

}  // namespace momed
