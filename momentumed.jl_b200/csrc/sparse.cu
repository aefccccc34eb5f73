// GPU sparse method: the Hamiltonian stored as a CSR matrix built on the device, and y = H x
// as a CSR SpMV.
//
// Reference: EDsolve(...; method = :sparse, device = :gpu) builds the matrix on host threads
// (ED_HamiltonianMatrix_threaded_CSCdirect, MomentumED/src/method/sparse_matrix.jl:64-190: for
// every basis state, every term of the Hermitian-completed list, index_fit drops targets
// outside the subspace, duplicates summed), uploads it (create_gpu_matrix,
// ext/MomentumEDCUDAExt.jl:145-152) and runs the library SpMV inside KrylovKit
// (krylov_matrix_solve, MomentumEDCUDAExt.jl:180-200).  Here the matrix is built where it is
// used, by the candidate machinery of the matrix-free map (candidates.cuh):
//
//   count pass   entries of row i = 1 (the diagonal) + its off-diagonal hits
//   host scan    row_ptr (int64), the total checked against the device budget
//   fill pass    row i: entry row_ptr[i] = (i, sum of the diagonal terms), then one entry
//                (j, sign * amp) per off-diagonal hit in candidate order; the value is
//                A + u B at the handle's current u (FP64), with an FP32 copy for c64 maps
//
// Rows are the output states, as in the map's H x (the reference's CSC columns are its input
// states; H is Hermitian, so both hold the same numbers).  An off-diagonal (row, column) pair
// reached by more than one term keeps one entry per term (the SpMV sums them); the reference
// merges such entries.  Dense H is therefore identical up to the rounding of that sum.
//
// SpMV: one warp per row, lanes stride over the row's entries four at a time (column and value
// streams coalesced, the x gathers in flight together), shuffle reduction, no atomics.  It
// streams 4 + s bytes per entry from HBM (column, value) and gathers x, which stays in L2 for
// sectors up to a few million states.
//
// For H(u) = A + u B the fill pass also keeps each entry's A and B parts in c64; the batched
// solver's block SpMV reads them for its FP32 maps (one u per right-hand side), accumulating
// the A and B products apart and scaling the B sum by u once per row as the matrix-free block
// map does.  A host matrix (create_gpu_matrix of the reference's host CSC) can be uploaded
// instead of built (upload_sparse), after validation of its row pointers and columns.
#include <algorithm>
#include <cstdlib>
#include <string>

#include "blockio.cuh"

namespace momed {

namespace {

__global__ void __launch_bounds__(kWarps * 32)
k_sparse_count(IndexView iv, OpView ov, int32_t* __restrict__ counts, int64_t rows) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpScratch& ws = s_ws[wid];
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        int nh = 0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                if (f < total) {
                    int t;
                    bool neg;
                    int64_t j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                    if (j >= 0 && j != row) ++nh;
                }
            }
            __syncwarp();
        });
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nh += __shfl_xor_sync(kFull, nh, o);
        if (lane == 0) counts[row] = 1 + nh;
    }
}

// bad[0]: entries that fell outside their row's range (count and fill passes disagree)
// pa32 / pb32 (HAS_B only, may be null): the A and B parts of each entry, rounded to c64
template <bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_sparse_fill(IndexView iv, OpView ov, const double* __restrict__ u_ptr, const int64_t* __restrict__ row_ptr,
              int32_t* __restrict__ col, double2* __restrict__ val, float2* __restrict__ val32,
              float2* __restrict__ pa32, float2* __restrict__ pb32, int64_t rows, unsigned long long* bad) {
    __shared__ SharedTables sh;
    __shared__ WarpScratch s_ws[kWarps];
    stage_tables(sh, iv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    WarpScratch& ws = s_ws[wid];
    const double u = HAS_B ? *u_ptr : 0.0;
    unsigned long long nbad = 0;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const uint64_t s = __ldg(iv.basis + row);
        const int64_t base = row_ptr[row], end = row_ptr[row + 1];
        int64_t pos = base + 1;            // warp-uniform: next free entry of the row
        double dr = 0.0, di = 0.0, dar = 0.0, dai = 0.0, dbr = 0.0, dbi = 0.0;
        for_each_group_batch(s, ov, [&](int g) {
            int total = stage_batch(g, ov, ws);
            int gi = 0;
            for (int f0 = 0; f0 < total; f0 += 32) {
                int f = f0 + lane;
                int64_t j = -1;
                int t = 0;
                bool neg = false;
                if (f < total) j = eval_term(f, gi, s, row, ov, iv, ws, sh, t, neg);
                double2 a = make_double2(0.0, 0.0), ta = a, tb = a;   // a = A + u B, ta = A, tb = B
                if (j >= 0) {
                    ta = load_amp(ov.t_amp, t);
                    if (neg) { ta.x = -ta.x; ta.y = -ta.y; }
                    a = ta;
                    if (HAS_B) {
                        tb = load_amp(ov.t_ampb, t);
                        if (neg) { tb.x = -tb.x; tb.y = -tb.y; }
                        a.x += u * tb.x;
                        a.y += u * tb.y;
                    }
                }
                if (j == row) {
                    dr += a.x; di += a.y;
                    dar += ta.x; dai += ta.y;
                    dbr += tb.x; dbi += tb.y;
                }
                const bool off = j >= 0 && j != row;
                const unsigned m = __ballot_sync(kFull, off);
                if (off) {
                    const int64_t p = pos + __popc(m & lt);
                    if (p < end) {
                        col[p] = (int32_t)j;
                        val[p] = a;
                        val32[p] = make_float2((float)a.x, (float)a.y);
                        if (HAS_B && pa32) {
                            pa32[p] = make_float2((float)ta.x, (float)ta.y);
                            pb32[p] = make_float2((float)tb.x, (float)tb.y);
                        }
                    } else {
                        ++nbad;
                    }
                }
                pos += __popc(m);
            }
            __syncwarp();
        });
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dr += __shfl_xor_sync(kFull, dr, o);
            di += __shfl_xor_sync(kFull, di, o);
            if (HAS_B) {
                dar += __shfl_xor_sync(kFull, dar, o);
                dai += __shfl_xor_sync(kFull, dai, o);
                dbr += __shfl_xor_sync(kFull, dbr, o);
                dbi += __shfl_xor_sync(kFull, dbi, o);
            }
        }
        if (lane == 0) {
            if (base < end) {
                col[base] = (int32_t)row;
                val[base] = make_double2(dr, di);
                val32[base] = make_float2((float)dr, (float)di);
                if (HAS_B && pa32) {
                    pa32[base] = make_float2((float)dar, (float)dai);
                    pb32[base] = make_float2((float)dbr, (float)dbi);
                }
            }
            if (pos != end) ++nbad;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nbad += __shfl_xor_sync(kFull, nbad, o);
    if (lane == 0 && nbad) atomicAdd(bad, nbad);
}

template <typename R> struct SpVal;
template <> struct SpVal<double> { using T = double2; };
template <> struct SpVal<float> { using T = float2; };

// Streaming loads of the column and value arrays: read once per SpMV, so they are not allocated
// in L1, which keeps it for the x gathers (ld.global.nc.L1::no_allocate).
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) {
    int32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double2 ld_stream(const double2* p) {
    double2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float2 ld_stream(const float2* p) {
    float2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}
template <bool STREAM, typename T> __device__ __forceinline__ T ld_cv(const T* p) {
    if constexpr (STREAM) return ld_stream(p);
    else return __ldg(p);
}

template <typename R, bool STREAM>
__global__ void __launch_bounds__(kWarps * 32)
k_spmv(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col, const typename SpVal<R>::T* __restrict__ val,
       const typename SpVal<R>::T* __restrict__ x, typename SpVal<R>::T* __restrict__ y, int64_t rows) {
    using C2 = typename SpVal<R>::T;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const int64_t b = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
        R ar = 0, ai = 0;
        int64_t p = b + lane;
        for (; p + 96 < e; p += 128) {      // four entries per lane in flight
            int c[4];
            C2 v[4], xv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                c[q] = ld_cv<STREAM>(col + p + 32 * q);
                v[q] = ld_cv<STREAM>(val + p + 32 * q);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) xv[q] = __ldg(x + c[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ar += v[q].x * xv[q].x - v[q].y * xv[q].y;
                ai += v[q].x * xv[q].y + v[q].y * xv[q].x;
            }
        }
        for (; p < e; p += 32) {
            const int c = ld_cv<STREAM>(col + p);
            const C2 v = ld_cv<STREAM>(val + p), xv = __ldg(x + c);
            ar += v.x * xv.x - v.y * xv.y;
            ai += v.x * xv.y + v.y * xv.x;
        }
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

// Block SpMV for the batched solver: NB right-hand sides interleaved as x[row * NB + r], the
// operator of right-hand side r is A + u[r] B (u null: val32 for all).  Each entry's NB values
// are read by NB / RPL lanes, RPL = min(NB, 4) values per lane (16-byte loads, laid out as
// blockio.cuh describes), so a warp iteration consumes 32 RPL / NB entries, two iterations in
// flight.
template <int NB, bool HAS_B>
__global__ void __launch_bounds__(kWarps * 32)
k_block_spmv(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col, const float2* __restrict__ pa,
             const float2* __restrict__ pb, const float2* __restrict__ x, float2* __restrict__ y,
             const float* __restrict__ u, int64_t rows) {
    using IO = BlkIO<float, NB>;
    constexpr int RPL = IO::RPL;
    constexpr int LPH = IO::LPH;       // lanes per entry
    constexpr int HPI = IO::HPI;       // entries per warp iteration
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hslot = lane / LPH, kk = lane % LPH;
    float ur[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) ur[q] = HAS_B ? __ldg(u + IO::rhs(kk, q)) : 0.f;
    auto entry = [&](int64_t p, float2* acc, float2* accb) {
        const int c = __ldg(col + p);
        const float2 a = __ldg(pa + p);
        float2 b = make_float2(0.f, 0.f);
        if (HAS_B) b = __ldg(pb + p);
        float2 xv[RPL];
        load_lane<float, NB>(x + (int64_t)c * NB, kk, xv);
#pragma unroll
        for (int q = 0; q < RPL; ++q) {     // A and B parts apart; B is scaled by u once per row
            acc[q].x += a.x * xv[q].x - a.y * xv[q].y;
            acc[q].y += a.x * xv[q].y + a.y * xv[q].x;
            if (HAS_B) {
                accb[q].x += b.x * xv[q].x - b.y * xv[q].y;
                accb[q].y += b.x * xv[q].y + b.y * xv[q].x;
            }
        }
    };
    for (int64_t row = (int64_t)blockIdx.x * kWarps + wid; row < rows; row += (int64_t)gridDim.x * kWarps) {
        const int64_t b0 = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
        float2 acc[RPL], accb[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            acc[q] = make_float2(0.f, 0.f);
            accb[q] = make_float2(0.f, 0.f);
        }
        int64_t p = b0 + hslot;
        for (; p + HPI < e; p += 2 * HPI) {
            entry(p, acc, accb);
            entry(p + HPI, acc, accb);
        }
        if (p < e) entry(p, acc, accb);
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            if (HAS_B) {
                acc[q].x += ur[q] * accb[q].x;
                acc[q].y += ur[q] * accb[q].y;
            }
#pragma unroll
            for (int o = LPH; o < 32; o <<= 1) {
                acc[q].x += __shfl_xor_sync(kFull, acc[q].x, o);
                acc[q].y += __shfl_xor_sync(kFull, acc[q].y, o);
            }
        }
        if (hslot == 0) store_lane<float, NB>(y + row * NB, kk, acc);
    }
}

__global__ void k_round_c64(const double2* __restrict__ v, float2* __restrict__ o, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        o[i] = make_float2((float)v[i].x, (float)v[i].y);
}

// MOMED_SPMV_STREAM=0 reads the column and value arrays through L1 like the x gathers
bool spmv_stream() {
    static const bool on = [] {
        const char* e = std::getenv("MOMED_SPMV_STREAM");
        return !(e && e[0] == '0');
    }();
    return on;
}

int spmv_grid(int64_t rows) {
    static const int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    int64_t need = (rows + kWarps - 1) / kWarps;
    return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * 8));   // 8 blocks of 8 warps per SM
}

}  // namespace

// column, FP64 value and its FP32 rounding; a parametrised operator also keeps A and B in c64
int64_t sparse_bytes_per_entry(bool pair) { return 4 + 16 + 8 + (pair ? 16 : 0); }

void build_sparse(momed_handle* h, double u) {
    SparseMatrix& sp = h->sparse;
    sp.release();
    h->hcache.release();          // maps read the matrix while it is built
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    MOMED_REQUIRE(n <= (int64_t)INT32_MAX, MOMED_EINVAL, "sparse method: basis larger than 2^31-1 states");
    const IndexView iv = index_view(h);
    const OpView ov = h->op.view();

    DevBuf<int32_t> counts;
    counts.resize(std::max<int64_t>(n, 1));
    k_sparse_count<<<persistent_grid(k_sparse_count, n), kWarps * 32, 0, st>>>(iv, ov, counts.p, n);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    std::vector<int32_t> hc(n);
    MOMED_CUDA_TRY(cudaMemcpyAsync(hc.data(), counts.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    counts.release();
    std::vector<int64_t> rp(n + 1);
    rp[0] = 0;
    for (int64_t i = 0; i < n; ++i) rp[i + 1] = rp[i] + hc[i];
    const int64_t nnz = rp[n];

    // admission: row pointers plus column, FP64 value and FP32 value per entry
    const bool hb = h->op.has_b;
    const int64_t need = (n + 1) * 8 + nnz * sparse_bytes_per_entry(hb);
    size_t free_b = 0, total_b = 0;
    MOMED_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    int64_t limit = (int64_t)(0.9 * (double)free_b);
    if (h->hbm_budget > 0) limit = std::min<int64_t>(limit, h->hbm_budget);
    if (need > limit)
        throw Error{MOMED_ENOMEM, "sparse method: the matrix needs " + std::to_string(need) + " bytes, " +
                                     std::to_string(limit) + " available"};

    sp.row_ptr.resize(n + 1);
    sp.col.resize(std::max<int64_t>(nnz, 1));
    sp.val.resize(std::max<int64_t>(nnz, 1));
    sp.val32.resize(std::max<int64_t>(nnz, 1));
    if (hb) {
        sp.pa32.resize(std::max<int64_t>(nnz, 1));
        sp.pb32.resize(std::max<int64_t>(nnz, 1));
    }
    MOMED_CUDA_TRY(cudaMemcpyAsync(sp.row_ptr.p, rp.data(), (n + 1) * 8, cudaMemcpyHostToDevice, st));
    h->counters.resize(16);
    MOMED_CUDA_TRY(cudaMemsetAsync(h->counters.p + 3, 0, sizeof(unsigned long long), st));
    DevBuf<double> ud;
    if (hb) {
        ud.resize(1);
        MOMED_CUDA_TRY(cudaMemcpyAsync(ud.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
        auto k = k_sparse_fill<true>;
        k<<<persistent_grid(k, n), kWarps * 32, 0, st>>>(iv, ov, ud.p, sp.row_ptr.p, sp.col.p, sp.val.p, sp.val32.p,
                                                          sp.pa32.p, sp.pb32.p, n, h->counters.p + 3);
    } else {
        auto k = k_sparse_fill<false>;
        k<<<persistent_grid(k, n), kWarps * 32, 0, st>>>(iv, ov, nullptr, sp.row_ptr.p, sp.col.p, sp.val.p, sp.val32.p,
                                                          nullptr, nullptr, n, h->counters.p + 3);
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    unsigned long long bad = 0;
    MOMED_CUDA_TRY(cudaMemcpyAsync(&bad, h->counters.p + 3, sizeof(bad), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad != 0) {
        sp.release();
        throw Error{MOMED_EINVAL, "sparse method: count and fill passes disagree on " + std::to_string(bad) + " rows"};
    }
    sp.nnz = nnz;
    sp.u = u;
    sp.built = true;
}

// A host CSR matrix (validated by the caller: row_ptr monotone from 0, columns in [0, n)).
void upload_sparse(momed_handle* h, int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val) {
    SparseMatrix& sp = h->sparse;
    sp.release();
    cudaStream_t st = h->stream;
    const int64_t nnz = row_ptr[n];
    const int64_t need = (n + 1) * 8 + nnz * sparse_bytes_per_entry(false);
    size_t free_b = 0, total_b = 0;
    MOMED_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    int64_t limit = (int64_t)(0.9 * (double)free_b);
    if (h->hbm_budget > 0) limit = std::min<int64_t>(limit, h->hbm_budget);
    if (need > limit)
        throw Error{MOMED_ENOMEM, "sparse method: the matrix needs " + std::to_string(need) + " bytes, " +
                                     std::to_string(limit) + " available"};
    sp.row_ptr.resize(n + 1);
    sp.col.resize(std::max<int64_t>(nnz, 1));
    sp.val.resize(std::max<int64_t>(nnz, 1));
    sp.val32.resize(std::max<int64_t>(nnz, 1));
    MOMED_CUDA_TRY(cudaMemcpyAsync(sp.row_ptr.p, row_ptr, (n + 1) * 8, cudaMemcpyHostToDevice, st));
    if (nnz > 0) {
        MOMED_CUDA_TRY(cudaMemcpyAsync(sp.col.p, col, nnz * 4, cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(sp.val.p, val, nnz * 16, cudaMemcpyHostToDevice, st));
        const int g = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 16);
        k_round_c64<<<g, 256, 0, st>>>(sp.val.p, sp.val32.p, nnz);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(1);
    }
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    sp.nnz = nnz;
    sp.u = h->u;
    sp.built = true;
}

void launch_spmv_c128(const SparseMatrix& sp, const double2* x, double2* y, int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    if (spmv_stream()) k_spmv<double, true><<<spmv_grid(rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, sp.val.p, x, y, rows);
    else k_spmv<double, false><<<spmv_grid(rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, sp.val.p, x, y, rows);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

void launch_spmv_c64(const SparseMatrix& sp, const float2* x, float2* y, int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    if (spmv_stream()) k_spmv<float, true><<<spmv_grid(rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, sp.val32.p, x, y, rows);
    else k_spmv<float, false><<<spmv_grid(rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, sp.val32.p, x, y, rows);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

}  // namespace momed

namespace momed {

void launch_block_spmv_c64(const SparseMatrix& sp, const float2* x, float2* y, const float* u, int32_t nb,
                           int64_t rows, cudaStream_t st) {
    if (rows <= 0) return;
    const bool hb = u != nullptr && sp.pb32.p != nullptr;
    const float2* pa = hb ? sp.pa32.p : sp.val32.p;
    // grid = the CTAs that are resident at once (the wide variants hold up to 70 registers, 3 CTAs
    // per SM): a grid-strided launch larger than that runs its surplus CTAs as a partial wave
#define MOMED_BSP(NBV)                                                                                   \
    case NBV:                                                                                            \
        if (hb) {                                                                                        \
            auto k = k_block_spmv<NBV, true>;                                                            \
            k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, pa, sp.pb32.p, x, y, u, rows); \
        } else {                                                                                         \
            auto k = k_block_spmv<NBV, false>;                                                           \
            k<<<persistent_grid(k, rows), kWarps * 32, 0, st>>>(sp.row_ptr.p, sp.col.p, pa, nullptr, x, y, nullptr, rows); \
        }                                                                                                \
        break;
    switch (nb) {
        MOMED_BSP(1)
        MOMED_BSP(2)
        MOMED_BSP(4)
        MOMED_BSP(8)
        MOMED_BSP(16)
        MOMED_BSP(32)
        default:
            throw Error{MOMED_EINVAL, "block width must be a power of two <= 32"};
    }
#undef MOMED_BSP
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

}  // namespace momed
