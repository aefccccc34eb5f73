// Block reorthogonalisation coefficients C = Q^H W on the 5th-generation tensor cores.
//
// The block Lanczos basis Q (ncol complex FP32 columns, stored as blocks [N][B]) is projected
// on the newest block W ([N][B]): C[c][r] = sum_n conj(Q_c[n]) W[n][r].  With complex values
// split into real and imaginary columns this is one real GEMM G = Qr^T Wr of shape
// (2 ncol) x (2B) over K = N rows, from which C[c][r] = (G[2c][2r] + G[2c+1][2r+1],
// G[2c][2r+1] - G[2c+1][2r]).  It is a real dense contraction with a shared operand (W for all
// basis columns), the one in the solver that belongs on the tensor pipe.
//
// Precision: FP32 inputs are split x = hi + lo, hi and lo rounded to TF32; tcgen05.mma
// kind::tf32 accumulates hi*hi + hi*lo + lo*hi in FP32 in tensor memory over 256 rows, and the
// accumulator is then added into FP64 registers, so the cross-chunk sum is FP64 and each
// product carries ~2^-21 relative error (the FP32 basis itself is rounded at 2^-24).
//
// Kernel layout: one CTA = 128 threads = one M tile of 128 real basis columns (64 complex) and
// one range of rows; grid (M tiles, row splits).  Per chunk of 32 rows the threads load Q and
// W with coalesced 16-byte loads, split them and write hi / lo tiles into shared memory in the
// K-major no-swizzle canonical layout (core matrices of 8 rows x 16 bytes; the stride between
// 8-row groups padded to 1040 bytes so the transposing stores do not collide on banks); one
// elected thread issues 12 MMAs (M 128, N 2B, K 8: four K steps x three split terms) and a
// commit to an mbarrier; every 8 chunks the 128 threads read their accumulator row back with
// tcgen05.ld and add it in FP64.  Each (tile, split) writes partial sums [split][c][r]; the
// caller reduces them over splits.  Every mbarrier wait is bounded (a timeout sets *err and
// the kernel frees its tensor memory and returns).
#include <algorithm>
#include <cstdint>

#include "momed_internal.cuh"

namespace momed {

namespace {

constexpr int kTcThreads = 128;
constexpr int kKC = 32;                         // rows (K) per staged chunk
constexpr int kFlush = 8;                       // chunks accumulated in tensor memory between FP64 flushes
constexpr int kLBO = 128;                       // bytes between K-adjacent core matrices
constexpr int kSBO = (kKC / 4) * 128 + 16;      // bytes between 8-row groups (padded: 1040)
constexpr int kTileA = 16 * kSBO;               // 128 rows
constexpr int kTileB = 4 * kSBO;                // up to 32 rows

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    // start address, leading / stride byte offsets (16-byte units), version 1, no swizzle
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// byte offset of element (row, k) of a K-major canonical tile
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
    return (uint32_t)((row >> 3) * kSBO + (k >> 2) * kLBO + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void put_split(unsigned char* hi, unsigned char* lo, int row, int k, float x) {
    const uint32_t h = to_tf32(x);
    const uint32_t l = to_tf32(x - __uint_as_float(h));
    const uint32_t o = tile_off(row, k);
    *reinterpret_cast<uint32_t*>(hi + o) = h;
    *reinterpret_cast<uint32_t*>(lo + o) = l;
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(phase)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 4000000000ll) return false;     // ~2 s: give up
    }
}

template <int B>
__global__ void __launch_bounds__(kTcThreads)
k_proj_tc(const float2* __restrict__ Q, int ncol, int64_t N, const float2* __restrict__ W, int64_t rows_per_split,
          double2* __restrict__ partial, int* __restrict__ err) {
    constexpr int NN = 2 * B;                     // MMA N: real columns of W
    constexpr uint32_t kIdesc = (1u << 4)         // D format F32
                                | (2u << 7)       // A format TF32
                                | (2u << 10)      // B format TF32
                                | ((uint32_t)(NN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* a_hi = smem;
    unsigned char* a_lo = smem + kTileA;
    unsigned char* b_hi = smem + 2 * kTileA;
    unsigned char* b_lo = smem + 2 * kTileA + kTileB;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;

    const int t = threadIdx.x, warp = t >> 5;
    const int c0 = blockIdx.x * 64;               // first complex basis column of this tile
    const int blk0 = c0 / B;
    const int nblk = (ncol + B - 1) / B;
    const int64_t r0 = (int64_t)blockIdx.y * rows_per_split;
    const int64_t r1 = r0 + rows_per_split < N ? r0 + rows_per_split : N;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&tmem_base)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        abort_flag = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    double acc[NN];
#pragma unroll
    for (int j = 0; j < NN; ++j) acc[j] = 0.0;
    uint32_t phase = 0;
    int in_group = 0;

    for (int64_t n0 = r0; n0 < r1; n0 += kKC) {
        // ---- stage Q (64 complex columns = 64/B blocks x kKC rows) and W (kKC rows) as hi / lo tiles
        constexpr int QF4 = (64 / B) * kKC * (B / 2);   // float4 units of the Q chunk
        for (int u = t; u < QF4; u += kTcThreads) {
            const int q = u % (B / 2), k = (u / (B / 2)) % kKC, bl = u / (kKC * (B / 2));
            const int64_t n = n0 + k;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n < r1 && blk0 + bl < nblk && c0 + bl * B + 2 * q < ncol)
                v = *reinterpret_cast<const float4*>(Q + ((size_t)(blk0 + bl) * N + n) * B + 2 * q);
            const int m = bl * NN + 4 * q;
            put_split(a_hi, a_lo, m, k, v.x);
            put_split(a_hi, a_lo, m + 1, k, v.y);
            put_split(a_hi, a_lo, m + 2, k, v.z);
            put_split(a_hi, a_lo, m + 3, k, v.w);
        }
        constexpr int WF4 = kKC * (B / 2);
        for (int u = t; u < WF4; u += kTcThreads) {
            const int q = u % (B / 2), k = u / (B / 2);
            const int64_t n = n0 + k;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n < r1) v = *reinterpret_cast<const float4*>(W + (size_t)n * B + 2 * q);
            const int m = 4 * q;
            put_split(b_hi, b_lo, m, k, v.x);
            put_split(b_hi, b_lo, m + 1, k, v.y);
            put_split(b_hi, b_lo, m + 2, k, v.z);
            put_split(b_hi, b_lo, m + 3, k, v.w);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic-proxy stores -> tensor core reads
        __syncthreads();
        // ---- MMAs: hi*hi, hi*lo, lo*hi over four K steps of 8
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bo = smem_u32(b_lo);
#pragma unroll
            for (int term = 0; term < 3; ++term) {
                const uint32_t abase = term == 2 ? al : ah;
                const uint32_t bbase = term == 1 ? bo : bh;
#pragma unroll
                for (int s = 0; s < kKC / 8; ++s) {
                    const uint64_t ad = umma_desc(abase + s * 2 * kLBO);
                    const uint64_t bd = umma_desc(bbase + s * 2 * kLBO);
                    const uint32_t accum = (in_group > 0 || term > 0 || s > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                        :
                        : "r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&mbar)) : "memory");
        }
        // the MMAs must finish before the tiles are rewritten (and before the accumulator is read)
        if (!mbar_wait(smem_u32(&mbar), phase)) abort_flag = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        ++in_group;
        const bool last = n0 + kKC >= r1;
        if (in_group == kFlush || last) {
            uint32_t v[NN];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);    // this warp's 32 lanes
            if constexpr (NN == 16) {
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(taddr));
            } else {
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < NN; ++j) acc[j] += (double)__uint_as_float(v[j]);
            in_group = 0;
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (abort_flag) break;
    }
    // ---- complex coefficients of this tile: thread 2c holds G[2c][*], thread 2c + 1 G[2c + 1][*]
    double odd[NN];
#pragma unroll
    for (int j = 0; j < NN; ++j) odd[j] = __shfl_down_sync(0xffffffffu, acc[j], 1);
    const int c = c0 + t / 2;
    if (!abort_flag && (t & 1) == 0 && c < ncol) {
        double2* out = partial + ((size_t)blockIdx.y * ncol + c) * B;
#pragma unroll
        for (int r = 0; r < B; ++r)
            out[r] = make_double2(acc[2 * r] + odd[2 * r + 1], acc[2 * r + 1] - odd[2 * r]);
    }
    if (abort_flag && t == 0) atomicExch(err, 1);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem));
}

}  // namespace

int proj_tc_smem_bytes() { return 2 * kTileA + 2 * kTileB + 1024; }

// Launch: partial[split][c][r] for splits < *nsplit (set here); B = 8 or 16.
void launch_proj_tc_c64(const float2* Q, int ncol, int64_t N, const float2* W, int B, double2* partial,
                        int max_splits, int* nsplit, int* err, cudaStream_t st) {
    const int mtiles = (ncol + 63) / 64;
    int64_t chunks = (N + kKC - 1) / kKC;
    int splits = (int)std::max<int64_t>(1, std::min<int64_t>(chunks / 8, (int64_t)max_splits / mtiles));
    int64_t rows = ((N + splits - 1) / splits + kKC - 1) / kKC * kKC;
    splits = (int)((N + rows - 1) / rows);
    *nsplit = splits;
    const int smem = proj_tc_smem_bytes();
    dim3 grid((unsigned)mtiles, (unsigned)splits);
    if (B == 8) {
        auto k = k_proj_tc<8>;
        MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k<<<grid, kTcThreads, smem, st>>>(Q, ncol, N, W, rows, partial, err);
    } else if (B == 16) {
        auto k = k_proj_tc<16>;
        MOMED_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k<<<grid, kTcThreads, smem, st>>>(Q, ncol, N, W, rows, partial, err);
    } else {
        throw Error{MOMED_EINVAL, "tensor-core projection: block size must be 8 or 16"};
    }
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
}

}  // namespace momed
