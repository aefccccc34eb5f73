// Kernel (a): per-momentum-sector basis enumeration.
//
// Reference: ED_momentum_subspaces (MomentumED/src/preparation/momentum_decomposition.jl:188-273)
// recurses over the conserved components, last component outermost and in the
// highest bits (accumulated_mbs * mbs_smaller, EDCore manybodystate_basis.jl:81-83),
// each component walked in colex order (EDCore colex_mbslist.jl), and pushes
// every state into the sector of its total momentum residue (init_parameter.jl:148-152).
// Walking the mixed-radix rank r = sum_c rank_c * stride_c (component 0 fastest)
// in increasing order yields the states in increasing uint64 order, so each
// sector's list comes out sorted exactly as the reference builds it.
//
// GPU scheme: the rank space is cut into one contiguous chunk per thread.  A
// thread unranks its chunk start (combinadic unranking per component) and then
// steps with the next-combination rule.  Pass 1 counts per (sector, block);
// the host scans those counts; pass 2 recounts, scans per sector inside the
// block and writes every state at its final position.
#include <algorithm>
#include <climits>
#include <mutex>
#include <numeric>

#include "momed_internal.cuh"

namespace momed {

namespace {

constexpr int kMaxComp = 8;
constexpr int kSecWin = 32;      // sectors handled per pass window
constexpr int kThreads = 256;

struct Comp {
    int32_t t;            // particles (|N|)
    int32_t len;          // available positions
    int32_t shift;        // first bit of the component
    int32_t masked;       // positions come from pos[] (mask) instead of 0..len-1
    int64_t count;        // C(len, t)
    int64_t stride;       // rank stride
    int8_t pos[64];       // bit offsets (within the component) of available positions
};

struct EnumParams {
    int32_t ncomp, dim;
    Comp comp[kMaxComp];
    int64_t total;        // product of counts
    int64_t chunk;        // ranks per thread
    int32_t kv[64][3];    // signed momentum of each global orbital (dim <= 3)
    int32_t Gk[3];
    int32_t box_lo[3];
    int32_t box_ext[3];
    const int32_t* sec_of; // [prod box_ext] sector id or -1
    const uint64_t* binom;  // [65 * 65] C(n, k) as uint64
    int64_t box_n;          // entries of sec_of
    int64_t out_cap;        // entries of the output buffer (write pass)
    unsigned long long* err; // [8]: count of out-of-range accesses found and skipped (must stay 0),
                             //      then kind, a, b, c of the first one
};

__host__ __device__ __forceinline__ void note_err(const EnumParams& P, long long kind = 0, long long a = 0,
                                                  long long b = 0, long long c = 0) {
#ifdef __CUDA_ARCH__
    if (P.err) {
        if (atomicAdd(P.err, 1ull) == 0ull) {
            P.err[1] = (unsigned long long)kind;
            P.err[2] = (unsigned long long)a;
            P.err[3] = (unsigned long long)b;
            P.err[4] = (unsigned long long)c;
        }
    }
#else
    if (P.err && (*P.err)++ == 0) { P.err[1] = kind; P.err[2] = a; P.err[3] = b; P.err[4] = c; }
#endif
}

// Helpers are host-callable too so the index arithmetic can be exercised on the CPU.
__host__ __device__ __forceinline__ int ffs64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __ffsll((long long)x);
#else
    return __builtin_ffsll((long long)x);
#endif
}
template <typename T>
__host__ __device__ __forceinline__ T ld_ro(const T* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

__host__ __device__ __forceinline__ uint64_t dbinom(const uint64_t* b, int n, int k) {
    return (k < 0 || n < 0 || k > n) ? 0ull : b[n * 65 + k];
}

// pattern (over len positions, t set bits) of the rank-th combination in colex order
__host__ __device__ uint64_t unrank_pattern(const uint64_t* binom, int len, int t, int64_t rank) {
    uint64_t pat = 0;
    int64_t x = rank;
    for (int i = t; i >= 1; --i) {
        int c = i - 1;
        while (c + 1 < len && (int64_t)dbinom(binom, c + 1, i) <= x) ++c;
        pat |= 1ull << c;
        x -= (int64_t)dbinom(binom, c, i);
    }
    return pat;
}

// next larger integer with the same popcount
__host__ __device__ __forceinline__ uint64_t next_comb(uint64_t x) {
    uint64_t c = x & (~x + 1ull);
    uint64_t r = x + c;
    return r | (((x ^ r) >> 2) >> (ffs64(c) - 1));
}

__host__ __device__ __forceinline__ uint64_t deposit(const Comp& c, uint64_t pat) {
    if (!c.masked) return pat << c.shift;
    uint64_t out = 0;
    while (pat) {
        int p = ffs64(pat) - 1;
        out |= 1ull << (c.shift + c.pos[p]);
        pat &= pat - 1ull;
    }
    return out;
}

__host__ __device__ __forceinline__ int sector_of(const EnumParams& P, uint64_t s) {
    int k[3] = {0, 0, 0};
    while (s) {
        int o = ffs64(s) - 1;
        for (int d = 0; d < P.dim && d < 3; ++d) k[d] += P.kv[o][d];
        s &= s - 1ull;
    }
    int64_t idx = 0, stride = 1;
    for (int d = 0; d < P.dim; ++d) {
        int v = k[d];
        if (P.Gk[d] != 0) { v %= P.Gk[d]; if (v < 0) v += P.Gk[d]; }
        v -= P.box_lo[d];
        if (v < 0 || v >= P.box_ext[d]) return -1;
        idx += (int64_t)v * stride;
        stride *= P.box_ext[d];
    }
    if (idx < 0 || idx >= P.box_n) { note_err(P, 1, idx, P.box_n, (long long)s); return -1; }
    return ld_ro(P.sec_of + idx);
}

// Iterator over ranks in increasing order (component 0 fastest, with carry).
struct Walker {
    uint64_t pat[kMaxComp], part[kMaxComp];
    int64_t rk[kMaxComp];
    uint64_t state;

    __host__ __device__ void init(const EnumParams& P, int64_t r0) {
        int64_t rem = r0;
        for (int c = P.ncomp - 1; c >= 0; --c) {
            rk[c] = rem / P.comp[c].stride;
            rem -= rk[c] * P.comp[c].stride;
        }
        state = 0;
        for (int c = 0; c < P.ncomp; ++c) {
            pat[c] = unrank_pattern(P.binom, P.comp[c].len, P.comp[c].t, rk[c]);
            part[c] = deposit(P.comp[c], pat[c]);
            state |= part[c];
        }
    }
    __host__ __device__ void advance(const EnumParams& P) {
        for (int c = 0; c < P.ncomp; ++c) {
            state &= ~part[c];
            if (rk[c] + 1 < P.comp[c].count) {
                ++rk[c];
                pat[c] = next_comb(pat[c]);
                part[c] = deposit(P.comp[c], pat[c]);
                state |= part[c];
                return;
            }
            rk[c] = 0;
            pat[c] = P.comp[c].t ? ((1ull << P.comp[c].t) - 1ull) : 0ull;
            part[c] = deposit(P.comp[c], pat[c]);
            state |= part[c];
        }
    }
};

__host__ __device__ __forceinline__ void thread_ranks(const EnumParams& P, int64_t tid, int64_t& r0, int64_t& r1) {
    r0 = tid * P.chunk;
    r1 = r0 + P.chunk;
    if (r1 > P.total) r1 = P.total;
    if (r0 > r1) r0 = r1;
}

// Per-thread sector counts of the block live in shared memory: cnt[sector][thread].
struct EnumShared {
    EnumParams P;
    int32_t cnt[kSecWin][kThreads];
};

__device__ void count_chunk(EnumShared& sh, int win0, int nwin, int64_t r0, int64_t r1) {
    const int t = threadIdx.x;
    for (int i = 0; i < kSecWin; ++i) sh.cnt[i][t] = 0;
    if (r0 >= r1) return;
    Walker w;
    w.init(sh.P, r0);
    for (int64_t r = r0; r < r1; ++r) {
        int sec = sector_of(sh.P, w.state) - win0;
        if (sec >= 0 && sec < nwin) sh.cnt[sec][t] += 1;
        if (r + 1 < r1) w.advance(sh.P);
    }
}

__global__ void __launch_bounds__(kThreads)
k_enum_count(EnumParams Pp, int win0, int nwin, int32_t* block_counts /* [kSecWin][nblocks] */) {
    __shared__ EnumShared sh;
    if (threadIdx.x == 0) sh.P = Pp;
    __syncthreads();
    int64_t r0, r1;
    thread_ranks(sh.P, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, r0, r1);
    count_chunk(sh, win0, nwin, r0, r1);
    __syncthreads();
    if (threadIdx.x < nwin) {
        int32_t s = 0;
        for (int t = 0; t < kThreads; ++t) s += sh.cnt[threadIdx.x][t];
        block_counts[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kThreads)
k_enum_write(EnumParams Pp, int win0, int nwin, const int64_t* block_offsets /* [kSecWin][nblocks] */, uint64_t* out) {
    __shared__ EnumShared sh;
    if (threadIdx.x == 0) sh.P = Pp;
    __syncthreads();
    int64_t r0, r1;
    thread_ranks(sh.P, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, r0, r1);
    count_chunk(sh, win0, nwin, r0, r1);
    __syncthreads();
    // exclusive scan of each sector's row over the block's threads (thread order = rank order)
    if (threadIdx.x < nwin) {
        int32_t run = 0;
        for (int t = 0; t < kThreads; ++t) {
            int32_t v = sh.cnt[threadIdx.x][t];
            sh.cnt[threadIdx.x][t] = run;
            run += v;
        }
    }
    __syncthreads();
    if (r0 >= r1) return;
    const int t = threadIdx.x;
    Walker w;
    w.init(sh.P, r0);
    for (int64_t r = r0; r < r1; ++r) {
        uint64_t s = w.state;
        int sec = sector_of(sh.P, s) - win0;
        if (sec >= 0 && sec < nwin) {
            int64_t p = block_offsets[(int64_t)sec * gridDim.x + blockIdx.x] + sh.cnt[sec][t];
            sh.cnt[sec][t] += 1;
            if (p >= 0 && p < sh.P.out_cap) out[p] = s;
            else note_err(sh.P, 2, p, sh.P.out_cap, sec);
        }
        if (r + 1 < r1) w.advance(sh.P);
    }
}

int64_t hbinom(int n, int k) {
    if (k < 0 || n < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    __int128 r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r > (__int128)INT64_MAX ? INT64_MAX : (int64_t)r;
}

int64_t jmod(int64_t a, int64_t g) { int64_t r = a % g; return r < 0 ? r + g : r; }

}  // namespace

// Host-side plan of one enumeration: kernel parameters (device pointers left null),
// the sector momenta in the reference order, the momentum-box -> sector table and
// the launch shape.
struct EnumPlan {
    EnumParams P{};
    int dim = 0;
    std::vector<int64_t> moms;      // [nsec * dim]
    int64_t nsec = 0;
    std::vector<int32_t> sec_of;    // [box_n]
    std::vector<uint64_t> binom;    // [65 * 65]
    int nblocks = 1;
};

EnumPlan plan_enumeration(const momed_para* p, const int64_t* N_each, int ncc, const int64_t* mask, int mlen,
                          const int64_t* momentum_list, int nmom) {
    MOMED_REQUIRE(p && p->k_list && p->Gk, MOMED_EINVAL, "para, k_list and Gk are required");
    MOMED_REQUIRE(ncc == p->Nc_conserve && ncc >= 1 && ncc <= kMaxComp, MOMED_EINVAL,
                  "length of N_each must equal Nc_conserve (<= 8)");
    MOMED_REQUIRE(p->dim >= 1 && p->dim <= 3, MOMED_EINVAL, "dim must be 1..3");
    const int dim = p->dim, Nk = p->Nk;
    const int ncomp_bits = Nk * p->Nc_mix;
    MOMED_REQUIRE((int64_t)ncomp_bits * ncc <= 64 && Nk >= 1, MOMED_EINVAL, "Nk * Nc must be <= 64");

    EnumPlan plan{};
    plan.dim = dim;
    EnumParams& P = plan.P;
    P.ncomp = ncc;
    P.dim = dim;
    for (int d = 0; d < dim; ++d) P.Gk[d] = (int32_t)p->Gk[d];

    // components (component 0 = N_each[0] = lowest bits)
    std::vector<int64_t> smask;
    if (mask && mlen >= 0) { smask.assign(mask, mask + mlen); std::sort(smask.begin(), smask.end()); }
    int64_t total = 1;
    for (int c = 0; c < ncc; ++c) {
        Comp& C = P.comp[c];
        int64_t Nc = N_each[c];
        C.t = (int32_t)(Nc < 0 ? -Nc : Nc);
        C.shift = c * ncomp_bits;
        if (mask && mlen >= 0) {
            C.masked = 1;
            C.len = 0;
            for (int64_t m : smask) {
                int64_t rel = m - (int64_t)c * ncomp_bits;
                if (rel >= 1 && rel <= ncomp_bits) C.pos[C.len++] = (int8_t)(rel - 1);
            }
        } else {
            C.masked = 0;
            C.len = ncomp_bits;
            for (int i = 0; i < ncomp_bits; ++i) C.pos[i] = (int8_t)i;
        }
        MOMED_REQUIRE(C.t <= ncomp_bits, MOMED_EINVAL, "Invalid number of electrons in one component");
        C.count = hbinom(C.len, C.t);
        C.stride = total;
        MOMED_REQUIRE(C.count == 0 || total <= INT64_MAX / std::max<int64_t>(C.count, 1), MOMED_EINVAL,
                      "combination space too large");
        total *= C.count;
        int sgn = Nc > 0 ? 1 : (Nc < 0 ? -1 : 0);
        for (int i = 0; i < ncomp_bits; ++i) {
            int ik = i % Nk;
            for (int d = 0; d < dim; ++d) P.kv[C.shift + i][d] = sgn * (int32_t)p->k_list[d + dim * ik];
        }
    }
    P.total = total;

    // momentum list in the reference order
    std::vector<int64_t> moms;   // [nsec * dim]
    int64_t Ntot = 0;
    for (int c = 0; c < ncc; ++c) Ntot += N_each[c];
    if (nmom >= 0) {
        for (int s = 0; s < nmom; ++s) {
            int64_t r[3];
            for (int d = 0; d < dim; ++d)
                r[d] = p->Gk[d] == 0 ? momentum_list[s * dim + d] : jmod(momentum_list[s * dim + d], p->Gk[d]);
            bool dup = false;
            for (size_t u = 0; u < moms.size() / dim && !dup; ++u) {
                bool eq = true;
                for (int d = 0; d < dim; ++d) eq = eq && moms[u * dim + d] == r[d];
                dup = eq;
            }
            if (!dup) moms.insert(moms.end(), r, r + dim);
        }
    } else {
        int64_t lo[3], cnt[3];
        int64_t nsec = 1;
        for (int d = 0; d < dim; ++d) {
            if (p->Gk[d] == 0) {
                int64_t mn = INT64_MAX, mx = INT64_MIN;
                for (int i = 0; i < Nk; ++i) { mn = std::min(mn, p->k_list[d + dim * i]); mx = std::max(mx, p->k_list[d + dim * i]); }
                lo[d] = mn * Ntot;
                cnt[d] = std::max<int64_t>(0, mx * Ntot - mn * Ntot + 1);
            } else {
                lo[d] = 0;
                cnt[d] = p->Gk[d];
            }
            nsec *= cnt[d];
        }
        MOMED_REQUIRE(nsec <= (1 << 20), MOMED_EINVAL, "too many momentum sectors");
        for (int64_t s = 0; s < nsec; ++s) {
            int64_t r = s;
            for (int d = 0; d < dim; ++d) { moms.push_back(lo[d] + r % cnt[d]); r /= cnt[d]; }
        }
    }
    const int64_t nsec = (int64_t)moms.size() / dim;

    // box of reachable (residue or raw) momenta and its sector table
    int64_t box_n = 1;
    for (int d = 0; d < dim; ++d) {
        if (p->Gk[d] != 0) { P.box_lo[d] = 0; P.box_ext[d] = (int32_t)p->Gk[d]; }
        else {
            int64_t lo = 0, hi = 0;
            for (int c = 0; c < ncc; ++c) {
                std::vector<int64_t> v;
                for (int i = 0; i < P.comp[c].len; ++i) v.push_back(P.kv[P.comp[c].shift + P.comp[c].pos[i]][d]);
                std::sort(v.begin(), v.end());
                for (int i = 0; i < P.comp[c].t && i < (int)v.size(); ++i) { lo += v[i]; hi += v[v.size() - 1 - i]; }
            }
            P.box_lo[d] = (int32_t)lo;
            P.box_ext[d] = (int32_t)(hi - lo + 1);
        }
        box_n *= P.box_ext[d];
    }
    MOMED_REQUIRE(box_n <= (1 << 24), MOMED_EINVAL, "momentum box too large");
    std::vector<int32_t> sec_of(box_n, -1);
    for (int64_t s = 0; s < nsec; ++s) {
        int64_t idx = 0, stride = 1;
        bool in = true;
        for (int d = 0; d < dim; ++d) {
            int64_t v = moms[s * dim + d] - P.box_lo[d];
            if (v < 0 || v >= P.box_ext[d]) { in = false; break; }
            idx += v * stride;
            stride *= P.box_ext[d];
        }
        if (in) sec_of[idx] = (int32_t)s;
    }
    plan.binom.assign(65 * 65, 0);
    for (int n = 0; n <= 64; ++n)
        for (int k = 0; k <= n; ++k) plan.binom[n * 65 + k] = (uint64_t)hbinom(n, k);
    plan.nblocks = 1;
    P.chunk = 16;
    if (total > 0) {
        int64_t threads_target = (int64_t)148 * 2048;
        P.chunk = std::max<int64_t>(16, (total + threads_target - 1) / threads_target);
        int64_t nthreads = (total + P.chunk - 1) / P.chunk;
        plan.nblocks = (int)((nthreads + kThreads - 1) / kThreads);
    }
    plan.moms = std::move(moms);
    plan.nsec = nsec;
    plan.sec_of = std::move(sec_of);
    return plan;
}

void enumerate_basis(momed_handle* h, const momed_para* p, const int64_t* N_each, int ncc, const int64_t* mask,
                     int mlen, const int64_t* momentum_list, int nmom) {
    EnumPlan plan = plan_enumeration(p, N_each, ncc, mask, mlen, momentum_list, nmom);
    EnumParams& P = plan.P;
    const int dim = plan.dim;
    const int64_t nsec = plan.nsec;
    const int64_t total = P.total;
    const int nblocks = plan.nblocks;
    const std::vector<int64_t>& moms = plan.moms;
    cudaStream_t st = h->stream;
    DevBuf<int32_t> d_sec;
    d_sec.resize(plan.sec_of.size());
    MOMED_CUDA_TRY(cudaMemcpyAsync(d_sec.p, plan.sec_of.data(), plan.sec_of.size() * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, st));
    P.sec_of = d_sec.p;
    DevBuf<uint64_t> d_binom;
    d_binom.resize(plan.binom.size());
    MOMED_CUDA_TRY(cudaMemcpyAsync(d_binom.p, plan.binom.data(), plan.binom.size() * 8, cudaMemcpyHostToDevice, st));
    P.binom = d_binom.p;
    P.box_n = (int64_t)plan.sec_of.size();
    P.out_cap = 0;
    DevBuf<unsigned long long> d_err;
    d_err.resize(8);
    MOMED_CUDA_TRY(cudaMemsetAsync(d_err.p, 0, 8 * sizeof(unsigned long long), st));
    P.err = d_err.p;

    Enumeration& E = h->enumer;
    E.dim = dim;
    E.sizes.assign(nsec, 0);
    E.offsets.assign(nsec + 1, 0);
    E.sector_k.clear();
    // pass 1: counts per window of sectors
    std::vector<int64_t> counts(nsec * (int64_t)nblocks, 0);   // [sector][block]
    if (total > 0) {
        DevBuf<int32_t> d_cnt;
        d_cnt.resize((size_t)kSecWin * nblocks);
        std::vector<int32_t> hc((size_t)kSecWin * nblocks);
        for (int64_t w0 = 0; w0 < nsec; w0 += kSecWin) {
            int nwin = (int)std::min<int64_t>(kSecWin, nsec - w0);
            k_enum_count<<<nblocks, kThreads, 0, st>>>(P, (int)w0, nwin, d_cnt.p);
            MOMED_CUDA_TRY(cudaGetLastError());
            MOMED_CUDA_TRY(cudaMemcpyAsync(hc.data(), d_cnt.p, (size_t)nwin * nblocks * 4, cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            for (int i = 0; i < nwin; ++i)
                for (int b = 0; b < nblocks; ++b) counts[(w0 + i) * nblocks + b] = hc[(size_t)i * nblocks + b];
        }
    }
    // sector sizes and block offsets (sector-major concatenation)
    std::vector<int64_t> offs(counts.size(), 0);
    int64_t run = 0;
    for (int64_t s = 0; s < nsec; ++s) {
        E.offsets[s] = run;
        for (int b = 0; b < nblocks; ++b) { offs[s * nblocks + b] = run; run += counts[s * nblocks + b]; }
        E.sizes[s] = run - E.offsets[s];
    }
    E.offsets[nsec] = run;
    E.states.release();
    P.out_cap = run;
    if (run > 0) {
        E.states.resize(run);
        DevBuf<int64_t> d_off;
        d_off.resize((size_t)kSecWin * nblocks);
        for (int64_t w0 = 0; w0 < nsec; w0 += kSecWin) {
            int nwin = (int)std::min<int64_t>(kSecWin, nsec - w0);
            MOMED_CUDA_TRY(cudaMemcpyAsync(d_off.p, offs.data() + w0 * nblocks, (size_t)nwin * nblocks * 8,
                                           cudaMemcpyHostToDevice, st));
            k_enum_write<<<nblocks, kThreads, 0, st>>>(P, (int)w0, nwin, d_off.p, E.states.p);
            MOMED_CUDA_TRY(cudaGetLastError());
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        }
    }
    // drop empty sectors (momentum_decomposition.jl:408-410)
    std::vector<int64_t> ks, sz, of;
    for (int64_t s = 0; s < nsec; ++s) {
        if (E.sizes[s] == 0) continue;
        ks.insert(ks.end(), moms.begin() + s * dim, moms.begin() + (s + 1) * dim);
        sz.push_back(E.sizes[s]);
        of.push_back(E.offsets[s]);
    }
    of.push_back(run);
    E.sector_k = ks;
    E.sizes = sz;
    E.offsets = of;
    unsigned long long herr[8] = {0};
    MOMED_CUDA_TRY(cudaMemcpyAsync(herr, d_err.p, sizeof(herr), cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr[0] != 0) {
        std::string msg = "basis enumeration skipped " + std::to_string(herr[0]) + " out-of-range accesses; first: kind " +
                          std::to_string((long long)herr[1]) + " values " + std::to_string((long long)herr[2]) + " " +
                          std::to_string((long long)herr[3]) + " " + std::to_string((long long)herr[4]) +
                          "; sector sizes:";
        for (size_t s = 0; s < E.sizes.size() && s < 40; ++s) msg += " " + std::to_string(E.sizes[s]);
        msg += "; chunk " + std::to_string(P.chunk) + " blocks " + std::to_string(nblocks) + " total " +
               std::to_string(total);
        throw Error{MOMED_ECUDA, msg};
    }
}

// ---------------------------------------------------------------------------------------
// Enumeration of one sector that allocates no device memory.
//
// For callers that cannot call cudaMalloc: hosts whose device memory is owned by another
// allocator (a Julia CUDA.jl memory pool, a framework's caching allocator) that hands this
// library only the output buffer, and services that reserve all of HBM up front for their
// solve slots and allow no allocation afterwards.  The caller passes the output buffer; the
// working space (binomial table, momentum-to-sector table, per-block counts and offsets,
// error counters and the state count) lives in the static array below, 148,864 bytes that
// every GPU that loads the library keeps until the process exits.
//
// The first call on a device looks the array's device address up (cudaGetSymbolAddress,
// with that device current); make that first call before any stream capture.  Every call
// shares the array and it keeps the last call's contents: the error counters and the count
// are cleared at the start of each call, and calls that overlap on the GPU (two streams, two
// host threads) race on it.
// ---------------------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxBox = 4096;      // momentum-box entries (sector table)
constexpr int kNoAllocMaxBlocks = 8192;   // grid blocks of the count / write passes
constexpr size_t kNoAllocBinomOff = 0;                                            // uint64 [65 * 65]
constexpr size_t kNoAllocSecOff = 34048;                                          // int32  [kNoAllocMaxBox]
constexpr size_t kNoAllocCntOff = kNoAllocSecOff + 4 * kNoAllocMaxBox;            // int32  [kNoAllocMaxBlocks]
constexpr size_t kNoAllocOffOff = kNoAllocCntOff + 4 * kNoAllocMaxBlocks;         // int64  [kNoAllocMaxBlocks]
constexpr size_t kNoAllocErrOff = kNoAllocOffOff + 8 * kNoAllocMaxBlocks;         // uint64 [8] errors, [8] total
constexpr size_t kNoAllocBytes = kNoAllocErrOff + 16 * 8;                         // 148,864 bytes
static_assert(kNoAllocBytes == 148864, "the documented size of the no-allocation scratch array");
static_assert(kNoAllocSecOff >= 65 * 65 * 8 && kNoAllocSecOff % 256 == 0, "binomial table overlaps the sector table");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// exclusive scan of the per-block counts (one block; nblocks <= kNoAllocMaxBlocks)
__global__ void k_noalloc_scan(const int32_t* counts, int nblocks, int64_t* offsets, unsigned long long* total) {
    __shared__ int64_t part[1024];
    const int t = threadIdx.x;
    const int per = (nblocks + 1023) / 1024;
    int64_t s = 0;
    for (int i = t * per; i < min(nblocks, (t + 1) * per); ++i) s += counts[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        int64_t run = 0;
        for (int i = 0; i < 1024; ++i) { int64_t v = part[i]; part[i] = run; run += v; }
        *total = (unsigned long long)run;
    }
    __syncthreads();
    int64_t run = part[t];
    for (int i = t * per; i < min(nblocks, (t + 1) * per); ++i) { offsets[i] = run; run += counts[i]; }
}

// Device address of the scratch array, looked up once per device (with that device current).
unsigned char* noalloc_scratch(int dev) {
    static std::mutex mu;
    static unsigned char* addr[64] = {nullptr};
    std::lock_guard<std::mutex> lk(mu);
    MOMED_REQUIRE(dev >= 0 && dev < 64, MOMED_ENODEV, "device index out of range");
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw Error{MOMED_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)};
        addr[dev] = static_cast<unsigned char*>(p);
    }
    return addr[dev];
}

}  // namespace

}  // namespace momed

extern "C" MOMED_API int momed_enumerate_sector_noalloc(const momed_para* p, const int64_t* N_each, int32_t ncc,
                                                        const int64_t* momentum, uint64_t* out_dev,
                                                        int64_t out_capacity, int64_t* n_states, void* cuda_stream) {
    using namespace momed;
    try {
        MOMED_REQUIRE(p && p->k_list && p->Gk && N_each && momentum && n_states, MOMED_EINVAL, "null argument");
        MOMED_REQUIRE(ncc == p->Nc_conserve && ncc >= 1 && ncc <= kMaxComp, MOMED_EINVAL,
                      "length of N_each must equal Nc_conserve (<= 8)");
        MOMED_REQUIRE(p->dim >= 1 && p->dim <= 3, MOMED_EINVAL, "dim must be 1..3");
        const int dim = p->dim, Nk = p->Nk, ncomp_bits = Nk * p->Nc_mix;
        MOMED_REQUIRE(Nk >= 1 && (int64_t)ncomp_bits * ncc <= 64, MOMED_EINVAL, "Nk * Nc must be <= 64");
        int dev = 0;
        MOMED_CUDA_TRY(cudaGetDevice(&dev));
        unsigned char* scratch = noalloc_scratch(dev);
        cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

        // kernel parameters, planned on the stack (no heap, no device allocation)
        EnumParams P{};
        P.ncomp = ncc;
        P.dim = dim;
        for (int d = 0; d < dim; ++d) P.Gk[d] = (int32_t)p->Gk[d];
        int64_t total = 1;
        for (int c = 0; c < ncc; ++c) {
            Comp& C = P.comp[c];
            int64_t Nc = N_each[c];
            C.t = (int32_t)(Nc < 0 ? -Nc : Nc);
            C.shift = c * ncomp_bits;
            C.masked = 0;
            C.len = ncomp_bits;
            for (int i = 0; i < ncomp_bits; ++i) C.pos[i] = (int8_t)i;
            MOMED_REQUIRE(C.t <= ncomp_bits, MOMED_EINVAL, "Invalid number of electrons in one component");
            C.count = hbinom(C.len, C.t);
            C.stride = total;
            MOMED_REQUIRE(C.count == 0 || total <= (int64_t(1) << 62) / std::max<int64_t>(C.count, 1), MOMED_EINVAL,
                          "combination space too large");
            total *= C.count;
            int sgn = Nc > 0 ? 1 : (Nc < 0 ? -1 : 0);
            for (int i = 0; i < ncomp_bits; ++i)
                for (int d = 0; d < dim; ++d) P.kv[C.shift + i][d] = sgn * (int32_t)p->k_list[d + dim * (i % Nk)];
        }
        P.total = total;
        int64_t box_n = 1;
        int64_t target = 0, tstride = 1;
        bool target_in = true;
        for (int d = 0; d < dim; ++d) {
            if (p->Gk[d] != 0) {
                P.box_lo[d] = 0;
                P.box_ext[d] = (int32_t)p->Gk[d];
            } else {
                int64_t lo = 0, hi = 0;
                for (int c = 0; c < ncc; ++c) {
                    int64_t v[64];
                    int nv = P.comp[c].len;
                    for (int i = 0; i < nv; ++i) v[i] = P.kv[P.comp[c].shift + i][d];
                    for (int a = 1; a < nv; ++a) {   // insertion sort
                        int64_t x = v[a];
                        int b = a - 1;
                        while (b >= 0 && v[b] > x) { v[b + 1] = v[b]; --b; }
                        v[b + 1] = x;
                    }
                    for (int i = 0; i < P.comp[c].t && i < nv; ++i) { lo += v[i]; hi += v[nv - 1 - i]; }
                }
                P.box_lo[d] = (int32_t)lo;
                P.box_ext[d] = (int32_t)(hi - lo + 1);
            }
            box_n *= P.box_ext[d];
            MOMED_REQUIRE(box_n <= kNoAllocMaxBox, MOMED_EINVAL,
                          "momentum box exceeds the 4096-entry table of the no-allocation enumerator");
            int64_t k = p->Gk[d] == 0 ? momentum[d] : jmod(momentum[d], p->Gk[d]);
            int64_t v = k - P.box_lo[d];
            if (v < 0 || v >= P.box_ext[d]) target_in = false;
            target += v * tstride;
            tstride *= P.box_ext[d];
        }
        int32_t sec_of[kNoAllocMaxBox];
        for (int64_t i = 0; i < box_n; ++i) sec_of[i] = -1;
        if (target_in) sec_of[target] = 0;
        uint64_t binom[65 * 65];
        for (int n = 0; n <= 64; ++n)
            for (int k = 0; k <= 64; ++k) binom[n * 65 + k] = k <= n ? (uint64_t)hbinom(n, k) : 0ull;
        int nblocks = 1;
        P.chunk = 16;
        if (total > 0) {
            P.chunk = std::max<int64_t>(16, (total + (int64_t)kNoAllocMaxBlocks * kThreads - 1) /
                                                ((int64_t)kNoAllocMaxBlocks * kThreads));
            int64_t nthreads = (total + P.chunk - 1) / P.chunk;
            nblocks = (int)((nthreads + kThreads - 1) / kThreads);
        }
        MOMED_REQUIRE(nblocks <= kNoAllocMaxBlocks, MOMED_EINVAL, "combination space too large for the scratch");

        auto* d_binom = reinterpret_cast<uint64_t*>(scratch + kNoAllocBinomOff);
        auto* d_sec = reinterpret_cast<int32_t*>(scratch + kNoAllocSecOff);
        auto* d_cnt = reinterpret_cast<int32_t*>(scratch + kNoAllocCntOff);
        auto* d_off = reinterpret_cast<int64_t*>(scratch + kNoAllocOffOff);
        auto* d_err = reinterpret_cast<unsigned long long*>(scratch + kNoAllocErrOff);
        MOMED_CUDA_TRY(cudaMemcpyAsync(d_binom, binom, sizeof(binom), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(d_sec, sec_of, box_n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaMemsetAsync(d_err, 0, 16 * 8, st));   // the previous call's errors and total
        P.binom = d_binom;
        P.sec_of = d_sec;
        P.box_n = box_n;
        P.out_cap = 0;
        P.err = d_err;
        unsigned long long res[16] = {0};
        if (total > 0 && target_in) {
            k_enum_count<<<nblocks, kThreads, 0, st>>>(P, 0, 1, d_cnt);
            k_noalloc_scan<<<1, 1024, 0, st>>>(d_cnt, nblocks, d_off, d_err + 8);
            MOMED_CUDA_TRY(cudaGetLastError());
            note_launches(2);
            MOMED_CUDA_TRY(cudaMemcpyAsync(res, d_err, sizeof(res), cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            MOMED_REQUIRE(res[0] == 0, MOMED_ECUDA, "basis enumeration count pass skipped out-of-range accesses");
        } else {
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));   // the table uploads above, before returning
        }
        const int64_t n = (int64_t)res[8];
        *n_states = n;
        if (n > out_capacity) return MOMED_EINVAL;   // *n_states tells the caller the size needed
        if (n > 0) {
            MOMED_REQUIRE(out_dev, MOMED_EINVAL, "null output buffer");
            P.out_cap = out_capacity;
            k_enum_write<<<nblocks, kThreads, 0, st>>>(P, 0, 1, d_off, out_dev);
            MOMED_CUDA_TRY(cudaGetLastError());
            note_launches(1);
            MOMED_CUDA_TRY(cudaMemcpyAsync(res, d_err, 8 * 8, cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            MOMED_REQUIRE(res[0] == 0, MOMED_ECUDA, "basis enumeration skipped out-of-range accesses");
        }
        return MOMED_OK;
    } catch (const Error& e) {
        return e.code;
    }
}
