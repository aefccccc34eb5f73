// Internal declarations of libmomed_b200: the handle, device data layouts and
// the kernels' host-side launchers.  Not part of the public ABI (include/momed.h).
#pragma once

#include <cuda_runtime.h>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/momed.h"

namespace momed {

// ---------------------------------------------------------------- errors
struct Error {
    int code;
    std::string msg;
};

inline std::string base_name(const char* path) {
    std::string s(path);
    size_t k = s.find_last_of('/');
    return k == std::string::npos ? s : s.substr(k + 1);
}

#define MOMED_CUDA_TRY(expr)                                                                 \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) {                                                             \
            throw ::momed::Error{MOMED_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e) +  \
                                                  " (" + ::momed::base_name(__FILE__) + ":" +           \
                                                  std::to_string(__LINE__) + ")"};                    \
        }                                                                                    \
    } while (0)

#define MOMED_REQUIRE(cond, code, text)                       \
    do {                                                      \
        if (!(cond)) throw ::momed::Error{(code), (text)};    \
    } while (0)

// ---------------------------------------------------------------- device buffer
// Stream on which the calling thread's DevBuf allocations and frees are ordered: the handle's
// stream for the duration of an API call (AllocScope).  Allocation is stream-ordered
// (cudaMallocAsync / cudaFreeAsync from the device's default memory pool), so freeing a solve's
// buffers does not synchronise the device and solves on other streams keep running.
extern thread_local cudaStream_t g_alloc_stream;
struct AllocScope {
    cudaStream_t prev;
    explicit AllocScope(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
    ~AllocScope() { g_alloc_stream = prev; }
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;
};

// Owning device allocation, ordered on g_alloc_stream; moves only.
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, g_alloc_stream);
        p = nullptr;
        n = 0;
    }
    void resize(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), g_alloc_stream);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            throw Error{MOMED_ENOMEM, std::string("device allocation of ") + std::to_string(count * sizeof(T)) +
                                          " bytes failed: " + cudaGetErrorString(e)};
        }
        n = count;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------- index tables
// A basis state is split into a high part (bits >= L) and a low part (bits < L).
// Each part maps to a table slot either directly (slot = bits) or through its
// combinadic rank: slot = base[popcount - cmin] + sum_k C(pos_k, k) over the set
// bits (colex rank among patterns of equal popcount).
enum PartMode : int32_t { PART_DIRECT = 0, PART_COMBINADIC = 1 };

struct PartDesc {
    int32_t shift;      // first bit of the part
    int32_t width;      // bits in the part (<= 32 for combinadic, <= 24 direct)
    int32_t mode;       // PartMode
    int32_t cmin, cmax; // popcount range present in the basis
    uint32_t size;      // table entries
    uint32_t base[34];  // base[c - cmin] for combinadic
};

enum IndexMode : int32_t { INDEX_RANKED = 0, INDEX_CHECKED = 1, INDEX_SEARCH = 2 };

static constexpr uint32_t kInvalid = 0xFFFFFFFFu;

struct IndexView {       // passed by value to kernels
    const uint64_t* basis;
    int64_t n;
    const uint32_t* off_hi;   // [hi.size]  first basis index of each high pattern (kInvalid: absent)
    const uint32_t* rank_lo;  // [lo.size]  rank of the low pattern inside its high group
    PartDesc hi, lo;
    int32_t mode;             // IndexMode
    const uint32_t* binom;    // [33 * 33] C(n, k) for n, k <= 32
};

// ---------------------------------------------------------------- operator terms
// The Hermitian-completed term list regrouped by the creation mask `out`: a row
// state s meets the terms of group g only when out_g is a subset of s.  Groups
// with |out| = 1 or 2 are found by table lookup; other groups are tested directly.
struct OpView {
    int32_t ngroups;
    const uint64_t* g_out;     // [ngroups]
    const int32_t* g_start;    // [ngroups + 1] term ranges
    const int32_t* single;     // [64]        group of out = {a} or -1
    const int32_t* pair;       // [64 * 64]   group of out = {a, b}, a < b, or -1
    const int32_t* generic;    // [ngeneric]  other groups
    int32_t ngeneric;
    const uint64_t* t_in;      // [nterms]
    const uint64_t* t_out;     // [nterms] (the group's out mask, per term)
    const uint64_t* t_pm;      // [nterms]
    const double2* t_amp;      // [nterms] c128 (A part)
    const float2* t_amp32;     // [nterms] c64  (A part)
    const double2* t_ampb;     // [nterms] c128 B part (parametrised operators) or null
    const float2* t_ampb32;    // [nterms] c64 B part or null
    int32_t nterms;
    int32_t max_groups_per_row;   // bound on candidate groups of one row
};

// ---------------------------------------------------------------- handle
struct Enumeration {
    int32_t dim = 0;
    std::vector<int64_t> sector_k;     // [nsec * dim]
    std::vector<int64_t> sizes;        // [nsec]
    std::vector<int64_t> offsets;      // [nsec + 1]
    DevBuf<uint64_t> states;           // concatenated sectors
};

struct Operator {
    int64_t nterms = 0;
    int32_t ngroups = 0, ngeneric = 0, max_groups = 0;
    bool has_b = false;
    DevBuf<uint64_t> g_out, t_in, t_out, t_pm;
    DevBuf<int32_t> g_start, single, pair, generic;
    DevBuf<double2> amp, ampb;
    DevBuf<float2> amp32, ampb32;
    OpView view() const;
};

// Device recipe of the two-body terms for twisted-boundary sweeps (recipe.cu): the raw
// contributions of every upper term of the working operator, so that its amplitudes can be
// regenerated on the device for any kshift (momed_set_kshift) without rebuilding the list.
struct TwoBodyRecipe {
    bool set = false;
    int32_t kind = 0, dim = 0, Nk = 0, Nc_mix = 1, Ncc = 1;
    double sys_size = 1.0;
    double params[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double Gk[3] = {0, 0, 0};
    int64_t nraw = 0, nupper = 0;
    DevBuf<double> kcoord;         // [Nk][dim] momentum coordinates k (before / Gk)
    DevBuf<int32_t> raw;           // [nraw][9]: kf1 kf2 ki2 ki1 (0-based), cf1 cf2 ci2 ci1 (1-based), flags
    DevBuf<int64_t> upper_start;   // [nupper + 1] contributions of each upper term, in merge order
    DevBuf<int32_t> slot_upper;    // per device term slot: its upper term (-1: keep the amplitude)
    DevBuf<int32_t> slot_partner;  // per device term slot: 1 for the Hermitian partner (conjugate)
    DevBuf<double2> upper_amp;     // [nupper] scratch of the regeneration
    DevBuf<double> shift;          // [Ncc][dim]
};

// CSR matrix of the working operator on the working basis (the sparse method, sparse.cu):
// row_ptr[n + 1]; per entry a column, the FP64 value at u and its FP32 rounding.
struct SparseMatrix {
    bool built = false;
    double u = 0.0;                // parameter the values were built at (H = A + u B)
    int64_t nnz = 0;
    DevBuf<int64_t> row_ptr;
    DevBuf<int32_t> col;
    DevBuf<double2> val;
    DevBuf<float2> val32;
    // the A and B parts of H(u) = A + u B per entry (c64), for the batched solver's block SpMV
    // (parametrised operators only; a single operator's block SpMV reads val32)
    DevBuf<float2> pa32, pb32;
    void release() {
        built = false;
        nnz = 0;
        row_ptr.release();
        col.release();
        val.release();
        val32.release();
        pa32.release();
        pb32.release();
    }
};

// Hit cache of the matrix-free map (hitcache.cu): per sector basis and term list, every
// off-diagonal hit's target row and term slot (sign in bit 31), in runs by amplitude kind.
struct HitCacheView {
    const int64_t* row_ptr;    // [n + 1]
    const int2* seg;           // [n] ends of the B-only and A-only runs, relative to row_ptr[row]
    const uint2* hit;          // [nnz] {target row, term slot | sign << 31}
    const double2* dg64;       // [2n] diagonal sums: A part, B part
    const float2* dg32;        // [2n] the same in c64
    const uint16_t* slot;      // [nnz] slot mode: the term slot of each off-diagonal hit
};

struct HitCache {
    bool built = false;
    int mode = 0;               // 1: full (target and term slot per hit), 2: term slots only
    int64_t nnz = 0, bytes = 0;
    double build_ms = 0.0;
    DevBuf<int64_t> row_ptr;
    DevBuf<int2> seg;
    DevBuf<uint2> hit;
    DevBuf<double2> dg64;
    DevBuf<float2> dg32;
    DevBuf<uint16_t> slot;
    // A + u B per term slot at the u of the single-vector map (one amplitude load per hit)
    DevBuf<double2> comb64;
    DevBuf<float2> comb32;
    double comb_u64 = 0.0, comb_u32 = 0.0;
    bool comb_ok64 = false, comb_ok32 = false;
    HitCacheView view() const;
    bool full() const { return built && mode == 1; }   // the block maps read full caches only
    void release() {
        built = false;
        mode = 0;
        nnz = bytes = 0;
        slot.release();
        comb64.release();
        comb32.release();
        comb_ok64 = comb_ok32 = false;
        row_ptr.release();
        seg.release();
        hit.release();
        dg64.release();
        dg32.release();
    }
};

struct Index {
    int32_t mode = INDEX_SEARCH;
    PartDesc hi{}, lo{};
    DevBuf<uint32_t> off_hi, rank_lo;
    int64_t misses_checked = -1;   // misses found by the validation pass (-1: not run)
};

}  // namespace momed

struct momed_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    int64_t hbm_budget = 0;

    int64_t n = 0;                         // basis size
    momed::DevBuf<uint64_t> basis;
    uint64_t basis_or = 0;                 // OR of all basis states
    momed::Index index;
    bool index_dirty = true;
    uint64_t index_bits = 0;               // bits the index tables cover
    momed::Operator op;
    std::vector<int64_t> op_order;         // device term slot q holds entry op_order[q] of the uploaded list
    momed::TwoBodyRecipe recipe;           // amplitudes regenerated on the device (momed_set_kshift)
    int32_t block_solver = -1;             // -1: the block solver when it pays, 0: single-vector only
    momed::SparseMatrix sparse;           // built by momed_build_sparse; maps use it while built
    momed::HitCache hcache;               // maps use it while built (and no sparse matrix is)
    bool hit_cache_ok = true;              // the solvers may build it (not on serving slots)
    bool sparse_only = false;              // an uploaded matrix (momed_set_sparse_csr) without a basis
    bool op_set = false;
    bool op_validated = false;
    uint64_t op_mask_or = 0;               // OR of all term masks
    int64_t nnz = 0;                       // (row, term) hits of the validated operator
    momed::DevBuf<double> u_dev;           // parameter u of H(u) = A + u B
    double u = 1.0;                        // host copy of u
    momed::DevBuf<float> u_dev32;
    momed::DevBuf<uint32_t> binom;         // C(n, k), n, k <= 32

    momed::Enumeration enumer;

    // scratch reused across calls
    momed::DevBuf<double2> xbuf, ybuf;
    momed::DevBuf<float2> xbuf32, ybuf32;
    momed::DevBuf<unsigned long long> counters;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_kernel_ms = 0.f;

    // optional per-launch timing of the matvec kernels
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev;      // pairs (start, stop)
    std::vector<int> prof_kind;            // kind of each pair
    size_t prof_used = 0;                  // events used in the current record
    int64_t prof_launches[MOMED_KERNEL_KINDS] = {};
    double prof_ms[MOMED_KERNEL_KINDS] = {};        // folded-in time of pairs already read
};

namespace momed {

// binomial table C(n, k), n, k in [0, 32], on the device (built once per process per device)
const uint32_t* device_binomials();

// index.cu
void build_index(momed_handle* h);
IndexView index_view(const momed_handle* h);
int64_t validate_operator(momed_handle* h);   // counts (row, term) targets missing from the basis

// hitcache.cu
int64_t hit_cache_bytes(int64_t n, int64_t hits);
int64_t slot_cache_bytes(int64_t n, int64_t hits);
int hit_cache_wanted(const momed_handle* h);             // 0 none, 1 full, 2 term slots only
void build_hit_cache(momed_handle* h, int mode = 1);
void ensure_hit_cache(momed_handle* h);
void launch_matvec_hc_c128(momed_handle* h, const double2* x, double2* y, const double* u, int64_t rows,
                           cudaStream_t st);
void launch_matvec_hc_c64(momed_handle* h, const float2* x, float2* y, const float* u, int64_t rows,
                          cudaStream_t st);
void launch_block_hc_c64(const momed_handle* h, const float2* x, float2* y, const float* u, int32_t nb, int64_t rows,
                         cudaStream_t st);
void launch_block_hc_c128(const momed_handle* h, const double2* x, double2* y, const double* u, int32_t nb,
                          int64_t rows, cudaStream_t st);

// matvec.cu
void launch_matvec_c128(const IndexView& iv, const OpView& ov, const double2* x, double2* y,
                        const double* u_scale, int64_t rows, cudaStream_t st);
void launch_matvec_c64(const IndexView& iv, const OpView& ov, const float2* x, float2* y,
                       const float* u_scale, int64_t rows, cudaStream_t st);
void launch_count_hits(const IndexView& iv, const OpView& ov, unsigned long long* hits,
                       unsigned long long* misses, int64_t rows, cudaStream_t st);
// <bra| H |ket>: rows over row_states (the bra space), lookups in iv (the ket space); one partial
// sum per block (grid from bracket_grid)
int bracket_grid(int64_t rows);
void launch_bracket(const IndexView& iv, const OpView& ov, const uint64_t* row_states, const double2* bra,
                    const double2* ket, const double* u, int64_t rows, double2* partial, int grid, cudaStream_t st);
// block matvec: nb right-hand sides interleaved [row][nb], H_u = A + u[b] B
void launch_block_matvec_c64(const IndexView& iv, const OpView& ov, const float2* x, float2* y,
                             const float* u, int32_t nb, int64_t rows, cudaStream_t st);
void launch_block_matvec_c128(const IndexView& iv, const OpView& ov, const double2* x, double2* y,
                              const double* u, int32_t nb, int64_t rows, cudaStream_t st);

// the block map autotuner's choice for this operator, sector size class and block width
bool block_tuning_lookup(const OpView& ov, int64_t rows, int nb, bool dbl, bool hb, int* grid_mult, int* rpw,
                         float* ms, float* ms_default);

// analysis.cu: one-body reduced density matrix of psi on the working basis ([norb][norb] c128)
void rdm1(momed_handle* h, const double* psi, int norb, double* rdm);
// ED_step_inner_prod of g vectors [g][N] on the working basis, orbital overlaps orb[norb] ([g][g] c128)
void step_inner_prod(momed_handle* h, const double* psi_f, const double* psi_i, int g, const double* orb, int norb,
                     double* out);

// sparse.cu: CSR build at parameter u (after ensure_ready) and the CSR SpMV
void build_sparse(momed_handle* h, double u);
void upload_sparse(momed_handle* h, int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val);
int64_t sparse_bytes_per_entry(bool pair);
void launch_block_spmv_c64(const SparseMatrix& sp, const float2* x, float2* y, const float* u, int32_t nb,
                           int64_t rows, cudaStream_t st);
void launch_spmv_c128(const SparseMatrix& sp, const double2* x, double2* y, int64_t rows, cudaStream_t st);
void launch_spmv_c64(const SparseMatrix& sp, const float2* x, float2* y, int64_t rows, cudaStream_t st);

// operator.cpp-side (in abi.cu)
void upload_operator(momed_handle* h, const double* amp_a, const double* amp_b, const uint64_t* in,
                     const uint64_t* out, const uint64_t* parity, int64_t nscat);

// enumerate.cu
void enumerate_basis(momed_handle* h, const momed_para* p, const int64_t* N_each, int ncc, const int64_t* mask,
                     int mlen, const int64_t* momentum_list, int nmom);

// tc_proj.cu: C = Q^H W of a c64 block basis on the tensor cores (B = 8 or 16 right-hand
// sides, ncol basis columns in blocks [N][B]); writes partial[split][c][r] for the *nsplit
// splits it chose (at most max_splits), to be summed over splits; *err = 1 if a wait timed out
void launch_proj_tc_c64(const float2* Q, int ncol, int64_t N, const float2* W, int B, double2* partial,
                        int max_splits, int* nsplit, int* err, cudaStream_t st);

// recipe.cu: device regeneration of the two-body amplitudes for a kshift
void set_twobody_recipe(momed_handle* h, const momed_para* p, int32_t kind, const double* params, int32_t nparams,
                        const int32_t* raw, int64_t nraw, const int64_t* upper_start, int64_t nupper,
                        const int64_t* entry_upper, const int32_t* entry_partner, int64_t nentries);
void set_kshift(momed_handle* h, const double* kshift);

// y = H x in FP64 on the working basis/operator (parameter u from the handle)
void apply_h_fp64(momed_handle* h, const double2* x, double2* y);

// bracket a matvec launch with timing events when profiling is on (abi.cu)
void prof_begin(momed_handle* h);
void prof_end(momed_handle* h, int kind);

// process-wide count of kernel launches issued by this library (diagnostics)
void note_launches(int64_t n);
int64_t launches_total();
int64_t launches_this_thread();   // launches noted by the calling thread

// small dense symmetric eigensolver (host, FP64): A n x n row-major (destroyed),
// eigenvalues ascending in w, eigenvectors as columns of V (row-major n x n)
void symeig(int n, double* A, double* w, double* V);
// small dense Hermitian eigensolver (host, FP64): A n x n row-major complex (destroyed),
// eigenvalues ascending in w, eigenvectors as columns of Z (row-major n x n complex)
void herm_eig(int n, std::complex<double>* A, double* w, std::complex<double>* Z);

}  // namespace momed

// Lanczos drivers (lanczos.cu)
int momed_eigsolve_impl(momed_handle* h, const momed_solve_opts* o, const double* vec0, double* vals, double* resid,
                        void* vecs, momed_info* info);
// arnoldi.cu: the non-Hermitian solver (vals [nev] complex, ordered by real part)
int momed_eigsolve_general_impl(momed_handle* h, const momed_solve_opts* o, const double* vec0, double* vals,
                                double* resid, void* vecs, momed_info* info);
int momed_batch_solve_impl(momed_handle* h, const momed_solve_opts* o, const double* u, int32_t nu, double* vals,
                           double* resid, double* vecs, momed_info* info);
