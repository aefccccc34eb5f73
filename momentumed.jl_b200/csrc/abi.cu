// C ABI of libmomed_b200 (include/momed.h): handles, uploads, dispatch, errors.
//
// Every entry point catches momed::Error and CUDA failures and turns them into
// an int status plus momed_last_error(h); nothing throws across the boundary.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "index.cuh"

#define MOMED_VERSION_STRING "momed-b200 0.1.0 (sm_100a)"

using namespace momed;

namespace momed {

static std::atomic<int64_t> g_launches{0};
static thread_local int64_t t_launches = 0;   // this thread's share (graph captures count their own)
void note_launches(int64_t n) {
    g_launches.fetch_add(n, std::memory_order_relaxed);
    t_launches += n;
}
int64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
int64_t launches_this_thread() { return t_launches; }

// Fold the elapsed time of recorded event pairs into prof_ms and recycle them.
static void prof_drain(momed_handle* h) {
    if (h->prof_used == 0) return;
    MOMED_CUDA_TRY(cudaEventSynchronize(h->prof_ev[h->prof_used - 1]));
    for (size_t i = 0; i + 1 < h->prof_used; i += 2) {
        float ms = 0.f;
        MOMED_CUDA_TRY(cudaEventElapsedTime(&ms, h->prof_ev[i], h->prof_ev[i + 1]));
        h->prof_ms[h->prof_kind[i / 2]] += ms;
    }
    h->prof_used = 0;
}

void prof_begin(momed_handle* h) {
    if (!h->prof) return;
    if (h->prof_used + 2 > h->prof_ev.size()) {
        if (h->prof_ev.size() >= 4096) prof_drain(h);   // bounded pool
        while (h->prof_used + 2 > h->prof_ev.size()) {
            cudaEvent_t e;
            MOMED_CUDA_TRY(cudaEventCreate(&e));
            h->prof_ev.push_back(e);
        }
        h->prof_kind.resize(h->prof_ev.size() / 2 + 1, 0);
    }
    MOMED_CUDA_TRY(cudaEventRecord(h->prof_ev[h->prof_used++], h->stream));
}

void prof_end(momed_handle* h, int kind) {
    if (!h->prof) return;
    h->prof_kind[(h->prof_used - 1) / 2] = kind;
    MOMED_CUDA_TRY(cudaEventRecord(h->prof_ev[h->prof_used++], h->stream));
    if (kind >= 0 && kind < MOMED_KERNEL_KINDS) ++h->prof_launches[kind];
}

OpView Operator::view() const {
    OpView v{};
    v.ngroups = ngroups;
    v.g_out = g_out.p;
    v.g_start = g_start.p;
    v.single = single.p;
    v.pair = pair.p;
    v.generic = generic.p;
    v.ngeneric = ngeneric;
    v.t_in = t_in.p;
    v.t_out = t_out.p;
    v.t_pm = t_pm.p;
    v.t_amp = amp.p;
    v.t_amp32 = amp32.p;
    v.t_ampb = has_b ? ampb.p : nullptr;
    v.t_ampb32 = has_b ? ampb32.p : nullptr;
    v.nterms = (int32_t)nterms;
    v.max_groups_per_row = max_groups;
    return v;
}

static uint64_t parity_mask_host(uint64_t occ) {
    // EDCore scattering.jl:7-18 with Julia's (1 << 64) == 0
    auto shl = [](int s) -> uint64_t { return s >= 64 ? 0ull : (1ull << s); };
    uint64_t mask = 0;
    while (occ) {
        int tz1 = __builtin_ctzll(occ);
        occ &= occ - 1;
        int tz2 = occ ? __builtin_ctzll(occ) : 64;
        occ &= occ - 1;
        mask += shl(tz2);
        mask -= shl(tz1 + 1);
    }
    return mask;
}

// Regroup the term list by creation mask and upload it (the struct-of-arrays flattening of
// create_gpu_linearmap, MomentumEDCUDAExt.jl:94-113, in a layout the kernel can index).
void upload_operator(momed_handle* h, const double* amp_a, const double* amp_b, const uint64_t* in,
                     const uint64_t* out, const uint64_t* parity, int64_t nscat) {
    MOMED_REQUIRE(nscat >= 0 && nscat < (1ll << 31), MOMED_EINVAL, "nscat out of range");
    MOMED_REQUIRE(nscat == 0 || (amp_a && in && out), MOMED_EINVAL, "amp, in and out are required");
    std::vector<int64_t> ord(nscat);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) {
        return out[a] < out[b] || (out[a] == out[b] && in[a] < in[b]);
    });
    std::vector<uint64_t> t_in(nscat), t_out(nscat), t_pm(nscat), g_out;
    std::vector<double2> A(nscat), B(amp_b ? nscat : 0);
    std::vector<float2> A32(nscat), B32(amp_b ? nscat : 0);
    std::vector<int32_t> g_start;
    uint64_t mask_or = 0;
    for (int64_t q = 0; q < nscat; ++q) {
        int64_t s = ord[q];
        if (q == 0 || out[s] != out[ord[q - 1]]) {
            g_out.push_back(out[s]);
            g_start.push_back((int32_t)q);
        }
        t_in[q] = in[s];
        t_out[q] = out[s];
        uint64_t pm = parity_mask_host(out[s]) ^ parity_mask_host(in[s]);
        MOMED_REQUIRE(!parity || parity[s] == pm, MOMED_EINVAL,
                      "parity mask does not match parity_mask(out) xor parity_mask(in)");
        MOMED_REQUIRE(__builtin_popcountll(in[s]) == __builtin_popcountll(out[s]), MOMED_EINVAL,
                      "scatter term does not conserve particle number");
        t_pm[q] = pm;
        A[q] = make_double2(amp_a[2 * s], amp_a[2 * s + 1]);
        A32[q] = make_float2((float)amp_a[2 * s], (float)amp_a[2 * s + 1]);
        if (amp_b) {
            B[q] = make_double2(amp_b[2 * s], amp_b[2 * s + 1]);
            B32[q] = make_float2((float)amp_b[2 * s], (float)amp_b[2 * s + 1]);
        }
        mask_or |= in[s] | out[s];
    }
    g_start.push_back((int32_t)nscat);
    const int ng = (int)g_out.size();
    std::vector<int32_t> single(64, -1), pair(64 * 64, -1), generic;
    for (int g = 0; g < ng; ++g) {
        uint64_t o = g_out[g];
        int pc = __builtin_popcountll(o);
        if (pc == 1) single[__builtin_ctzll(o)] = g;
        else if (pc == 2) {
            int a = __builtin_ctzll(o), b = 63 - __builtin_clzll(o);
            pair[a * 64 + b] = g;
        } else generic.push_back(g);
    }
    Operator& op = h->op;
    cudaStream_t st = h->stream;
    op.nterms = nscat;
    op.ngroups = ng;
    op.ngeneric = (int32_t)generic.size();
    op.has_b = amp_b != nullptr;
    auto up = [&](auto& dst, const auto& src) {
        using T = typename std::decay_t<decltype(src)>::value_type;
        dst.resize(std::max<size_t>(src.size(), 1));
        if (!src.empty())
            MOMED_CUDA_TRY(cudaMemcpyAsync(dst.p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    };
    up(op.g_out, g_out);
    up(op.g_start, g_start);
    up(op.single, single);
    up(op.pair, pair);
    up(op.generic, generic);
    up(op.t_in, t_in);
    up(op.t_out, t_out);
    up(op.t_pm, t_pm);
    up(op.amp, A);
    up(op.amp32, A32);
    if (amp_b) {
        up(op.ampb, B);
        up(op.ampb32, B32);
    }
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    h->op_order = std::move(ord);
    h->recipe.set = false;                 // a recipe describes the operator it was attached to
    h->op_mask_or = mask_or;
    h->op_set = true;
    h->op_validated = false;
    h->sparse.release();
    h->hcache.release();
}

// Build the index when the basis changed or the operator reaches bits outside it, and
// validate the operator once: zero targets outside the basis enables the unchecked lookup.
void ensure_ready(momed_handle* h) {
    MOMED_REQUIRE(!h->sparse_only, MOMED_ESTATE,
                  "the handle holds an uploaded matrix without a basis (momed_set_sparse_csr); set a basis first");
    MOMED_REQUIRE(h->n > 0, MOMED_ESTATE, "set a basis first (momed_set_basis / momed_select_sector)");
    MOMED_REQUIRE(h->op_set, MOMED_ESTATE, "set an operator first (momed_set_scatter)");
    if (h->index_dirty || (h->op_mask_or & ~h->index_bits)) {
        h->index_bits = h->basis_or | h->op_mask_or;
        build_index(h);
        h->index_dirty = false;
        h->op_validated = false;
    }
    if (!h->op_validated) {
        if (h->index.mode != INDEX_SEARCH) {
            h->index.mode = INDEX_CHECKED;
            h->counters.resize(16);
            MOMED_CUDA_TRY(cudaMemsetAsync(h->counters.p, 0, 2 * sizeof(unsigned long long), h->stream));
            launch_count_hits(index_view(h), h->op.view(), h->counters.p, h->counters.p + 1, h->n, h->stream);
            unsigned long long hm[2];
            MOMED_CUDA_TRY(cudaMemcpyAsync(hm, h->counters.p, sizeof(hm), cudaMemcpyDeviceToHost, h->stream));
            MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
            h->nnz = (int64_t)hm[0];
            h->index.misses_checked = (int64_t)hm[1];
            if (hm[1] == 0) h->index.mode = INDEX_RANKED;
        } else {
            h->counters.resize(16);
            MOMED_CUDA_TRY(cudaMemsetAsync(h->counters.p, 0, 2 * sizeof(unsigned long long), h->stream));
            launch_count_hits(index_view(h), h->op.view(), h->counters.p, h->counters.p + 1, h->n, h->stream);
            unsigned long long hm[2];
            MOMED_CUDA_TRY(cudaMemcpyAsync(hm, h->counters.p, sizeof(hm), cudaMemcpyDeviceToHost, h->stream));
            MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
            h->nnz = (int64_t)hm[0];
            h->index.misses_checked = (int64_t)hm[1];
        }
        h->op_validated = true;
    }
}

thread_local cudaStream_t g_alloc_stream = nullptr;

}  // namespace momed

namespace {

template <typename F>
int guarded(momed_handle* h, F&& f) {
    try {
        AllocScope scope(h ? h->stream : g_alloc_stream);
        if (h) {
            cudaError_t e = cudaSetDevice(h->device);
            if (e != cudaSuccess) throw Error{MOMED_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e)};
        }
        int rc = f();
        if (h && rc == MOMED_OK) h->last_error.clear();
        return rc;
    } catch (const Error& e) {
        if (h) h->last_error = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        if (h) h->last_error = e.what();
        return MOMED_EINVAL;
    }
}

thread_local std::string g_create_error;

// The default memory pool of each device keeps freed blocks for reuse instead of returning them
// at every synchronisation (set once per device; process-local, gone at exit).
void keep_pool_memory(int device) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), device) != done.end()) return;
    cudaMemPool_t pool;
    MOMED_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    MOMED_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    done.push_back(device);
}

__global__ void k_or_basis(const uint64_t* b, int64_t n, unsigned long long* out) {
    uint64_t acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc |= b[i];
    for (int o = 16; o > 0; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicOr(out, (unsigned long long)acc);
}

void after_basis_change(momed_handle* h) {
    h->counters.resize(16);
    MOMED_CUDA_TRY(cudaMemsetAsync(h->counters.p + 2, 0, sizeof(unsigned long long), h->stream));
    if (h->n > 0) k_or_basis<<<std::min<int64_t>(1184, (h->n + 255) / 256), 256, 0, h->stream>>>(h->basis.p, h->n, h->counters.p + 2);
    unsigned long long v = 0;
    MOMED_CUDA_TRY(cudaMemcpyAsync(&v, h->counters.p + 2, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->basis_or = v;
    h->index_dirty = true;
    h->op_validated = false;
    h->sparse.release();
    h->hcache.release();
    h->sparse_only = false;
}

}  // namespace

extern "C" {

const char* momed_version(void) { return MOMED_VERSION_STRING; }

int momed_create(int device, momed_handle** out) {
    if (!out) return MOMED_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
        return MOMED_ENODEV;
    }
    if (device < 0 || device >= ndev) return MOMED_EINVAL;
    momed_handle* h = new momed_handle();
    h->device = device;
    int rc = guarded(h, [&]() {
        keep_pool_memory(device);
        MOMED_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
        g_alloc_stream = h->stream;   // this call's scope (set before the stream existed)
        MOMED_CUDA_TRY(cudaEventCreate(&h->ev0));
        MOMED_CUDA_TRY(cudaEventCreate(&h->ev1));
        std::vector<uint32_t> b(33 * 33, 0);
        for (int n = 0; n <= 32; ++n)
            for (int k = 0; k <= n; ++k) {
                uint64_t r = 1;
                for (int i = 1; i <= k; ++i) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
                b[n * 33 + k] = (uint32_t)r;
            }
        h->binom.resize(b.size());
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->binom.p, b.data(), b.size() * 4, cudaMemcpyHostToDevice, h->stream));
        h->u_dev.resize(1);
        h->u_dev32.resize(1);
        double one = 1.0;
        float onef = 1.0f;
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &one, sizeof(one), cudaMemcpyHostToDevice, h->stream));
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &onef, sizeof(onef), cudaMemcpyHostToDevice, h->stream));
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return MOMED_OK;
    });
    if (rc != MOMED_OK) {
        g_create_error = h->last_error;
        momed_destroy(h);
        return rc;
    }
    *out = h;
    return MOMED_OK;
}

int momed_destroy(momed_handle* h) {
    if (!h) return MOMED_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    cudaStream_t hs = h->stream;
    const bool own = h->own_stream;
    {
        AllocScope scope(hs);
        delete h;   // releases every DevBuf, ordered on the handle's stream
    }
    cudaStreamSynchronize(hs);
    if (own && hs) cudaStreamDestroy(hs);
    cudaMemPool_t pool;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);   // return blocks no other handle is using
    return MOMED_OK;
}

const char* momed_last_error(const momed_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->last_error.c_str();
}

int momed_set_stream(momed_handle* h, void* s) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        if (h->own_stream) cudaStreamDestroy(h->stream);
        h->stream = (cudaStream_t)s;
        h->own_stream = false;
        return MOMED_OK;
    });
}

int momed_set_hbm_budget(momed_handle* h, int64_t bytes) {
    if (!h || bytes < 0) return MOMED_EINVAL;
    h->hbm_budget = bytes;
    return MOMED_OK;
}

int momed_enumerate_basis(momed_handle* h, const momed_para* p, const int64_t* N_each, int32_t ncc, const int64_t* mask,
                          int32_t mlen, const int64_t* momentum_list, int32_t nmom, int64_t* n_sectors,
                          int64_t* n_total) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(N_each && n_sectors && n_total, MOMED_EINVAL, "null argument");
        enumerate_basis(h, p, N_each, ncc, mask, mlen, momentum_list, nmom);
        *n_sectors = (int64_t)h->enumer.sizes.size();
        *n_total = h->enumer.offsets.empty() ? 0 : h->enumer.offsets.back();
        return MOMED_OK;
    });
}

int momed_enumeration_copy(momed_handle* h, int64_t* sector_k, int64_t* sector_sizes, uint64_t* basis,
                           int32_t basis_on_device) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        Enumeration& E = h->enumer;
        if (sector_k && !E.sector_k.empty()) std::memcpy(sector_k, E.sector_k.data(), E.sector_k.size() * 8);
        if (sector_sizes && !E.sizes.empty()) std::memcpy(sector_sizes, E.sizes.data(), E.sizes.size() * 8);
        int64_t tot = E.offsets.empty() ? 0 : E.offsets.back();
        if (basis && tot > 0) {
            MOMED_CUDA_TRY(cudaMemcpyAsync(basis, E.states.p, tot * 8,
                                           basis_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                           h->stream));
            MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        }
        return MOMED_OK;
    });
}

int momed_select_sector(momed_handle* h, int64_t s) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        Enumeration& E = h->enumer;
        MOMED_REQUIRE(s >= 0 && s < (int64_t)E.sizes.size(), MOMED_EINVAL, "sector index out of range");
        int64_t n = E.sizes[s];
        h->basis.resize(std::max<int64_t>(n, 1));
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->basis.p, E.states.p + E.offsets[s], n * 8, cudaMemcpyDeviceToDevice,
                                       h->stream));
        h->n = n;
        after_basis_change(h);
        return MOMED_OK;
    });
}

int momed_set_basis(momed_handle* h, const uint64_t* basis, int64_t n, int32_t on_device) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(n >= 0 && (n == 0 || basis), MOMED_EINVAL, "bad basis");
        h->basis.resize(std::max<int64_t>(n, 1));
        if (n > 0)
            MOMED_CUDA_TRY(cudaMemcpyAsync(h->basis.p, basis, n * 8,
                                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
        h->n = n;
        after_basis_change(h);
        return MOMED_OK;
    });
}

int momed_set_scatter(momed_handle* h, const double* amp, const uint64_t* in, const uint64_t* out,
                      const uint64_t* parity, int64_t nscat) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        upload_operator(h, amp, nullptr, in, out, parity, nscat);
        return MOMED_OK;
    });
}

int momed_block_tuning(momed_handle* h, int32_t nb, int32_t precision, int32_t has_param, int32_t* rows_per_warp,
                       int32_t* grid_mult, double* ms, double* ms_default) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(h->op_set && h->n > 0, MOMED_ESTATE, "no working basis and operator");
        MOMED_REQUIRE(rows_per_warp && grid_mult, MOMED_EINVAL, "null output");
        int g = 0, r = 0;
        float a = 0.f, b = 0.f;
        const bool hb = has_param && h->op.has_b;
        if (!block_tuning_lookup(h->op.view(), h->n, nb, precision == MOMED_PREC_FP64, hb, &g, &r, &a, &b))
            return (int)MOMED_ESTATE;
        *rows_per_warp = r;
        *grid_mult = g;
        if (ms) *ms = a;
        if (ms_default) *ms_default = b;
        return (int)MOMED_OK;
    });
}

int momed_set_twobody_recipe(momed_handle* h, const momed_para* p, int32_t recipe, const double* params,
                             int32_t nparams, const int32_t* raw, int64_t nraw, const int64_t* upper_start,
                             int64_t nupper, const int64_t* entry_upper, const int32_t* entry_partner,
                             int64_t nentries) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        set_twobody_recipe(h, p, recipe, params, nparams, raw, nraw, upper_start, nupper, entry_upper, entry_partner,
                           nentries);
        return MOMED_OK;
    });
}

int momed_set_kshift(momed_handle* h, const double* kshift) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        set_kshift(h, kshift);
        return MOMED_OK;
    });
}

int momed_set_scatter_pair(momed_handle* h, const double* amp_a, const double* amp_b, const uint64_t* in,
                           const uint64_t* out, const uint64_t* parity, int64_t nscat) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        upload_operator(h, amp_a, amp_b, in, out, parity, nscat);
        return MOMED_OK;
    });
}

int momed_set_param(momed_handle* h, double u) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        float uf = (float)u;
        h->u = u;
        if (h->sparse.built && h->op.has_b && h->sparse.u != u) h->sparse.release();   // values were built at the old u
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &u, sizeof(u), cudaMemcpyHostToDevice, h->stream));
        MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &uf, sizeof(uf), cudaMemcpyHostToDevice, h->stream));
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return MOMED_OK;
    });
}

int momed_matvec(momed_handle* h, const void* x, void* y, int32_t precision, int32_t on_device) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(x && y, MOMED_EINVAL, "null vector");
        MOMED_REQUIRE(precision == MOMED_C128 || precision == MOMED_C64, MOMED_EINVAL, "unknown precision");
        if (!h->sparse.built) ensure_ready(h);
        const int64_t n = h->n;
        cudaStream_t st = h->stream;
        const size_t es = precision == MOMED_C128 ? 16 : 8;
        const void* dx = x;
        void* dy = y;
        if (!on_device) {
            if (precision == MOMED_C128) { h->xbuf.resize(n); h->ybuf.resize(n); dx = h->xbuf.p; dy = h->ybuf.p; }
            else { h->xbuf32.resize(n); h->ybuf32.resize(n); dx = h->xbuf32.p; dy = h->ybuf32.p; }
            MOMED_CUDA_TRY(cudaMemcpyAsync(const_cast<void*>(dx), x, n * es, cudaMemcpyHostToDevice, st));
        }
        MOMED_CUDA_TRY(cudaEventRecord(h->ev0, st));
        if (h->sparse.built && precision == MOMED_C128)
            launch_spmv_c128(h->sparse, (const double2*)dx, (double2*)dy, n, st);
        else if (h->sparse.built)
            launch_spmv_c64(h->sparse, (const float2*)dx, (float2*)dy, n, st);
        else if (h->hcache.built && precision == MOMED_C128)
            launch_matvec_hc_c128(h, (const double2*)dx, (double2*)dy, h->op.has_b ? h->u_dev.p : nullptr, n, st);
        else if (h->hcache.built)
            launch_matvec_hc_c64(h, (const float2*)dx, (float2*)dy, h->op.has_b ? h->u_dev32.p : nullptr, n, st);
        else if (precision == MOMED_C128)
            launch_matvec_c128(index_view(h), h->op.view(), (const double2*)dx, (double2*)dy,
                               h->op.has_b ? h->u_dev.p : nullptr, n, st);
        else
            launch_matvec_c64(index_view(h), h->op.view(), (const float2*)dx, (float2*)dy,
                              h->op.has_b ? h->u_dev32.p : nullptr, n, st);
        MOMED_CUDA_TRY(cudaEventRecord(h->ev1, st));
        if (!on_device) MOMED_CUDA_TRY(cudaMemcpyAsync(y, dy, n * es, cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        h->last_kernel_ms = ms;
        return MOMED_OK;
    });
}

int momed_eigsolve(momed_handle* h, const momed_solve_opts* opts, const double* vec0, double* vals, double* resid,
                   void* vecs, momed_info* info) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(opts && vals, MOMED_EINVAL, "opts and vals are required");
        return momed_eigsolve_impl(h, opts, vec0, vals, resid, vecs, info);
    });
}

int momed_eigsolve_general(momed_handle* h, const momed_solve_opts* opts, const double* vec0, double* vals,
                           double* resid, void* vecs, momed_info* info) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(opts && vals, MOMED_EINVAL, "opts and vals are required");
        return momed_eigsolve_general_impl(h, opts, vec0, vals, resid, vecs, info);
    });
}

int momed_batch_solve(momed_handle* h, const momed_solve_opts* opts, const double* u, int32_t nu, double* vals,
                      double* resid, double* vecs, momed_info* info) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(opts && u && vals && nu >= 1, MOMED_EINVAL, "opts, u and vals are required");
        return momed_batch_solve_impl(h, opts, u, nu, vals, resid, vecs, info);
    });
}

int momed_build_sparse(momed_handle* h, int64_t* nnz) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        ensure_ready(h);
        build_sparse(h, h->u);
        if (nnz) *nnz = h->sparse.nnz;
        return MOMED_OK;
    });
}

int momed_sparse_copy(momed_handle* h, int64_t* row_ptr, int32_t* col, double* val) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(h->sparse.built, MOMED_ESTATE, "no sparse matrix (momed_build_sparse)");
        const SparseMatrix& sp = h->sparse;
        cudaStream_t st = h->stream;
        if (row_ptr)
            MOMED_CUDA_TRY(cudaMemcpyAsync(row_ptr, sp.row_ptr.p, (h->n + 1) * 8, cudaMemcpyDeviceToHost, st));
        if (col) MOMED_CUDA_TRY(cudaMemcpyAsync(col, sp.col.p, sp.nnz * 4, cudaMemcpyDeviceToHost, st));
        if (val) MOMED_CUDA_TRY(cudaMemcpyAsync(val, sp.val.p, sp.nnz * 16, cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        return MOMED_OK;
    });
}

int momed_release_sparse(momed_handle* h) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->sparse.release();
        if (h->sparse_only) {          // nothing left to multiply by: back to an empty handle
            h->sparse_only = false;
            h->n = 0;
        }
        return MOMED_OK;
    });
}

int momed_set_sparse_csr(momed_handle* h, int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(n >= 1 && n <= (int64_t)INT32_MAX, MOMED_EINVAL, "matrix size must be in [1, 2^31 - 1]");
        MOMED_REQUIRE(row_ptr && col && val, MOMED_EINVAL, "row_ptr, col and val are required");
        MOMED_REQUIRE(row_ptr[0] == 0, MOMED_EINVAL, "row_ptr[0] must be 0");
        for (int64_t i = 0; i < n; ++i)
            MOMED_REQUIRE(row_ptr[i + 1] >= row_ptr[i], MOMED_EINVAL, "row_ptr must not decrease");
        const int64_t nnz = row_ptr[n];
        for (int64_t p = 0; p < nnz; ++p)
            MOMED_REQUIRE(col[p] >= 0 && (int64_t)col[p] < n, MOMED_EINVAL, "column index out of range");
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        upload_sparse(h, n, row_ptr, col, val);
        h->basis.release();
        h->n = n;
        h->basis_or = 0;
        h->index_dirty = true;
        h->op_validated = false;
        h->sparse_only = true;
        return MOMED_OK;
    });
}

int momed_bracket(momed_handle* h, const uint64_t* bra_basis, int64_t n_bra, const double* bra, const double* ket,
                  double* out) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(bra && ket && out, MOMED_EINVAL, "bra, ket and out are required");
        MOMED_REQUIRE(!bra_basis || n_bra >= 1, MOMED_EINVAL, "bad bra basis");
        ensure_ready(h);
        const int64_t n = h->n;
        cudaStream_t st = h->stream;
        IndexView iv = index_view(h);
        DevBuf<uint64_t> rows_b;
        const uint64_t* rows = h->basis.p;
        int64_t nrows = n;
        if (bra_basis) {
            for (int64_t i = 1; i < n_bra; ++i)
                MOMED_REQUIRE(bra_basis[i] > bra_basis[i - 1], MOMED_EINVAL, "bra basis must be sorted ascending");
            rows_b.resize(n_bra);
            MOMED_CUDA_TRY(cudaMemcpyAsync(rows_b.p, bra_basis, n_bra * 8, cudaMemcpyHostToDevice, st));
            rows = rows_b.p;
            nrows = n_bra;
            // targets of another space may be absent from this one: compare keys on every lookup
            if (iv.mode == INDEX_RANKED) iv.mode = INDEX_CHECKED;
        }
        DevBuf<double2> kd, bd, part;
        kd.resize(n);
        bd.resize(nrows);
        MOMED_CUDA_TRY(cudaMemcpyAsync(kd.p, ket, n * 16, cudaMemcpyHostToDevice, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(bd.p, bra, nrows * 16, cudaMemcpyHostToDevice, st));
        const int grid = bracket_grid(nrows);
        part.resize(grid);
        launch_bracket(iv, h->op.view(), rows, bd.p, kd.p, h->op.has_b ? h->u_dev.p : nullptr, nrows, part.p, grid, st);
        std::vector<double2> hp(grid);
        MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, grid * 16, cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        double re = 0.0, im = 0.0;
        for (const double2& v : hp) { re += v.x; im += v.y; }
        out[0] = re;
        out[1] = im;
        return MOMED_OK;
    });
}

int momed_rdm1(momed_handle* h, const double* psi, int32_t norb, double* rdm) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(psi && rdm, MOMED_EINVAL, "psi and rdm are required");
        rdm1(h, psi, norb, rdm);
        return MOMED_OK;
    });
}

int momed_step_inner_prod(momed_handle* h, const double* psi_f, const double* psi_i, int32_t g, const double* orb,
                          int32_t norb, double* out) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(psi_f && psi_i && orb && out, MOMED_EINVAL, "psi_f, psi_i, orb and out are required");
        step_inner_prod(h, psi_f, psi_i, g, orb, norb, out);
        return MOMED_OK;
    });
}

int momed_stats(momed_handle* h, int64_t* nnz, int32_t* index_mode, int64_t* table_bytes) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        ensure_ready(h);
        if (nnz) *nnz = h->nnz;
        if (index_mode) *index_mode = h->index.mode;
        if (table_bytes) *table_bytes = (int64_t)(h->index.off_hi.bytes() + h->index.rank_lo.bytes());
        return MOMED_OK;
    });
}

int momed_last_kernel_ms(momed_handle* h, double* ms) {
    if (!h || !ms) return MOMED_EINVAL;
    *ms = h->last_kernel_ms;
    return MOMED_OK;
}

int64_t momed_kernel_launches(void) { return launches_total(); }

int momed_build_hit_cache(momed_handle* h, int64_t* hits, int64_t* bytes) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_REQUIRE(!h->sparse.built && !h->sparse_only, MOMED_ESTATE,
                      "a sparse matrix is built: maps read it (momed_release_sparse first)");
        ensure_ready(h);
        const char* e = std::getenv("MOMED_HITCACHE");
        build_hit_cache(h, (e && e[0] == '2') ? 2 : 1);     // MOMED_HITCACHE=2: the slot mode
        if (hits) *hits = h->hcache.nnz;
        if (bytes) *bytes = h->hcache.bytes;
        return MOMED_OK;
    });
}

int momed_hit_cache_info(momed_handle* h, int32_t* built, int64_t* hits, int64_t* bytes, double* build_ms) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        if (built) *built = h->hcache.built ? h->hcache.mode : 0;   // 1 full, 2 slot mode
        if (hits) *hits = h->hcache.nnz;
        if (bytes) *bytes = h->hcache.bytes;
        if (build_ms) *build_ms = h->hcache.build_ms;
        return MOMED_OK;
    });
}

int momed_release_hit_cache(momed_handle* h) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->hcache.release();
        return MOMED_OK;
    });
}

int momed_profile(momed_handle* h, int32_t enable) {
    if (!h) return MOMED_EINVAL;
    return guarded(h, [&]() {
        MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->prof_used = 0;
        for (int k = 0; k < MOMED_KERNEL_KINDS; ++k) { h->prof_launches[k] = 0; h->prof_ms[k] = 0.0; }
        h->prof = enable != 0;
        return MOMED_OK;
    });
}

int momed_profile_read(momed_handle* h, int32_t kind, int64_t* launches, double* total_ms) {
    if (!h || kind < 0 || kind >= MOMED_KERNEL_KINDS) return MOMED_EINVAL;
    return guarded(h, [&]() {
        prof_drain(h);
        if (launches) *launches = h->prof_launches[kind];
        if (total_ms) *total_ms = h->prof_ms[kind];
        return MOMED_OK;
    });
}

}  // extern "C"
