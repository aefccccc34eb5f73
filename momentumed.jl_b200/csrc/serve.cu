// Serving form: a continuous-batching eigensolve server.
//
// Requests (operator id, sector basis, parameter u, nev, tolerance, precision) arrive at any
// time.  A fixed set of worker slots, each with its own library handle and CUDA stream,
// takes requests in arrival order as soon as (a) a slot is free and (b) the request's HBM
// estimate fits the server's budget; every admitted solve keeps its Krylov basis and
// recurrence coefficients in HBM for its whole life, and the slots' kernels overlap on the
// device.  Continuous batching: a worker that takes the head request also takes every queued
// request on the same operator, sector basis and precision (up to 32, as long as the group
// fits the budget) and solves them as one batched solve, one right-hand side per request's
// parameter u; the block map then evaluates each candidate term once for the whole group.  A
// request alone runs the FP64 single-vector solver, the fastest form for one right-hand side,
// with the sparse method (a CSR matrix built on the device) when the matrix fits the budget.  A request larger than the whole budget fails at once with MOMED_ENOMEM; a request
// can be cancelled while queued; every wait the API offers is bounded and returns
// MOMED_ETIMEOUT when it runs out.
//
// A solve is deterministic (seeded start vector, fixed reduction order), so a request's
// result is the same alone and in any mix.
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "momed_internal.cuh"

namespace momed {
void ensure_ready(momed_handle* h);
}

using namespace momed;

namespace {

using clock_t_ = std::chrono::steady_clock;

struct HostOperator {
    std::vector<double> amp_a, amp_b;
    std::vector<uint64_t> in, out, parity;
    bool has_b = false;
};

struct Request {
    int64_t id = 0;
    int32_t op = 0;
    std::vector<uint64_t> basis;
    uint64_t bhash = 0;          // hash of the basis, to find requests on the same sector
    double u = 1.0;
    momed_solve_opts opts{};
    int64_t bytes = 0;
    bool single = false;         // solved by the single-vector solver (the block basis exceeds the budget)
    clock_t_::time_point arrival, start, done;
    int32_t status = 0;          // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
    int32_t rc = MOMED_OK;
    std::string err;
    std::vector<double> vals, resid;
    momed_info info{};
};

}  // namespace

struct momed_server {
    int device = 0;
    int64_t budget = 0;
    int64_t used = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<int64_t, std::shared_ptr<Request>> all;
    std::vector<std::shared_ptr<const HostOperator>> ops;   // read by workers under mu
    std::vector<double> op_hits_per_row;                    // learned from validated solves (0: none yet)
    std::vector<std::thread> workers;
    std::vector<momed_handle*> handles;
    int64_t next_id = 1;
    bool stopping = false;
    std::string last_error;
    int64_t completed = 0, failed = 0;
    int large_running = 0;   // groups of at least kLargeRows states on the device
};

namespace {

// A solve of at least this many states keeps the GPU (and its L2, which holds the map's input
// vector and index tables) busy on its own; two at once only evict each other's working sets.
// Such requests run one at a time (MOMED_SERVE_LARGE_MAX raises that count); smaller ones still
// overlap with them and with each other.
constexpr int64_t kLargeRows = 1 << 17;
// Smallest group that the batched solver serves faster per request than the single-vector solver.
constexpr int kMinGroup = 3;
// Largest nev of a request that may join a group (groups run the mixed-precision batched solver).
constexpr int kMaxMixedNev = 12;
// A request alone of at least this many states is solved with the sparse method when its CSR
// matrix fits what the budget has left: the matrix costs about two maps to build and its SpMV
// runs 3-4x faster than the map on large sectors.  Below it both are launch-bound.
constexpr int64_t kSparseMinRows = 1 << 12;

// HBM a solve needs: basis, index tables (bounded), Krylov basis, Ritz/refinement buffers.
// nb: right-hand sides of a batched solve (a power of two), 0 for the single-vector solver.
int64_t estimate_bytes(int64_t N, const momed_solve_opts& o, int64_t nb = 0, bool single = false) {
    int64_t m = o.krylovdim > 0 ? o.krylovdim : 30;
    if (m > N) m = N;
    int64_t nev = o.nev;
    int64_t b = 8 * N;                                // basis
    if (nb == 0 && !single && nev >= 2 && N >= 500000) {
        // the block solver (momed_eigsolve for nev >= 2 on large sectors): a block basis of mb
        // blocks of B vectors and its restart copy (FP64 at worst), the Ritz and returned vectors
        const int64_t B = nev <= 4 ? 4 : (nev <= 10 ? 8 : 16);
        int64_t mb = B <= 4 ? 20 : (B <= 8 ? 16 : 8);
        mb = std::max<int64_t>(mb, (m + B - 1) / B + 2);
        mb = std::min<int64_t>(mb, std::min<int64_t>(256, 2048 / B) / B);
        b += 2 * (mb + 1) * N * B * 16;
        b += 4 * (nev + 4) * N * 16;
    } else if (nb > 0) {
        // batched solver: the Krylov basis and its restart copy (FP64 fallback at worst), Ritz
        // vectors X, W = H X and scratch, the fallback's vectors and the returned vectors
        const int64_t k1 = nev + 4;
        b += 2 * (m + 1) * N * nb * 16;
        b += 3 * k1 * N * nb * 16;
        b += 2 * std::max<int64_t>(k1, nev) * N * nb * 16;
    } else if (o.precision == MOMED_PREC_MIXED) {
        const int64_t k1 = nev + 4;                   // single vector: FP32 basis, FP64 finish
        b += 2 * (m + 1) * N * 16;
        b += 3 * k1 * N * 16;
        b += 2 * std::max<int64_t>(k1, nev) * N * 16;
    } else {
        b += 2 * (m + 1) * N * 16;                    // Krylov basis and restart scratch
        b += 2 * std::max<int64_t>(nev, 1) * N * 16;  // output vectors + residual workspace
    }
    b += 16ll << 20;                                  // index tables, term lists, partial sums
    return b;
}

// Group parameters of a batched solve: nev, krylovdim and maxiter the largest, tol the smallest.
momed_solve_opts group_opts(const std::vector<std::shared_ptr<Request>>& g) {
    momed_solve_opts o = g[0]->opts;
    for (const auto& q : g) {
        o.nev = std::max(o.nev, q->opts.nev);
        o.krylovdim = std::max(o.krylovdim, q->opts.krylovdim);
        o.maxiter = std::max(o.maxiter, q->opts.maxiter);
        if (q->opts.tol > 0 && (o.tol <= 0 || q->opts.tol < o.tol)) o.tol = q->opts.tol;
    }
    o.want_vectors = 0;
    o.vecs_on_device = 0;
    return o;
}

// policy switches read per request (environment; for measurements of the serving policy)
std::string knob(const char* name, const char* dflt) {
    const char* e = std::getenv(name);
    return e ? std::string(e) : std::string(dflt);
}

int64_t pow2_at_least(int64_t n) {
    int64_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

void worker_loop(momed_server* S, int slot) {
    momed_handle* h = S->handles[slot];
    cudaSetDevice(S->device);
    AllocScope scope(h->stream);       // this slot's buffers are ordered on its own stream
    int32_t cur_op = -1;               // operator resident on this slot's handle
    for (;;) {
        std::vector<std::shared_ptr<Request>> grp;
        std::shared_ptr<const HostOperator> opp;
        int64_t gbytes = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // admission in arrival order: the first queued request that fits the free budget and,
            // if it is large, finds no other large group running (a request waiting for memory
            // holds back the ones behind it)
            std::deque<std::shared_ptr<Request>>::iterator pick;
            auto find = [&]() {
                while (!S->queue.empty() && S->queue.front()->status == 4) S->queue.pop_front();
                const int large_max = std::max(1, std::atoi(knob("MOMED_SERVE_LARGE_MAX", "1").c_str()));
                for (auto it = S->queue.begin(); it != S->queue.end(); ++it) {
                    if ((*it)->status == 4) continue;
                    if ((int64_t)(*it)->basis.size() >= kLargeRows && S->large_running >= large_max) continue;
                    if (S->used + (*it)->bytes > S->budget) return false;
                    pick = it;
                    return true;
                }
                return false;
            };
            S->cv_work.wait(lk, [&] { return S->stopping || find(); });
            if (S->stopping) return;
            auto r = *pick;
            S->queue.erase(pick);
            grp.push_back(r);
            gbytes = r->bytes;
            if (r->op >= 0 && r->op < (int32_t)S->ops.size()) opp = S->ops[r->op];
            // continuous batching: queued requests on the same operator, sector and precision join
            // the head when the group reaches kMinGroup (smaller groups cost as much per solve as
            // the single-vector solver)
            // Only mixed-precision requests with nev <= kMaxMixedNev form groups: an FP64 group (the
            // block Lanczos in FP64 on the matrix-free map) took longer than its requests solved
            // one by one with the sparse method (3x10, nev 15/8/11: 6.4 s against ~0.8 s each).
            const int64_t N = (int64_t)r->basis.size();
            // Without the hit cache (MOMED_SERVE_HITCACHE=0), a request whose sparse matrix will fit
            // is solved alone on it: measured on the serving stream, a group of three 3x10 requests
            // (nev 12) took 7.2 s on the batched solver over the candidate map and ~0.8 s each alone
            // on the sparse method.  The matrix size comes from the hits per row that earlier
            // solves on the operator measured.  Over the hit cache a group is one batched solve
            // whose block map serves every member's right-hand side.
            const bool use_hc = knob("MOMED_SERVE_HITCACHE", "1") != "0";
            bool sparse_fits = false;
            if (!use_hc && N >= kSparseMinRows && opp && r->op < (int32_t)S->op_hits_per_row.size() &&
                knob("MOMED_SERVE_SPARSE", "1") != "0") {
                const double hpr = S->op_hits_per_row[r->op];
                const int64_t sp = (N + 1) * 8 + (int64_t)((hpr + 1.0) * (double)N) * sparse_bytes_per_entry(opp->has_b);
                sparse_fits = hpr > 0.0 && S->used + r->bytes + sp <= S->budget;
            }
            const bool groupable = r->opts.precision == MOMED_PREC_MIXED && r->opts.nev <= kMaxMixedNev && !sparse_fits;
            for (auto it = S->queue.begin(); groupable && it != S->queue.end() && grp.size() < 32; ++it) {
                const auto& q = *it;
                const bool same = q->status == 0 && q->op == r->op && q->opts.precision == r->opts.precision &&
                                  q->opts.nev <= kMaxMixedNev && q->bhash == r->bhash &&
                                  (int64_t)q->basis.size() == N &&
                                  std::memcmp(q->basis.data(), r->basis.data(), (size_t)N * 8) == 0;
                if (!same) continue;
                grp.push_back(q);
                const int64_t need = estimate_bytes(N, group_opts(grp), pow2_at_least((int64_t)grp.size()));
                if (S->used + need > S->budget) {
                    grp.pop_back();
                    break;
                }
            }
            const int min_group = std::max(2, std::atoi(knob("MOMED_SERVE_MIN_GROUP", std::to_string(kMinGroup).c_str()).c_str()));
            if ((int)grp.size() >= min_group) {
                gbytes = estimate_bytes(N, group_opts(grp), pow2_at_least((int64_t)grp.size()));
                auto taken = [&](const std::shared_ptr<Request>& q) {
                    return std::find(grp.begin() + 1, grp.end(), q) != grp.end();
                };
                S->queue.erase(std::remove_if(S->queue.begin(), S->queue.end(), taken), S->queue.end());
            } else {
                grp.resize(1);
            }
            S->used += gbytes;
            if (N >= kLargeRows) ++S->large_running;
            const auto now = clock_t_::now();
            for (auto& q : grp) {
                q->status = 1;
                q->start = now;
            }
        }
        int rc = MOMED_OK;
        std::string err;
        std::vector<double> gvals, gres;
        momed_info ginfo{};
        const auto& r = grp[0];
        const int nu = (int)grp.size();
        try {
            MOMED_REQUIRE(opp != nullptr, MOMED_EINVAL, "unknown operator id");
            const HostOperator& op = *opp;
            const int64_t N = (int64_t)r->basis.size();
            h->basis.resize(std::max<int64_t>(N, 1));
            MOMED_CUDA_TRY(cudaMemcpyAsync(h->basis.p, r->basis.data(), N * 8, cudaMemcpyHostToDevice, h->stream));
            h->n = N;
            h->hcache.release();
            h->index_dirty = true;
            h->op_validated = false;
            h->basis_or = 0;
            for (uint64_t v : r->basis) h->basis_or |= v;
            if (cur_op != r->op) {
                cur_op = -1;
                upload_operator(h, op.amp_a.data(), op.has_b ? op.amp_b.data() : nullptr, op.in.data(),
                                op.out.data(), op.parity.empty() ? nullptr : op.parity.data(), (int64_t)op.in.size());
                cur_op = r->op;
            }
            momed_solve_opts o = group_opts(grp);
            const int nev = (int)std::min<int64_t>(o.nev, N);
            gvals.assign((size_t)nu * nev, 0.0);
            gres.assign((size_t)nu * nev, 0.0);
            const double u = r->u;
            if (nu == 1) {
                // the handle's u, host copy and device copies alike: the solvers read the host copy
                // (the mixed path's batched solve, the combined amplitudes of the cached map)
                float uf = (float)u;
                h->u = u;
                MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev.p, &u, sizeof(u), cudaMemcpyHostToDevice, h->stream));
                MOMED_CUDA_TRY(cudaMemcpyAsync(h->u_dev32.p, &uf, sizeof(uf), cudaMemcpyHostToDevice, h->stream));
                MOMED_CUDA_TRY(cudaStreamSynchronize(h->stream));
            }
            // The map's hit cache when it fits what the budget has left, else the sparse method
            // when its matrix fits (their bytes are held for this solve only); otherwise the
            // candidate map.  A group's batched solver runs its FP32 maps over the cache (or as a
            // block SpMV over the matrix).  MOMED_SERVE_HITCACHE=0 / MOMED_SERVE_SPARSE=0 skip one.
            int64_t sp_bytes = 0, hc_bytes = 0;
            int hc_mode = 1;
            if (N >= kSparseMinRows) {
                ensure_ready(h);                      // index and validation: h->nnz counts every hit
                std::lock_guard<std::mutex> lk(S->mu);
                S->op_hits_per_row[r->op] = (double)h->nnz / (double)N;
                if (knob("MOMED_SERVE_HITCACHE", "1") != "0") {
                    const int64_t need = hit_cache_bytes(N, h->nnz);
                    if (S->used + need <= S->budget) {
                        S->used += need;
                        hc_bytes = need;
                    }
                }
                if (hc_bytes == 0 && knob("MOMED_SERVE_SPARSE", "1") != "0") {
                    const int64_t need = (N + 1) * 8 + (h->nnz + N) * sparse_bytes_per_entry(h->op.has_b);
                    if (S->used + need <= S->budget) {
                        S->used += need;
                        sp_bytes = need;
                    }
                }
                // neither fits (the 35M-state sectors): the cache's slot mode, 2 bytes per hit,
                // for the single-vector map
                if (hc_bytes == 0 && sp_bytes == 0 && h->op.nterms <= 65536 &&
                    knob("MOMED_SERVE_HITCACHE", "1") != "0") {
                    const int64_t need = slot_cache_bytes(N, h->nnz);
                    if (S->used + need <= S->budget) {
                        S->used += need;
                        hc_bytes = need;
                        hc_mode = 2;
                    }
                }
            }
            auto unreserve = [&]() {
                h->sparse.release();
                h->hcache.release();
                if (sp_bytes > 0 || hc_bytes > 0) {
                    std::lock_guard<std::mutex> lk(S->mu);
                    S->used -= sp_bytes + hc_bytes;
                    sp_bytes = hc_bytes = 0;
                }
            };
            try {
                if (hc_bytes > 0) {
                    try {
                        build_hit_cache(h, hc_mode);
                    } catch (const Error& e) {
                        if (e.code != MOMED_ENOMEM) throw;
                        unreserve();          // the device is shorter than the budget: candidate map
                    }
                }
                if (sp_bytes > 0) {
                    try {
                        build_sparse(h, u);
                    } catch (const Error& e) {
                        if (e.code != MOMED_ENOMEM) throw;
                        unreserve();          // the device is shorter than the budget: use the map
                    }
                }
                h->block_solver = (nu == 1 && r->single) ? 0 : -1;
                if (nu == 1) {
                    // one right-hand side, in the request's precision: a mixed request runs the
                    // batched solver with one right-hand side over the hit cache (seed-4 stream:
                    // 4.35 served solves/s against 3.98 with FP64 for every request alone,
                    // eigenvalues within 4e-13 of FP64).  MOMED_SERVE_ALONE=fp64 gives every
                    // request alone FP64 arithmetic.
                    // (over a slot-mode cache the batched solver's block maps would fall back to the
                    // candidate map, so such a request runs FP64 on the single-vector map)
                    const bool alone_mixed = knob("MOMED_SERVE_ALONE", "mixed") == "mixed" &&
                                             !(h->hcache.built && h->hcache.mode == 2);
                    o.precision = (alone_mixed && r->opts.precision == MOMED_PREC_MIXED) ? MOMED_PREC_MIXED
                                                                                         : MOMED_PREC_FP64;
                    rc = momed_eigsolve_impl(h, &o, nullptr, gvals.data(), gres.data(), nullptr, &ginfo);
                } else {
                    std::vector<double> us(nu);
                    for (int i = 0; i < nu; ++i) us[i] = grp[i]->u;
                    rc = momed_batch_solve_impl(h, &o, us.data(), nu, gvals.data(), gres.data(), nullptr, &ginfo);
                }
            } catch (...) {
                unreserve();
                throw;
            }
            unreserve();
            if (rc == MOMED_ENOTCONV) rc = MOMED_OK;   // results written; info.converged tells
            for (int i = 0; i < nu; ++i) {
                const int ni = (int)std::min<int64_t>(grp[i]->opts.nev, N);
                grp[i]->vals.assign(gvals.begin() + (size_t)i * nev, gvals.begin() + (size_t)i * nev + ni);
                grp[i]->resid.assign(gres.begin() + (size_t)i * nev, gres.begin() + (size_t)i * nev + ni);
                grp[i]->info = ginfo;
                grp[i]->info.converged = std::min<int32_t>(ginfo.converged, ni);
            }
        } catch (const Error& e) {
            rc = e.code;
            err = e.msg;
        } catch (const std::exception& e) {
            rc = MOMED_EINVAL;
            err = e.what();
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            const auto now = clock_t_::now();
            for (auto& q : grp) {
                q->done = now;
                q->rc = rc;
                q->err = err;
                q->status = rc == MOMED_OK ? 2 : 3;
                if (rc == MOMED_OK) ++S->completed; else ++S->failed;
            }
            S->used -= gbytes;
            if ((int64_t)r->basis.size() >= kLargeRows) --S->large_running;
        }
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

MOMED_API int momed_serve_start(int device, int32_t slots, int64_t hbm_budget, momed_server** out) {
    if (!out || slots < 1 || slots > 64) return MOMED_EINVAL;
    *out = nullptr;
    momed_server* S = new momed_server();
    S->device = device;
    size_t freeb = 0, totalb = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) {
        delete S;
        return MOMED_ENODEV;
    }
    S->budget = hbm_budget > 0 ? std::min<int64_t>(hbm_budget, (int64_t)(freeb * 0.9)) : (int64_t)(freeb * 0.85);
    for (int i = 0; i < slots; ++i) {
        momed_handle* h = nullptr;
        int rc = momed_create(device, &h);
        if (rc != MOMED_OK) {
            for (auto* x : S->handles) momed_destroy(x);
            delete S;
            return rc;
        }
        h->hit_cache_ok = false;           // the admission budget does not count a hit cache
        S->handles.push_back(h);
    }
    for (int i = 0; i < slots; ++i) S->workers.emplace_back(worker_loop, S, i);
    *out = S;
    return MOMED_OK;
}

MOMED_API int momed_serve_register_operator(momed_server* S, const double* amp_a, const double* amp_b,
                                            const uint64_t* in, const uint64_t* out, const uint64_t* parity,
                                            int64_t nscat, int32_t* op_id) {
    if (!S || !amp_a || !in || !out || nscat < 0 || !op_id) return MOMED_EINVAL;
    HostOperator op;
    op.amp_a.assign(amp_a, amp_a + 2 * nscat);
    if (amp_b) { op.amp_b.assign(amp_b, amp_b + 2 * nscat); op.has_b = true; }
    op.in.assign(in, in + nscat);
    op.out.assign(out, out + nscat);
    if (parity) op.parity.assign(parity, parity + nscat);
    else op.parity.clear();
    std::lock_guard<std::mutex> lk(S->mu);
    S->ops.push_back(std::make_shared<const HostOperator>(std::move(op)));
    S->op_hits_per_row.push_back(0.0);
    *op_id = (int32_t)S->ops.size() - 1;
    return MOMED_OK;
}

MOMED_API int momed_serve_submit(momed_server* S, int32_t op_id, const uint64_t* basis, int64_t n, double u,
                                 const momed_solve_opts* opts, int64_t* request_id) {
    if (!S || !basis || n <= 0 || !opts || !request_id || opts->nev < 1) return MOMED_EINVAL;
    auto r = std::make_shared<Request>();
    r->op = op_id;
    r->basis.assign(basis, basis + n);
    r->u = u;
    r->opts = *opts;
    r->bytes = estimate_bytes(n, *opts);
    if (r->bytes > S->budget) {          // the block solver's basis does not fit: single-vector Lanczos
        r->single = true;
        r->bytes = estimate_bytes(n, *opts, 0, true);
    }
    uint64_t hsh = 0x9E3779B97F4A7C15ull ^ (uint64_t)n;
    for (int64_t i = 0; i < n; ++i) {
        hsh ^= basis[i] + 0x9E3779B97F4A7C15ull + (hsh << 6) + (hsh >> 2);
    }
    r->bhash = hsh;
    r->arrival = clock_t_::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (op_id < 0 || op_id >= (int32_t)S->ops.size()) {
        S->last_error = "unknown operator id";
        return MOMED_EINVAL;
    }
    r->id = S->next_id++;
    *request_id = r->id;
    S->all[r->id] = r;
    if (r->bytes > S->budget) {   // can never be admitted: refuse now
        r->status = 3;
        r->rc = MOMED_ENOMEM;
        r->err = "request needs " + std::to_string(r->bytes) + " bytes of HBM, budget is " + std::to_string(S->budget);
        r->done = r->arrival;
        ++S->failed;
        S->cv_done.notify_all();
        return MOMED_OK;
    }
    S->queue.push_back(r);
    S->cv_work.notify_all();
    return MOMED_OK;
}

MOMED_API int momed_serve_cancel(momed_server* S, int64_t request_id) {
    if (!S) return MOMED_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->all.find(request_id);
    if (it == S->all.end()) return MOMED_EINVAL;
    if (it->second->status != 0) return MOMED_ESTATE;   // only queued requests can be cancelled
    it->second->status = 4;
    it->second->done = clock_t_::now();
    S->cv_done.notify_all();
    return MOMED_OK;
}

// Wait up to wait_ms for the request to finish.  status: 0 queued, 1 running, 2 done,
// 3 failed, 4 cancelled.  Times in seconds from arrival.  vals/resid (nev each) may be NULL.
MOMED_API int momed_serve_poll(momed_server* S, int64_t request_id, int32_t wait_ms, int32_t* status, double* vals,
                               double* resid, momed_info* info, double* queue_s, double* latency_s) {
    if (!S || !status) return MOMED_EINVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(request_id);
    if (it == S->all.end()) return MOMED_EINVAL;
    auto r = it->second;
    auto finished = [&] { return r->status >= 2; };
    if (wait_ms > 0) S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), finished);
    *status = r->status;
    if (!finished()) return wait_ms > 0 ? MOMED_ETIMEOUT : MOMED_OK;
    if (r->status == 3) {
        S->last_error = r->err;
        return r->rc;
    }
    if (r->status == 2) {
        for (size_t i = 0; i < r->vals.size(); ++i) {
            if (vals) vals[i] = r->vals[i];
            if (resid) resid[i] = r->resid[i];
        }
        if (info) *info = r->info;
    }
    if (queue_s) *queue_s = std::chrono::duration<double>(r->start - r->arrival).count();
    if (latency_s) *latency_s = std::chrono::duration<double>(r->done - r->arrival).count();
    return MOMED_OK;
}

MOMED_API int momed_serve_stats(momed_server* S, int64_t* queued, int64_t* completed, int64_t* failed,
                                int64_t* hbm_used, int64_t* hbm_budget) {
    if (!S) return MOMED_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    if (queued) *queued = (int64_t)S->queue.size();
    if (completed) *completed = S->completed;
    if (failed) *failed = S->failed;
    if (hbm_used) *hbm_used = S->used;
    if (hbm_budget) *hbm_budget = S->budget;
    return MOMED_OK;
}

MOMED_API const char* momed_serve_last_error(momed_server* S) { return S ? S->last_error.c_str() : ""; }

MOMED_API int momed_serve_stop(momed_server* S) {
    if (!S) return MOMED_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto& t : S->workers) t.join();
    for (auto* h : S->handles) momed_destroy(h);
    delete S;
    return MOMED_OK;
}

}  // extern "C"
