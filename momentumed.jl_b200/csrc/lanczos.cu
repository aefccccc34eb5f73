// Thick-restart (Krylov-Schur) Lanczos eigensolver on the device.
//
// Replaces krylov_map_solve (MomentumEDCUDAExt.jl:159-179), which hands the GPU
// map to KrylovKit.eigsolve(H, x0, howmany, :SR; ishermitian) with KrylovKit's
// Lanczos + Krylov-Schur restart (krylovdim, maxiter, tol on the residual
// norm), a chunked GEMM restart (basistransform!, MomentumEDCUDAExt.jl:210-244)
// and a forced GC after every restart (shrink!, 248-272).  Here the Krylov
// basis, the recurrence coefficients and the reorthogonalisation coefficients
// live in HBM for the whole solve; the host sees only the small projected
// matrix once per restart cycle.  Nothing is allocated inside the loop.
//
// Precision forms:
//   FP64  - c128 matvec, c128 basis, FP64 everything.
//   MIXED - c64 matvec (FP32 accumulate) and c64 basis with FP64 dot
//           products, recurrences and projected eigensolve; then an FP64
//           Rayleigh-Ritz refinement (one FP64 matvec per Ritz vector, FP64
//           Gram matrices, generalized Hermitian eigensolve) that lifts the
//           eigenvalues to FP64 accuracy (error ~ residual^2 / gap); if the
//           estimated error is not below the target, an FP64 Lanczos run
//           warm-started from the refined vectors finishes the job.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>

#include "vecops.cuh"

namespace momed {

void ensure_ready(momed_handle* h);   // abi.cu

namespace {

__global__ void k_inv_sqrt(const double2* c, double* scal) {
    if (threadIdx.x == 0) {
        double v = c[0].x;
        scal[0] = v > 0.0 ? 1.0 / sqrt(v) : 0.0;
    }
}

template <typename VT> struct Prec;
template <> struct Prec<double2> { static constexpr int value = MOMED_C128; };
template <> struct Prec<float2> { static constexpr int value = MOMED_C64; };

// the CSR SpMV while a sparse matrix is built (momed_build_sparse), else the matrix-free map
// (over its hit cache while one is built)
void apply_h(momed_handle* h, const double2* x, double2* y) {
    prof_begin(h);
    if (h->sparse.built) {
        launch_spmv_c128(h->sparse, x, y, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_SPMV_C128);
        return;
    }
    if (h->hcache.built) {
        launch_matvec_hc_c128(h, x, y, h->op.has_b ? h->u_dev.p : nullptr, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_HC_MATVEC_C128);
        return;
    }
    launch_matvec_c128(index_view(h), h->op.view(), x, y, h->op.has_b ? h->u_dev.p : nullptr, h->n, h->stream);
    prof_end(h, MOMED_KERNEL_MATVEC_C128);
}
void apply_h(momed_handle* h, const float2* x, float2* y) {
    prof_begin(h);
    if (h->sparse.built) {
        launch_spmv_c64(h->sparse, x, y, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_SPMV_C64);
        return;
    }
    if (h->hcache.built) {
        launch_matvec_hc_c64(h, x, y, h->op.has_b ? h->u_dev32.p : nullptr, h->n, h->stream);
        prof_end(h, MOMED_KERNEL_HC_MATVEC_C64);
        return;
    }
    launch_matvec_c64(index_view(h), h->op.view(), x, y, h->op.has_b ? h->u_dev32.p : nullptr, h->n, h->stream);
    prof_end(h, MOMED_KERNEL_MATVEC_C64);
}

}  // namespace

void apply_h_fp64(momed_handle* h, const double2* x, double2* y) { apply_h(h, x, y); }

namespace {

struct RunOut {
    std::vector<double> theta, resid;   // all m Ritz values / residual estimates of the final cycle
    int nconv = 0, restarts = 0;
    int64_t matvecs = 0;
    int kept = 0;                       // Ritz vectors written to `vectors`
};

template <typename VT>
struct Lanczos {
    momed_handle* h;
    int64_t N;
    int m;
    cudaStream_t st;
    int grid;
    DevBuf<VT> V;
    DevBuf<double2> partial, coefA, coefB;
    DevBuf<double> scal, alpha, beta, Ud;
    DevBuf<int> flag;

    Lanczos(momed_handle* hh, int mm) : h(hh), N(hh->n), m(mm), st(hh->stream) {
        grid = vec_grid(N);
        V.resize((size_t)(m + 1) * N);
        partial.resize((size_t)grid * (kMaxCols + 1));
        coefA.resize(kMaxCols + 1);
        coefB.resize(kMaxCols + 1);
        scal.resize(4);
        alpha.resize(m);
        beta.resize(m);
        Ud.resize((size_t)m * m);
        flag.resize(1);
    }
    VT* col(int i) { return V.p + (size_t)i * N; }

    void normalize(VT* v) {
        vec_proj<VT>(v, N, 0, v, partial.p, grid, nullptr, st);
        vec_reduce(partial.p, grid, 1, coefA.p, nullptr, st);
        k_inv_sqrt<<<1, 32, 0, st>>>(coefA.p, scal.p);
        note_launches(1);
        vec_scale<VT>(v, N, scal.p, st);
    }
    // orthogonalise v against columns [0, ncols) twice, then normalise
    void orthonormalize(VT* v, int ncols) {
        for (int pass = 0; pass < 2 && ncols > 0; ++pass) {
            vec_proj<VT>(V.p, N, ncols, v, partial.p, grid, nullptr, st);
            vec_reduce(partial.p, grid, ncols + 1, coefA.p, nullptr, st);
            vec_update<VT>(V.p, N, ncols, coefA.p, v, partial.p, grid, nullptr, st);
        }
        normalize(v);
    }
    void step(int j) {
        VT* w = col(j + 1);
        apply_h(h, col(j), w);
        const int nc = j + 1;
        vec_proj<VT>(V.p, N, nc, w, partial.p, grid, nullptr, st);
        vec_reduce(partial.p, grid, nc + 1, coefA.p, nullptr, st);
        vec_update<VT>(V.p, N, nc, coefA.p, w, partial.p, grid, nullptr, st);
        vec_decide(coefA.p, nc, partial.p, grid, flag.p, scal.p, st);
        vec_proj<VT>(V.p, N, nc, w, partial.p, grid, flag.p, st);
        vec_reduce(partial.p, grid, nc + 1, coefB.p, flag.p, st);
        vec_update<VT>(V.p, N, nc, coefB.p, w, partial.p, grid, flag.p, st);
        vec_finalize(coefA.p, coefB.p, nc, partial.p, grid, flag.p, scal.p, alpha.p, beta.p, j, st);
        vec_scale<VT>(w, N, scal.p, st);
    }

    // Runs to convergence.  start: device vector of length N in VT (nullptr: random from seed).
    // rel_tol_floor: convergence also accepted at residual <= rel_tol_floor * max|theta|.
    // vectors (nullable, device double2, [nwant][N]): Ritz vectors of the nwant lowest pairs.
    RunOut run(int nev, double tol, double rel_tol_floor, int maxiter, const VT* start, uint64_t seed, int nwant,
               double2* vectors) {
        RunOut out;
        if (start) MOMED_CUDA_TRY(cudaMemcpyAsync(col(0), start, N * sizeof(VT), cudaMemcpyDeviceToDevice, st));
        else vec_random<VT>(col(0), N, seed, st);
        normalize(col(0));
        std::vector<double> T((size_t)m * m), A((size_t)m * m), U((size_t)m * m), th(m), ha(m), hb(m);
        std::vector<double> kept_theta, arrow;
        int k = 0;
        int restarts = 0;
        int64_t matvecs = 0;
        for (;;) {
            int jstart = k;
            int mm = m;
            for (int j = jstart; j < m; ++j) { step(j); ++matvecs; }
            MOMED_CUDA_TRY(cudaMemcpyAsync(ha.data(), alpha.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaMemcpyAsync(hb.data(), beta.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            // invariant-subspace breakdown inside the cycle
            double scale = 0.0;
            for (int j = k; j < m; ++j) scale = std::max(scale, std::fabs(ha[j]));
            for (double t : kept_theta) scale = std::max(scale, std::fabs(t));
            for (int j = k; j + 1 < m; ++j) {
                if (hb[j] <= 1e-13 * std::max(scale, 1e-300)) {
                    if (j + 1 >= nev) { mm = j + 1; break; }
                    // not enough vectors yet: continue the basis with a fresh random direction
                    vec_random<VT>(col(j + 1), N, seed + 7919u * (uint64_t)(restarts + 1) + (uint64_t)j, st);
                    orthonormalize(col(j + 1), j + 1);
                    hb[j] = 0.0;
                    double zero = 0.0;
                    MOMED_CUDA_TRY(cudaMemcpyAsync(beta.p + j, &zero, sizeof(double), cudaMemcpyHostToDevice, st));
                    for (int jj = j + 1; jj < m; ++jj) { step(jj); ++matvecs; }
                    MOMED_CUDA_TRY(cudaMemcpyAsync(ha.data(), alpha.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
                    MOMED_CUDA_TRY(cudaMemcpyAsync(hb.data(), beta.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
                    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                    hb[j] = 0.0;
                }
            }
            const double beta_last = (mm == m) ? hb[m - 1] : 0.0;
            std::fill(T.begin(), T.end(), 0.0);
            for (int i = 0; i < k; ++i) {
                T[(size_t)i * m + i] = kept_theta[i];
                T[(size_t)i * m + k] = arrow[i];
                T[(size_t)k * m + i] = arrow[i];
            }
            for (int j = k; j < mm; ++j) {
                T[(size_t)j * m + j] = ha[j];
                if (j + 1 < mm) { T[(size_t)j * m + j + 1] = hb[j]; T[(size_t)(j + 1) * m + j] = hb[j]; }
            }
            for (int a = 0; a < mm; ++a)
                for (int b = 0; b < mm; ++b) A[(size_t)a * mm + b] = T[(size_t)a * m + b];
            symeig(mm, A.data(), th.data(), U.data());
            double tmax = 0.0;
            for (int i = 0; i < mm; ++i) tmax = std::max(tmax, std::fabs(th[i]));
            const double eff_tol = std::max(tol, rel_tol_floor * tmax);
            std::vector<double> res(mm);
            for (int i = 0; i < mm; ++i) res[i] = std::fabs(beta_last * U[(size_t)(mm - 1) * mm + i]);
            int nconv = 0;
            while (nconv < nev && nconv < mm && res[nconv] <= eff_tol) ++nconv;
            if (nconv >= nev || restarts >= maxiter || mm < m) {
                out.theta.assign(th.begin(), th.begin() + mm);
                out.resid = res;
                out.nconv = nconv;
                out.restarts = restarts;
                out.matvecs = matvecs;
                int nv = std::min(nwant, mm);
                out.kept = nv;
                if (vectors && nv > 0) {
                    std::vector<double> Uc((size_t)mm * nv);
                    for (int i = 0; i < nv; ++i)
                        for (int a = 0; a < mm; ++a) Uc[(size_t)i * mm + a] = U[(size_t)a * mm + i];
                    MOMED_CUDA_TRY(cudaMemcpyAsync(Ud.p, Uc.data(), Uc.size() * 8, cudaMemcpyHostToDevice, st));
                    vec_combine<VT, double2>(V.p, N, mm, Ud.p, nv, vectors, N, -1, st);
                    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
                }
                return out;
            }
            int keep = (3 * m + 2 * nconv) / 5;
            keep = std::max(keep, std::min(nwant, m - 2));
            keep = std::max(keep, nev);
            keep = std::min(keep, m - 2);
            keep = std::max(keep, 1);
            std::vector<double> Uc((size_t)m * keep);
            for (int i = 0; i < keep; ++i)
                for (int a = 0; a < m; ++a) Uc[(size_t)i * m + a] = U[(size_t)a * m + i];
            MOMED_CUDA_TRY(cudaMemcpyAsync(Ud.p, Uc.data(), Uc.size() * 8, cudaMemcpyHostToDevice, st));
            vec_combine<VT, VT>(V.p, N, m, Ud.p, keep, V.p, N, m, st);
            kept_theta.assign(th.begin(), th.begin() + keep);
            arrow.resize(keep);
            for (int i = 0; i < keep; ++i) arrow[i] = beta_last * U[(size_t)(m - 1) * m + i];
            k = keep;
            ++restarts;
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));   // Uc must outlive the async copy
        }
    }
};

int pick_m(int64_t N, int nev, int krylovdim) {
    int m = krylovdim > 0 ? krylovdim : 30;
    if (m > kMaxCols - 1) m = kMaxCols - 1;
    if (m > N) m = (int)N;
    if (m < nev + 2 && m < N) m = (int)std::min<int64_t>(N, nev + 2);
    return std::max(m, 1);
}

}  // namespace

// Generalised Hermitian eigenproblem G y = theta S y (k x k, column-major complex) on the host:
// S = L L^H (Cholesky), C = L^-1 G L^-H, embed C in a real symmetric 2k x 2k matrix, pick
// one eigenvector per eigenvalue pair, Y = L^-H z.  Returns false if S is not positive definite.
bool gen_herm_eig(int k, const std::vector<std::complex<double>>& G, const std::vector<std::complex<double>>& S,
                  std::vector<double>& theta, std::vector<std::complex<double>>& Y) {
    using cd = std::complex<double>;
    auto g = [&](int r, int c) { return G[(size_t)c * k + r]; };
    auto s = [&](int r, int c) { return S[(size_t)c * k + r]; };
    std::vector<cd> L((size_t)k * k, 0.0);   // row-major lower
    for (int j = 0; j < k; ++j) {
        double d = s(j, j).real();
        for (int p = 0; p < j; ++p) d -= std::norm(L[(size_t)j * k + p]);
        if (d <= 0.0) return false;
        L[(size_t)j * k + j] = std::sqrt(d);
        for (int i = j + 1; i < k; ++i) {
            cd v = s(i, j);
            for (int p = 0; p < j; ++p) v -= L[(size_t)i * k + p] * std::conj(L[(size_t)j * k + p]);
            L[(size_t)i * k + j] = v / L[(size_t)j * k + j];
        }
    }
    // M = L^-1 G  (forward substitution on columns), then C = M L^-H = (L^-1 M^H)^H
    std::vector<cd> M((size_t)k * k), C((size_t)k * k);
    for (int c = 0; c < k; ++c)
        for (int r = 0; r < k; ++r) {
            cd v = g(r, c);
            for (int p = 0; p < r; ++p) v -= L[(size_t)r * k + p] * M[(size_t)p * k + c];
            M[(size_t)r * k + c] = v / L[(size_t)r * k + r];
        }
    // C^H = L^-1 M^H  -> solve for columns of M^H
    std::vector<cd> CH((size_t)k * k);
    for (int c = 0; c < k; ++c)
        for (int r = 0; r < k; ++r) {
            cd v = std::conj(M[(size_t)c * k + r]);
            for (int p = 0; p < r; ++p) v -= L[(size_t)r * k + p] * CH[(size_t)p * k + c];
            CH[(size_t)r * k + c] = v / L[(size_t)r * k + r];
        }
    for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) C[(size_t)r * k + c] = 0.5 * (std::conj(CH[(size_t)c * k + r]) + CH[(size_t)r * k + c]);
    // real embedding [[Re, -Im], [Im, Re]]
    const int n2 = 2 * k;
    std::vector<double> A((size_t)n2 * n2), w(n2), Z((size_t)n2 * n2);
    for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) {
            cd v = C[(size_t)r * k + c];
            A[(size_t)r * n2 + c] = v.real();
            A[(size_t)r * n2 + c + k] = -v.imag();
            A[(size_t)(r + k) * n2 + c] = v.imag();
            A[(size_t)(r + k) * n2 + c + k] = v.real();
        }
    symeig(n2, A.data(), w.data(), Z.data());
    // eigenvalues come in equal pairs; take every other one, orthogonalising within pairs
    theta.assign(k, 0.0);
    Y.assign((size_t)k * k, 0.0);
    std::vector<cd> zs((size_t)k * k);
    for (int i = 0; i < k; ++i) {
        int col = 2 * i;
        theta[i] = 0.5 * (w[col] + w[col + 1]);
        // complex vector z = x + i y from the real eigenvector (x; y)
        cd nrm = 0.0;
        std::vector<cd> z(k);
        for (int r = 0; r < k; ++r) z[r] = cd(Z[(size_t)r * n2 + col], Z[(size_t)(r + k) * n2 + col]);
        // Gram-Schmidt against previous z's (degenerate eigenvalues)
        for (int p = 0; p < i; ++p) {
            cd dot = 0.0;
            for (int r = 0; r < k; ++r) dot += std::conj(zs[(size_t)p * k + r]) * z[r];
            for (int r = 0; r < k; ++r) z[r] -= dot * zs[(size_t)p * k + r];
        }
        double nn = 0.0;
        for (int r = 0; r < k; ++r) nn += std::norm(z[r]);
        nn = std::sqrt(nn);
        if (nn < 1e-8) {   // the pair partner carries the independent direction
            for (int r = 0; r < k; ++r) z[r] = cd(Z[(size_t)r * n2 + col + 1], Z[(size_t)(r + k) * n2 + col + 1]);
            for (int p = 0; p < i; ++p) {
                cd dot = 0.0;
                for (int r = 0; r < k; ++r) dot += std::conj(zs[(size_t)p * k + r]) * z[r];
                for (int r = 0; r < k; ++r) z[r] -= dot * zs[(size_t)p * k + r];
            }
            nn = 0.0;
            for (int r = 0; r < k; ++r) nn += std::norm(z[r]);
            nn = std::sqrt(nn);
        }
        (void)nrm;
        for (int r = 0; r < k; ++r) zs[(size_t)i * k + r] = z[r] / nn;
    }
    // Y = L^-H Z  (back substitution with L^H upper)
    for (int c = 0; c < k; ++c)
        for (int r = k - 1; r >= 0; --r) {
            cd v = zs[(size_t)c * k + r];
            for (int p = r + 1; p < k; ++p) v -= std::conj(L[(size_t)p * k + r]) * Y[(size_t)c * k + p];
            Y[(size_t)c * k + r] = v / std::conj(L[(size_t)r * k + r]);
        }
    return true;
}

// FP64 Rayleigh-Ritz on the k columns of X (device c128, [k][N]): writes refined values,
// residual norms and (in place) refined vectors; W is scratch [k][N].
void rayleigh_ritz_fp64(momed_handle* h, double2* X, double2* W, double2* scratch, int k, std::vector<double>& theta,
                        std::vector<double>& resid, int64_t& matvecs) {
    const int64_t N = h->n;
    cudaStream_t st = h->stream;
    for (int i = 0; i < k; ++i) { apply_h(h, X + (size_t)i * N, W + (size_t)i * N); ++matvecs; }
    const int grid = vec_grid(N);
    DevBuf<double2> part, red;
    part.resize((size_t)grid * (kMaxCols + 1));
    red.resize(kMaxCols + 1);
    std::vector<std::complex<double>> G((size_t)k * k), S((size_t)k * k);
    std::vector<double2> tmp(kMaxCols + 1);
    for (int pass = 0; pass < 2; ++pass) {
        double2* rhs = pass == 0 ? W : X;
        for (int i = 0; i < k; ++i) {
            vec_proj<double2>(X, N, k, rhs + (size_t)i * N, part.p, grid, nullptr, st);
            vec_reduce(part.p, grid, k + 1, red.p, nullptr, st);
            MOMED_CUDA_TRY(cudaMemcpyAsync(tmp.data(), red.p, (k + 1) * sizeof(double2), cudaMemcpyDeviceToHost, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            for (int a = 0; a < k; ++a) {
                std::complex<double> v(tmp[a].x, tmp[a].y);   // X_a^H rhs_i
                (pass == 0 ? G : S)[(size_t)i * k + a] = v;
            }
        }
    }
    std::vector<std::complex<double>> Y;
    if (!gen_herm_eig(k, G, S, theta, Y)) throw Error{MOMED_ECUDA, "Rayleigh-Ritz Gram matrix is not positive definite"};
    DevBuf<double2> Yd;
    Yd.resize((size_t)k * k);
    std::vector<double2> Yh((size_t)k * k);
    for (size_t i = 0; i < Yh.size(); ++i) Yh[i] = make_double2(Y[i].real(), Y[i].imag());
    MOMED_CUDA_TRY(cudaMemcpyAsync(Yd.p, Yh.data(), Yh.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    vec_combine_complex(X, N, k, Yd.p, scratch, st);
    MOMED_CUDA_TRY(cudaMemcpyAsync(X, scratch, (size_t)k * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    vec_combine_complex(W, N, k, Yd.p, scratch, st);
    MOMED_CUDA_TRY(cudaMemcpyAsync(W, scratch, (size_t)k * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    resid.assign(k, 0.0);
    vec_residual_norms(W, X, N, k, theta.data(), resid.data(), st);
}

}  // namespace momed

namespace momed {
int block_size_for(momed_handle* h, int nev, int precision);                    // block_lanczos.cu
bool eigsolve_block(momed_handle* h, const momed_solve_opts* o, int nev, int B, const double2* start64, double2* X,
                    std::vector<double>& theta, std::vector<double>& res, int& nconv, int& restarts, int64_t& matvecs,
                    int64_t& matvecs64);
}  // namespace momed

using namespace momed;

int momed_eigsolve_impl(momed_handle* h, const momed_solve_opts* o, const double* vec0, double* vals, double* resid,
                        void* vecs, momed_info* info) {
    if (!h->sparse.built) {                  // a built sparse matrix needs no index or operator check
        ensure_ready(h);
        ensure_hit_cache(h);
    }
    const int64_t N = h->n;
    const int nev = (int)std::min<int64_t>(o->nev, N);
    MOMED_REQUIRE(o->nev >= 1, MOMED_EINVAL, "N should be at least 1");
    const int m = pick_m(N, nev, o->krylovdim);
    const double tol = o->tol > 0 ? o->tol : 1e-12;
    const int maxiter = o->maxiter > 0 ? o->maxiter : 100;
    cudaStream_t st = h->stream;
    MOMED_CUDA_TRY(cudaEventRecord(h->ev0, st));
    auto t0 = std::chrono::steady_clock::now();
    DevBuf<double2> X;
    X.resize((size_t)std::max(nev, 1) * N);
    DevBuf<double2> start64;
    if (vec0) {
        start64.resize(N);
        MOMED_CUDA_TRY(cudaMemcpyAsync(start64.p, vec0, N * sizeof(double2), cudaMemcpyHostToDevice, st));
    }
    std::vector<double> theta, res;
    int nconv = 0, restarts = 0;
    int64_t matvecs = 0, matvecs64 = 0;
    // several wanted pairs on a large sector: the block solver (B vectors per map launch); a
    // block that loses rank sends the solve back to the single-vector solver below
    const int B = block_size_for(h, nev, o->precision);
    const bool blocked = B > 0 && eigsolve_block(h, o, nev, B, vec0 ? start64.p : nullptr, X.p, theta, res, nconv,
                                                 restarts, matvecs, matvecs64);
    // mixed precision on the map without a start vector: the batched solver with one right-hand
    // side at the handle's u (FP32 Lanczos, then its anchored FP64 refinement of the Ritz block,
    // which a single-vector FP64 restart from one combined vector cannot match); it returns exact
    // FP64 residuals and the vectors on the device
    const char* mb_env = std::getenv("MOMED_MIXED_BATCHED");
    if (!blocked && o->precision == MOMED_PREC_MIXED && !vec0 && !h->sparse.built && !(mb_env && mb_env[0] == '0')) {
        momed_solve_opts o2 = *o;
        o2.want_vectors = 1;
        o2.vecs_on_device = 1;
        const double u = h->u;
        const int rc = momed_batch_solve_impl(h, &o2, &u, 1, vals, resid, reinterpret_cast<double*>(X.p), info);
        if (vecs && o->want_vectors) {
            cudaMemcpyKind kind = o->vecs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
            MOMED_CUDA_TRY(cudaMemcpyAsync(vecs, X.p, (size_t)nev * N * sizeof(double2), kind, st));
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        }
        return rc;
    }
    if (blocked) {
    } else if (o->precision == MOMED_PREC_MIXED) {
        // phase 1: FP32 Lanczos to the FP32 floor
        const int extra = std::min<int>(4, std::max<int>(0, m - 2 - nev));
        const int k1 = nev + extra;
        DevBuf<double2> X1, W1, S1;
        X1.resize((size_t)k1 * N);
        W1.resize((size_t)k1 * N);
        S1.resize((size_t)k1 * N);
        RunOut r1;
        {
            Lanczos<float2> L(h, m);
            DevBuf<float2> start32;
            if (vec0) {
                start32.resize(N);
                vec_convert_from<float2>(start64.p, start32.p, N, st);
            }
            r1 = L.run(k1, 0.0, 2e-6, maxiter, vec0 ? start32.p : nullptr, o->seed, k1, X1.p);
        }
        matvecs += r1.matvecs;
        restarts += r1.restarts;
        const int kk = std::min(k1, r1.kept);
        // phase 2: FP64 Rayleigh-Ritz on the FP32 Ritz vectors
        std::vector<double> th2, rs2;
        rayleigh_ritz_fp64(h, X1.p, W1.p, S1.p, kk, th2, rs2, matvecs64);
        matvecs += kk;
        // accept when residual <= tol, or the error estimate r^2/gap is 1e-11 relative
        double outside = (int)r1.theta.size() > kk ? r1.theta[kk] : th2.back() + 1.0;
        bool ok = true;
        nconv = 0;
        for (int i = 0; i < nev; ++i) {
            double gap = std::fabs(outside - th2[i]);
            for (int j = 0; j < kk; ++j)
                if (j != i && std::fabs(th2[j] - th2[i]) > 1e-9 * std::max(1.0, std::fabs(th2[i])))
                    gap = std::min(gap, std::fabs(th2[j] - th2[i]));
            double est = rs2[i] * rs2[i] / std::max(gap, 1e-300);
            bool good = rs2[i] <= tol || est <= 1e-11 * std::max(1.0, std::fabs(th2[i]));
            if (good && nconv == i) ++nconv;
            ok = ok && good;
        }
        if (ok) {
            theta = th2;
            res = rs2;
            MOMED_CUDA_TRY(cudaMemcpyAsync(X.p, X1.p, (size_t)nev * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        } else {
            // phase 3: FP64 Lanczos warm-started from the refined vectors
            DevBuf<double2> sv;
            sv.resize(N);
            std::vector<double> ones(kk, 1.0);
            DevBuf<double> Ud;
            Ud.resize(kk);
            MOMED_CUDA_TRY(cudaMemcpyAsync(Ud.p, ones.data(), kk * 8, cudaMemcpyHostToDevice, st));
            vec_combine<double2, double2>(X1.p, N, kk, Ud.p, 1, sv.p, N, -1, st);
            MOMED_CUDA_TRY(cudaStreamSynchronize(st));
            Lanczos<double2> L(h, m);
            RunOut r3 = L.run(nev, tol, 0.0, maxiter, sv.p, o->seed, nev, X.p);
            theta = r3.theta;
            res = r3.resid;
            nconv = r3.nconv;
            matvecs += r3.matvecs;
            matvecs64 += r3.matvecs;
            restarts += r3.restarts;
        }
    } else {
        Lanczos<double2> L(h, m);
        RunOut r = L.run(nev, tol, 0.0, maxiter, vec0 ? start64.p : nullptr, o->seed, nev, X.p);
        theta = r.theta;
        res = r.resid;
        nconv = r.nconv;
        restarts = r.restarts;
        matvecs = matvecs64 = r.matvecs;
    }
    // true residuals ||H x - e x|| in FP64 for the returned pairs
    {
        DevBuf<double2> W;
        W.resize((size_t)nev * N);
        for (int i = 0; i < nev; ++i) apply_h(h, X.p + (size_t)i * N, W.p + (size_t)i * N);
        std::vector<double> tr(nev);
        vec_residual_norms(W.p, X.p, N, nev, theta.data(), tr.data(), st);
        for (int i = 0; i < nev; ++i) res[i] = tr[i];
    }
    for (int i = 0; i < nev; ++i) {
        vals[i] = theta[i];
        if (resid) resid[i] = res[i];
    }
    if (vecs && o->want_vectors) {
        cudaMemcpyKind kind = o->vecs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        MOMED_CUDA_TRY(cudaMemcpyAsync(vecs, X.p, (size_t)nev * N * sizeof(double2), kind, st));
    }
    MOMED_CUDA_TRY(cudaEventRecord(h->ev1, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    (void)t0;
    if (info) {
        info->converged = nconv;
        info->restarts = restarts;
        info->matvecs = matvecs;
        info->matvecs_fp64 = matvecs64;
        info->seconds = ms * 1e-3;
    }
    return nconv >= nev ? MOMED_OK : MOMED_ENOTCONV;
}
