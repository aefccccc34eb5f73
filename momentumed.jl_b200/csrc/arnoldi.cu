// Non-Hermitian eigensolver: Arnoldi with Krylov-Schur restarts, FP64, on the device map.
//
// EDsolve(...; ishermitian = false) hands the map of a non-Hermitian operator (the term list
// taken as it is, linear_map.jl:22-37 without completion; its adjoint is AdjointLinearMap,
// linear_map.jl:46-55, 120-139) to krylov_map_solve (MomentumEDCUDAExt.jl:159-179), i.e. to
// KrylovKit.eigsolve(H, x0, howmany, :SR; ishermitian = false): Arnoldi with Krylov-Schur
// restarts, complex eigenvalues ordered by real part.  Here:
//   - the Krylov basis V ((m + 1) x N, c128) lives in HBM; a step is one map, two classical
//     Gram-Schmidt passes against all columns (vec_proj / vec_update, FP64 reductions) and a
//     normalisation; the column of the projected matrix comes back to the host (m + 1 values);
//   - per cycle the host takes the complex Schur form of the m x m projected matrix
//     (schur.cpp), orders it by real part (:SR), tests the residuals |beta * (Z y_i)_m|, and
//     restarts by keeping the leading Schur vectors V Z[:, :k] and the residual vector, the
//     projected matrix becoming [T_k; b^T] (Krylov-Schur form).
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "vecops.cuh"

namespace momed {

void ensure_ready(momed_handle* h);
void apply_h_fp64(momed_handle* h, const double2* x, double2* y);
bool schur_complex(int n, std::vector<std::complex<double>>& A, std::vector<std::complex<double>>& Z);
void schur_reorder(int n, std::vector<std::complex<double>>& T, std::vector<std::complex<double>>& Z,
                   const std::vector<int>& order);
void tri_eigvecs(int n, const std::vector<std::complex<double>>& T, std::vector<std::complex<double>>& Y);

namespace {

using cd = std::complex<double>;

__global__ void k_scale_by(double2* v, int64_t N, double s) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
        v[n] = make_double2(v[n].x * s, v[n].y * s);
}

struct Arnoldi {
    momed_handle* h;
    int64_t N;
    int m;
    cudaStream_t st;
    int grid;
    DevBuf<double2> V, S, partial, coefA, coefB, Yd;
    int64_t matvecs = 0;

    Arnoldi(momed_handle* hh, int mm) : h(hh), N(hh->n), m(mm), st(hh->stream) {
        grid = vec_grid(N);
        V.resize((size_t)(m + 1) * N);
        S.resize((size_t)m * N);
        partial.resize((size_t)grid * (kMaxCols + 1));
        coefA.resize(kMaxCols + 1);
        coefB.resize(kMaxCols + 1);
        Yd.resize((size_t)m * m);
        // columns a cycle that ends early never writes take part (with zero weight) in the
        // recombinations: they must hold finite values
        MOMED_CUDA_TRY(cudaMemsetAsync(V.p, 0, (size_t)(m + 1) * N * sizeof(double2), st));
    }
    double2* col(int i) { return V.p + (size_t)i * N; }

    void scale(double2* v, double s) {
        k_scale_by<<<std::max(1, std::min(vec_grid(N), 1024)), kVecThreads, 0, st>>>(v, N, s);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(1);
    }
    // |v|^2 and the projections of v on columns [0, ncols) (one pass), on the host
    std::vector<cd> project(int ncols, const double2* v, double2* coef, double* norm2) {
        vec_proj<double2>(V.p, N, ncols, v, partial.p, grid, nullptr, st);
        vec_reduce(partial.p, grid, ncols + 1, coef, nullptr, st);
        std::vector<double2> t(ncols + 1);
        MOMED_CUDA_TRY(cudaMemcpyAsync(t.data(), coef, (ncols + 1) * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        std::vector<cd> c(ncols);
        for (int i = 0; i < ncols; ++i) c[i] = cd(t[i].x, t[i].y);
        if (norm2) *norm2 = t[ncols].x;
        return c;
    }
    // v against columns [0, ncols) twice; returns the summed coefficients and |v| after
    std::vector<cd> orthogonalize(double2* v, int ncols, double& beta) {
        std::vector<cd> c(ncols, 0.0);
        double n2 = 0.0;
        for (int pass = 0; pass < 2 && ncols > 0; ++pass) {
            double2* coef = pass == 0 ? coefA.p : coefB.p;
            std::vector<cd> cp = project(ncols, v, coef, nullptr);
            vec_update<double2>(V.p, N, ncols, coef, v, partial.p, grid, nullptr, st);
            for (int i = 0; i < ncols; ++i) c[i] += cp[i];
        }
        project(0, v, coefA.p, &n2);
        beta = std::sqrt(std::max(n2, 0.0));
        return c;
    }
    // new columns [0, nout) = V[:, 0..m) Y (Y column-major m x m, complex; columns beyond nout unused)
    void combine(const std::vector<cd>& Y, int nout, double2* out) {
        std::vector<double2> yh((size_t)m * m);
        for (size_t i = 0; i < yh.size(); ++i) yh[i] = make_double2(Y[i].real(), Y[i].imag());
        MOMED_CUDA_TRY(cudaMemcpyAsync(Yd.p, yh.data(), yh.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
        vec_combine_complex(V.p, N, m, Yd.p, S.p, st);
        MOMED_CUDA_TRY(cudaMemcpyAsync(out, S.p, (size_t)nout * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    }

    struct Out {
        std::vector<cd> theta;
        std::vector<double> resid;
        int nconv = 0, restarts = 0;
    };

    Out run(int nev, double tol, int maxiter, const double2* start, uint64_t seed, double2* vectors) {
        Out out;
        if (start) MOMED_CUDA_TRY(cudaMemcpyAsync(col(0), start, N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        else vec_random<double2>(col(0), N, seed, st);
        {
            double b;
            orthogonalize(col(0), 0, b);
            MOMED_REQUIRE(b > 0.0, MOMED_EINVAL, "start vector is zero");
            scale(col(0), 1.0 / b);
        }
        // projected matrix P (row-major m x m) and the coupling of the residual vector
        std::vector<cd> P((size_t)m * m, 0.0);
        int k = 0, restarts = 0;
        double beta = 0.0;
        for (;;) {
            int mm = m;
            for (int j = k; j < m; ++j) {
                double2* w = col(j + 1);
                apply_h_fp64(h, col(j), w);
                ++matvecs;
                std::vector<cd> c = orthogonalize(w, j + 1, beta);
                for (int i = 0; i <= j; ++i) P[(size_t)i * m + j] = c[i];
                if (j + 1 < m) P[(size_t)(j + 1) * m + j] = beta;
                // an invariant subspace: the projected matrix is exact
                double scl = 0.0;
                for (int i = 0; i <= j; ++i) scl = std::max(scl, std::abs(c[i]));
                if (beta <= 1e-14 * std::max(scl, 1e-300)) {
                    mm = j + 1;
                    beta = 0.0;
                    break;
                }
                scale(w, 1.0 / beta);
            }
            // Schur form of the leading mm x mm block, ordered by real part (:SR)
            std::vector<cd> T((size_t)mm * mm), Z;
            for (int a = 0; a < mm; ++a)
                for (int b = 0; b < mm; ++b) T[(size_t)a * mm + b] = P[(size_t)a * m + b];
            if (!schur_complex(mm, T, Z)) throw Error{MOMED_ECUDA, "Schur decomposition did not converge"};
            std::vector<int> ord(mm);
            for (int i = 0; i < mm; ++i) ord[i] = i;
            std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
                const cd a = T[(size_t)x * mm + x], b = T[(size_t)y * mm + y];
                return a.real() < b.real() || (a.real() == b.real() && a.imag() < b.imag());
            });
            schur_reorder(mm, T, Z, ord);
            std::vector<cd> Y;
            tri_eigvecs(mm, T, Y);
            // residual of Ritz pair i: |beta| |(Z y_i)_{mm-1}|
            std::vector<double> res(mm);
            std::vector<cd> theta(mm);
            for (int i = 0; i < mm; ++i) {
                theta[i] = T[(size_t)i * mm + i];
                cd last = 0.0;
                for (int p = 0; p <= i; ++p) last += Z[(size_t)(mm - 1) * mm + p] * Y[(size_t)p * mm + i];
                res[i] = std::fabs(beta) * std::abs(last);
            }
            int nconv = 0;
            while (nconv < nev && nconv < mm && res[nconv] <= tol) ++nconv;
            if (nconv >= nev || restarts >= maxiter || mm < m) {
                out.theta = theta;
                out.resid = res;
                out.nconv = nconv;
                out.restarts = restarts;
                if (vectors) {
                    const int nv = std::min(nev, mm);
                    std::vector<cd> Yc((size_t)m * m, 0.0);    // column-major: Yc[a + i*m] = (Z y_i)_a
                    for (int i = 0; i < nv; ++i)
                        for (int a = 0; a < mm; ++a) {
                            cd s = 0.0;
                            for (int p = 0; p <= i; ++p) s += Z[(size_t)a * mm + p] * Y[(size_t)p * mm + i];
                            Yc[(size_t)i * m + a] = s;
                        }
                    combine(Yc, nv, vectors);
                }
                return out;
            }
            // Krylov-Schur restart: keep the leading Schur vectors
            int keep = std::max(nev + 1, (m + nev) / 2);
            keep = std::min(keep, m - 2);
            std::vector<cd> Zc((size_t)m * m, 0.0);
            for (int i = 0; i < keep; ++i)
                for (int a = 0; a < m; ++a) Zc[(size_t)i * m + a] = Z[(size_t)a * m + i];
            combine(Zc, keep, V.p);
            MOMED_CUDA_TRY(cudaMemcpyAsync(col(keep), col(m), N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
            std::fill(P.begin(), P.end(), cd(0.0));
            for (int a = 0; a < keep; ++a)
                for (int b = a; b < keep; ++b) P[(size_t)a * m + b] = T[(size_t)a * mm + b];
            for (int i = 0; i < keep; ++i) P[(size_t)keep * m + i] = beta * Z[(size_t)(mm - 1) * mm + i];
            k = keep;
            ++restarts;
        }
    }
};

}  // namespace

}  // namespace momed

using namespace momed;

// vals: [nev] complex (re, im) ordered by real part; resid [nev]; vecs [nev][N] c128
int momed_eigsolve_general_impl(momed_handle* h, const momed_solve_opts* o, const double* vec0, double* vals,
                                double* resid, void* vecs, momed_info* info) {
    MOMED_REQUIRE(!h->sparse.built && !h->sparse_only, MOMED_ESTATE,
                  "the non-Hermitian solver runs on the matrix-free map (release the sparse matrix first)");
    ensure_ready(h);
    ensure_hit_cache(h);
    const int64_t N = h->n;
    MOMED_REQUIRE(o->nev >= 1, MOMED_EINVAL, "N should be at least 1");
    const int nev = (int)std::min<int64_t>(o->nev, N);
    int m = o->krylovdim > 0 ? o->krylovdim : 30;
    m = std::min(m, kMaxCols - 1);
    if (m > N) m = (int)N;
    if (m < nev + 3 && m < N) m = (int)std::min<int64_t>(N, nev + 3);
    const double tol = o->tol > 0 ? o->tol : 1e-12;
    const int maxiter = o->maxiter > 0 ? o->maxiter : 100;
    cudaStream_t st = h->stream;
    MOMED_CUDA_TRY(cudaEventRecord(h->ev0, st));
    DevBuf<double2> start, X;
    if (vec0) {
        start.resize(N);
        MOMED_CUDA_TRY(cudaMemcpyAsync(start.p, vec0, N * sizeof(double2), cudaMemcpyHostToDevice, st));
    }
    X.resize((size_t)nev * N);
    Arnoldi A(h, m);
    auto r = A.run(nev, tol, maxiter, vec0 ? start.p : nullptr, o->seed, X.p);
    const int nout = std::min<int>(nev, (int)r.theta.size());
    // true residuals ||H x - theta x|| in FP64
    DevBuf<double2> W;
    W.resize((size_t)N);
    std::vector<double> tr(nout, 0.0);
    for (int i = 0; i < nout; ++i) {
        apply_h_fp64(h, X.p + (size_t)i * N, W.p);
        // r = W - theta x: |r|^2 by one projection pass over [x] and |W|^2 (host arithmetic)
        std::vector<double2> wx(N), xx(N);
        MOMED_CUDA_TRY(cudaMemcpyAsync(wx.data(), W.p, N * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaMemcpyAsync(xx.data(), X.p + (size_t)i * N, N * sizeof(double2), cudaMemcpyDeviceToHost, st));
        MOMED_CUDA_TRY(cudaStreamSynchronize(st));
        double s = 0.0;
        const cd th = r.theta[i];
        for (int64_t n = 0; n < N; ++n) {
            const cd d = cd(wx[n].x, wx[n].y) - th * cd(xx[n].x, xx[n].y);
            s += std::norm(d);
        }
        tr[i] = std::sqrt(s);
    }
    for (int i = 0; i < nout; ++i) {
        vals[2 * i] = r.theta[i].real();
        vals[2 * i + 1] = r.theta[i].imag();
        if (resid) resid[i] = tr[i];
    }
    if (vecs && o->want_vectors) {
        cudaMemcpyKind kind = o->vecs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        MOMED_CUDA_TRY(cudaMemcpyAsync(vecs, X.p, (size_t)nout * N * sizeof(double2), kind, st));
    }
    MOMED_CUDA_TRY(cudaEventRecord(h->ev1, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (info) {
        info->converged = r.nconv;
        info->restarts = r.restarts;
        info->matvecs = A.matvecs + nout;
        info->matvecs_fp64 = A.matvecs + nout;
        info->seconds = ms * 1e-3;
    }
    return r.nconv >= nev ? MOMED_OK : MOMED_ENOTCONV;
}
