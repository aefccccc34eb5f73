// Dense real symmetric eigensolver for the small Lanczos projected matrix
// (krylovdim x krylovdim, FP64, on the host).
//
// Method: Householder reduction to tridiagonal form with the orthogonal factor
// accumulated, then the implicitly shifted QL iteration (Wilkinson-type shift)
// on the tridiagonal matrix, rotating the accumulated factor along.  Both are
// textbook algorithms (Householder 1958; Bowdler, Martin, Reinsch & Wilkinson
// 1968); this is an independent implementation of them.
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <vector>

#include "momed_internal.cuh"

namespace momed {

namespace {

// Implicitly shifted QL on the symmetric tridiagonal (d, e), e[i] coupling d[i] and d[i+1];
// the rotations are applied to the columns of Q (row-major n x n).  d ends as the eigenvalues.
void tridiag_ql(int n, std::vector<double>& d, std::vector<double>& e, double* Q) {
    // implicit QL on (d, e); e[i] couples d[i] and d[i+1]
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        for (int iter = 0; iter < 60; ++iter) {
            int m = l;
            for (; m + 1 < n; ++m) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m == l) break;
            // shift from the leading 2x2 block
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, pshift = 0.0;
            int i;
            bool deflated = false;
            for (i = m - 1; i >= l; --i) {
                double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= pshift;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - pshift;
                r = (d[i] - g) * s + 2.0 * c * b;
                pshift = s * r;
                d[i + 1] = g + pshift;
                g = c * r - b;
                for (int k = 0; k < n; ++k) {
                    double qi1 = Q[(size_t)k * n + i + 1], qi = Q[(size_t)k * n + i];
                    Q[(size_t)k * n + i + 1] = s * qi + c * qi1;
                    Q[(size_t)k * n + i] = c * qi - s * qi1;
                }
            }
            if (deflated) continue;
            d[l] -= pshift;
            e[l] = g;
            e[m] = 0.0;
        }
    }

}

}  // namespace

void symeig(int n, double* A, double* w, double* V) {
    if (n <= 0) return;
    // Q accumulates the Householder reflections; A is reduced in place.
    std::vector<double> Q((size_t)n * n, 0.0), v(n), p(n), q(n);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
    auto a = [&](int r, int c) -> double& { return A[(size_t)r * n + c]; };

    for (int k = 0; k + 2 < n; ++k) {
        // reflect x = A[k+1:n, k] onto a multiple of e_{k+1}
        double xnorm = 0.0;
        for (int i = k + 1; i < n; ++i) xnorm += a(i, k) * a(i, k);
        xnorm = std::sqrt(xnorm);
        if (xnorm == 0.0) continue;
        double alpha = a(k + 1, k) > 0 ? -xnorm : xnorm;
        double vnorm2 = 0.0;
        for (int i = k + 1; i < n; ++i) {
            v[i] = a(i, k) - (i == k + 1 ? alpha : 0.0);
            vnorm2 += v[i] * v[i];
        }
        if (vnorm2 == 0.0) continue;
        double inv = 1.0 / std::sqrt(vnorm2);
        for (int i = k + 1; i < n; ++i) v[i] *= inv;
        // trailing block: B <- (I - 2vv^T) B (I - 2vv^T) = B - 2 v q^T - 2 q v^T
        for (int i = k + 1; i < n; ++i) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += a(i, j) * v[j];
            p[i] = s;
        }
        double K = 0.0;
        for (int i = k + 1; i < n; ++i) K += v[i] * p[i];
        for (int i = k + 1; i < n; ++i) q[i] = p[i] - K * v[i];
        for (int i = k + 1; i < n; ++i)
            for (int j = k + 1; j < n; ++j) a(i, j) -= 2.0 * (v[i] * q[j] + q[i] * v[j]);
        a(k + 1, k) = alpha;
        a(k, k + 1) = alpha;
        for (int i = k + 2; i < n; ++i) { a(i, k) = 0.0; a(k, i) = 0.0; }
        // Q <- Q (I - 2 v v^T)
        for (int r = 0; r < n; ++r) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += Q[(size_t)r * n + j] * v[j];
            s *= 2.0;
            for (int j = k + 1; j < n; ++j) Q[(size_t)r * n + j] -= s * v[j];
        }
    }

    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = a(i, i);
    for (int i = 0; i + 1 < n; ++i) e[i] = a(i + 1, i);
    tridiag_ql(n, d, e, Q.data());

    // ascending order
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int x, int y) { return d[x] < d[y]; });
    for (int c = 0; c < n; ++c) {
        w[c] = d[ord[c]];
        for (int r = 0; r < n; ++r) V[(size_t)r * n + c] = Q[(size_t)r * n + ord[c]];
    }
}

// Dense Hermitian eigensolver (host, FP64) for the block Lanczos projected matrix: complex
// Householder reduction to a Hermitian tridiagonal matrix with the unitary factor accumulated,
// a diagonal phase scaling that makes the off-diagonal real, then the same QL iteration.
// A: n x n row-major (destroyed); w ascending; Z: eigenvectors as columns (row-major n x n).
void herm_eig(int n, std::complex<double>* A, double* w, std::complex<double>* Z) {
    using cd = std::complex<double>;
    if (n <= 0) return;
    auto a = [&](int r, int c) -> cd& { return A[(size_t)r * n + c]; };
    std::vector<cd> Q((size_t)n * n, 0.0), v(n), p(n), q(n);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
    for (int k = 0; k + 2 < n; ++k) {
        double sigma = 0.0;
        for (int i = k + 1; i < n; ++i) sigma += std::norm(a(i, k));
        sigma = std::sqrt(sigma);
        if (sigma == 0.0) continue;
        const cd x0 = a(k + 1, k);
        const cd phase = std::abs(x0) > 0.0 ? x0 / std::abs(x0) : cd(1.0, 0.0);
        const cd alpha = -phase * sigma;
        double vv = 0.0;
        for (int i = k + 1; i < n; ++i) {
            v[i] = a(i, k);
            if (i == k + 1) v[i] -= alpha;
            vv += std::norm(v[i]);
        }
        if (vv == 0.0) continue;
        const double tau = 2.0 / vv;
        // A22 <- H A22 H with H = I - tau v v^H: p = tau A22 v, K = tau/2 v^H p, q = p - K v
        for (int i = k + 1; i < n; ++i) {
            cd s = 0.0;
            for (int j = k + 1; j < n; ++j) s += a(i, j) * v[j];
            p[i] = tau * s;
        }
        cd K = 0.0;
        for (int i = k + 1; i < n; ++i) K += std::conj(v[i]) * p[i];
        K *= 0.5 * tau;
        for (int i = k + 1; i < n; ++i) q[i] = p[i] - K * v[i];
        for (int i = k + 1; i < n; ++i)
            for (int j = k + 1; j < n; ++j) a(i, j) -= v[i] * std::conj(q[j]) + q[i] * std::conj(v[j]);
        a(k + 1, k) = alpha;
        a(k, k + 1) = std::conj(alpha);
        for (int i = k + 2; i < n; ++i) { a(i, k) = 0.0; a(k, i) = 0.0; }
        // Q <- Q H
        for (int r = 0; r < n; ++r) {
            cd s = 0.0;
            for (int j = k + 1; j < n; ++j) s += Q[(size_t)r * n + j] * v[j];
            s *= tau;
            for (int j = k + 1; j < n; ++j) Q[(size_t)r * n + j] -= s * std::conj(v[j]);
        }
    }
    // phases delta_{i+1} = delta_i beta_i / |beta_i| make the subdiagonal real and non-negative
    std::vector<cd> delta(n, cd(1.0, 0.0));
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = a(i, i).real();
    for (int i = 0; i + 1 < n; ++i) {
        const cd b = a(i + 1, i);
        const double mb = std::abs(b);
        e[i] = mb;
        delta[i + 1] = mb > 0.0 ? delta[i] * (b / mb) : delta[i];
    }
    std::vector<double> P((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) P[(size_t)i * n + i] = 1.0;
    tridiag_ql(n, d, e, P.data());
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int x, int y) { return d[x] < d[y]; });
    // Z = Q diag(delta) P
    for (int c = 0; c < n; ++c) {
        w[c] = d[ord[c]];
        for (int r = 0; r < n; ++r) {
            cd s = 0.0;
            for (int j = 0; j < n; ++j) s += Q[(size_t)r * n + j] * delta[j] * P[(size_t)j * n + ord[c]];
            Z[(size_t)r * n + c] = s;
        }
    }
}

}  // namespace momed
