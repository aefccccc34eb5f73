// Complex Schur decomposition of the small Arnoldi projected matrix (host, FP64), for the
// non-Hermitian eigensolver (arnoldi.cu).
//
// A general complex n x n matrix A is reduced to upper Hessenberg form by Householder
// reflections, then to upper triangular (Schur) form T = Z^H A Z by the shifted QR iteration
// (Wilkinson shift from the trailing 2 x 2 block, Givens rotations, deflation on negligible
// subdiagonal entries).  schur_reorder moves chosen eigenvalues to the leading diagonal
// positions by swapping neighbours with one rotation each (the standard exchange of two 1 x 1
// blocks), which is the Krylov-Schur restart; tri_eigvecs solves (T - t_ii) y = 0 by back
// substitution.  Textbook algorithms (Francis 1961; Golub & Van Loan, ch. 7); this is an
// independent implementation.
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <vector>

#include "momed_internal.cuh"

namespace momed {

using cd = std::complex<double>;

namespace {

// Givens rotation [c s; -conj(s) c] (c real) with [c s; -conj(s) c]^H ... chosen so that
// G [a; b] = [r; 0]:  c = |a| / h, s = (a / |a|) conj(b) / h, h = hypot(|a|, |b|)
void givens(cd a, cd b, double& c, cd& s) {
    const double aa = std::abs(a), bb = std::abs(b);
    if (bb == 0.0) { c = 1.0; s = 0.0; return; }
    if (aa == 0.0) { c = 0.0; s = std::conj(b) / bb; return; }
    const double h = std::hypot(aa, bb);
    c = aa / h;
    s = (a / aa) * std::conj(b) / h;
}

// rows (p, q) of M (n columns, row-major) <- G rows: [c s; -conj(s) c]
void rot_rows(std::vector<cd>& M, int n, int p, int q, double c, cd s, int c0 = 0) {
    for (int j = c0; j < n; ++j) {
        const cd x = M[(size_t)p * n + j], y = M[(size_t)q * n + j];
        M[(size_t)p * n + j] = c * x + s * y;
        M[(size_t)q * n + j] = -std::conj(s) * x + c * y;
    }
}
// columns (p, q) of M (rows [r0, r1)) <- M G^H
void rot_cols(std::vector<cd>& M, int n, int p, int q, double c, cd s, int r0, int r1) {
    for (int i = r0; i < r1; ++i) {
        const cd x = M[(size_t)i * n + p], y = M[(size_t)i * n + q];
        M[(size_t)i * n + p] = c * x + std::conj(s) * y;
        M[(size_t)i * n + q] = -s * x + c * y;
    }
}

}  // namespace

// A (n x n row-major) -> T upper triangular in place, Z unitary with A_in = Z T Z^H.
// Returns false if the QR iteration did not converge (30 n iterations).
bool schur_complex(int n, std::vector<cd>& A, std::vector<cd>& Z) {
    Z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Z[(size_t)i * n + i] = 1.0;
    if (n <= 1) return true;
    auto a = [&](int r, int c) -> cd& { return A[(size_t)r * n + c]; };
    // Householder reduction to Hessenberg form
    std::vector<cd> v(n);
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
            v[i] = a(i, k) - (i == k + 1 ? alpha : cd(0.0));
            vv += std::norm(v[i]);
        }
        if (vv == 0.0) continue;
        const double tau = 2.0 / vv;
        // A <- (I - tau v v^H) A
        for (int j = 0; j < n; ++j) {
            cd s = 0.0;
            for (int i = k + 1; i < n; ++i) s += std::conj(v[i]) * a(i, j);
            s *= tau;
            for (int i = k + 1; i < n; ++i) a(i, j) -= v[i] * s;
        }
        // A <- A (I - tau v v^H),  Z <- Z (I - tau v v^H)
        for (int r = 0; r < n; ++r) {
            cd s = 0.0, z = 0.0;
            for (int j = k + 1; j < n; ++j) { s += a(r, j) * v[j]; z += Z[(size_t)r * n + j] * v[j]; }
            s *= tau;
            z *= tau;
            for (int j = k + 1; j < n; ++j) {
                a(r, j) -= s * std::conj(v[j]);
                Z[(size_t)r * n + j] -= z * std::conj(v[j]);
            }
        }
        for (int i = k + 2; i < n; ++i) a(i, k) = 0.0;
    }
    // shifted QR on the active window [lo, hi]
    const double eps = std::numeric_limits<double>::epsilon();
    int hi = n - 1, iter = 0;
    while (hi > 0) {
        if (iter > 30 * n) return false;
        int lo = hi;
        while (lo > 0) {
            const double s = std::abs(a(lo - 1, lo - 1)) + std::abs(a(lo, lo));
            if (std::abs(a(lo, lo - 1)) <= eps * (s > 0.0 ? s : 1.0)) { a(lo, lo - 1) = 0.0; break; }
            --lo;
        }
        if (lo == hi) { --hi; iter = 0; continue; }
        ++iter;
        // Wilkinson shift: eigenvalue of the trailing 2 x 2 nearer to a(hi, hi)
        const cd p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), t = a(hi, hi);
        const cd tr = p + t, det = p * t - q * r;
        const cd disc = std::sqrt(tr * tr - 4.0 * det);
        const cd l1 = 0.5 * (tr + disc), l2 = 0.5 * (tr - disc);
        cd mu = std::abs(l1 - t) < std::abs(l2 - t) ? l1 : l2;
        if (iter % 11 == 10) mu = t + cd(std::abs(a(hi, hi - 1)), 0.0);   // exceptional shift
        // QR step on the window: rotations that triangularise (H - mu I), applied as H <- G H G^H
        std::vector<double> cs(hi - lo);
        std::vector<cd> ss(hi - lo);
        for (int k = lo; k < hi; ++k) {
            cd x = (k == lo) ? a(k, k) - mu : a(k, k - 1);
            cd y = (k == lo) ? a(k + 1, k) : a(k + 1, k - 1);
            double c;
            cd s;
            givens(x, y, c, s);
            // rows k, k+1 from column max(lo, k-1)
            rot_rows(A, n, k, k + 1, c, s, k == lo ? lo : k - 1);
            if (k > lo) a(k + 1, k - 1) = 0.0;
            // columns k, k+1 over rows [0, min(k+2, hi)]
            rot_cols(A, n, k, k + 1, c, s, 0, std::min(k + 3, hi + 1));
            rot_cols(Z, n, k, k + 1, c, s, 0, n);
            // the bulge (k+2, k) is chased by the next rotation
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) a(i, j) = 0.0;
    return true;
}

// Reorder the Schur form so that the diagonal entries with order[] (a permutation of 0..n-1,
// listed in the wanted order) come first: repeated swaps of neighbouring 1 x 1 blocks.
void schur_reorder(int n, std::vector<cd>& T, std::vector<cd>& Z, const std::vector<int>& order) {
    // position of each original diagonal entry as it moves
    std::vector<int> pos(n);
    for (int i = 0; i < n; ++i) pos[i] = i;
    std::vector<int> at(n);   // at[p] = original index now at position p
    for (int i = 0; i < n; ++i) at[i] = i;
    for (int target = 0; target < n; ++target) {
        int p = pos[order[target]];
        while (p > target) {
            // swap diagonal entries p-1 and p
            const int k = p - 1;
            const cd t11 = T[(size_t)k * n + k], t22 = T[(size_t)(k + 1) * n + k + 1], t12 = T[(size_t)k * n + k + 1];
            // rotation G with G [t12; t22 - t11] = [*; 0] makes the swap
            double c;
            cd s;
            givens(t12, t22 - t11, c, s);
            rot_rows(T, n, k, k + 1, c, s, k);
            rot_cols(T, n, k, k + 1, c, s, 0, k + 2);
            rot_cols(Z, n, k, k + 1, c, s, 0, n);
            T[(size_t)(k + 1) * n + k] = 0.0;
            T[(size_t)k * n + k] = t22;
            T[(size_t)(k + 1) * n + k + 1] = t11;
            const int a = at[k], b = at[k + 1];
            at[k] = b;
            at[k + 1] = a;
            pos[a] = k + 1;
            pos[b] = k;
            --p;
        }
    }
}

// eigenvectors of upper triangular T: column i solves (T - t_ii) y = 0 with y_i = 1, y_j = 0
// for j > i; normalised to unit 2-norm.  Y row-major n x n.
void tri_eigvecs(int n, const std::vector<cd>& T, std::vector<cd>& Y) {
    Y.assign((size_t)n * n, 0.0);
    double tmax = 0.0;
    for (int i = 0; i < n; ++i) tmax = std::max(tmax, std::abs(T[(size_t)i * n + i]));
    const double small = std::max(tmax, 1e-300) * std::numeric_limits<double>::epsilon();
    for (int i = 0; i < n; ++i) {
        const cd lam = T[(size_t)i * n + i];
        Y[(size_t)i * n + i] = 1.0;
        for (int r = i - 1; r >= 0; --r) {
            cd s = 0.0;
            for (int p = r + 1; p <= i; ++p) s += T[(size_t)r * n + p] * Y[(size_t)p * n + i];
            cd d = T[(size_t)r * n + r] - lam;
            if (std::abs(d) < small) d = small;
            Y[(size_t)r * n + i] = -s / d;
        }
        double nn = 0.0;
        for (int r = 0; r <= i; ++r) nn += std::norm(Y[(size_t)r * n + i]);
        nn = std::sqrt(nn);
        for (int r = 0; r <= i; ++r) Y[(size_t)r * n + i] /= nn;
    }
}

}  // namespace momed
