// tridiag.h — lowest eigenpair of the Lanczos tridiagonal.
//
// Replaces the MKL dstevx('V','A') call of src/lanczos_solver.f90:175-211, of
// which the reference only uses ev(1) and z(:,1) (lanczos_solver.f90:67-68).
// Sturm-sequence bisection to full precision gives the eigenvalue; inverse
// iteration on the LU factors of T - lambda I (partial pivoting) gives the
// eigenvector, normalised with its largest component positive.
#pragma once
#include <cmath>
#include <vector>

namespace edzt {

// d: diagonal a(1:n); e: b(1:n) with e[0] unused (the reference's b(1) = 0),
// off-diagonals e[1..n-1].
inline int lowest_eigenpair(int n, const double* d, const double* e, double* lambda, double* z)
{
    if (n < 1) return -1;
    for (int i = 0; i < n; i++)
        if (!std::isfinite(d[i]) || (i > 0 && !std::isfinite(e[i]))) return -2;
    if (n == 1) {
        *lambda = d[0];
        if (z) z[0] = 1.0;
        return 0;
    }
    const double ulp = 2.220446049250313e-16, tiny = 2.2250738585072014e-308;
    std::vector<double> e2(n, 0.0);
    double lo = d[0], hi = d[0], tn = 0.0, e2max = 0.0;
    for (int i = 0; i < n; i++) {
        const double r = (i > 0 ? std::fabs(e[i]) : 0.0) + (i + 1 < n ? std::fabs(e[i + 1]) : 0.0);
        lo = std::fmin(lo, d[i] - r);
        hi = std::fmax(hi, d[i] + r);
        tn = std::fmax(tn, std::fabs(d[i]) + r);
    }
    for (int i = 1; i < n; i++) {
        e2[i] = e[i] * e[i];
        e2max = std::fmax(e2max, e2[i]);
    }
    const double pivmin = tiny * std::fmax(1.0, e2max);
    lo -= 2.0 * ulp * tn + pivmin;
    hi += 2.0 * ulp * tn + pivmin;
    // count of eigenvalues < x
    auto below = [&](double x) {
        int c = 0;
        double q = d[0] - x;
        if (std::fabs(q) < pivmin) q = -pivmin;
        c += q < 0.0;
        for (int i = 1; i < n; i++) {
            q = d[i] - x - e2[i] / q;
            if (std::fabs(q) < pivmin) q = -pivmin;
            c += q < 0.0;
        }
        return c;
    };
    for (int it = 0; it < 256; it++) {
        const double mid = 0.5 * (lo + hi);
        if (!(mid > lo && mid < hi)) break;
        if (below(mid) >= 1) hi = mid; else lo = mid;
    }
    const double lam = 0.5 * (lo + hi);
    *lambda = lam;
    if (!z) return 0;
    // LU of T - lam I with row interchanges (bands: dl, dd, du, du2)
    std::vector<double> dl(n, 0.0), dd(n), du(n, 0.0), du2(n, 0.0);
    std::vector<char> swp(n, 0);
    for (int i = 0; i < n; i++) dd[i] = d[i] - lam;
    for (int i = 0; i + 1 < n; i++) { du[i] = e[i + 1]; dl[i] = e[i + 1]; }
    const double guard = ulp * tn + pivmin;
    for (int i = 0; i + 1 < n; i++) {
        if (std::fabs(dd[i]) >= std::fabs(dl[i])) {
            if (dd[i] == 0.0) dd[i] = guard;
            const double f = dl[i] / dd[i];
            dl[i] = f;
            dd[i + 1] -= f * du[i];
        } else {
            swp[i] = 1;
            const double f = dd[i] / dl[i];
            dd[i] = dl[i];
            dl[i] = f;
            const double t = du[i];
            du[i] = dd[i + 1];
            dd[i + 1] = t - f * dd[i + 1];
            if (i + 2 < n) { du2[i] = du[i + 1]; du[i + 1] = -f * du[i + 1]; }
        }
    }
    if (dd[n - 1] == 0.0) dd[n - 1] = guard;
    for (int i = 0; i < n; i++) z[i] = 1.0;
    for (int it = 0; it < 3; it++) {
        for (int i = 0; i + 1 < n; i++) {
            if (!swp[i]) z[i + 1] -= dl[i] * z[i];
            else { const double t = z[i]; z[i] = z[i + 1]; z[i + 1] = t - dl[i] * z[i]; }
        }
        z[n - 1] /= dd[n - 1];
        z[n - 2] = (z[n - 2] - du[n - 2] * z[n - 1]) / dd[n - 2];
        for (int i = n - 3; i >= 0; i--) z[i] = (z[i] - du[i] * z[i + 1] - du2[i] * z[i + 2]) / dd[i];
        double nrm = 0.0, big = 0.0;
        for (int i = 0; i < n; i++) {
            nrm += z[i] * z[i];
            if (std::fabs(z[i]) > std::fabs(big)) big = z[i];
        }
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return -3;
        if (big < 0.0) nrm = -nrm;
        for (int i = 0; i < n; i++) z[i] /= nrm;
    }
    return 0;
}

// All eigenpairs of a small dense symmetric matrix by the cyclic Jacobi
// method (Golub & Van Loan, Matrix Computations, §8.5): rotations
// annihilate each off-diagonal element in turn until the off-diagonal part
// is negligible against the diagonal.  A: row-major m x m (overwritten).
// w: eigenvalues ascending; Z: row-major, column i the eigenvector of w[i].
// For the projected matrix of the restarted Lanczos, m <= 8.
inline int symmetric_eig(int m, double* A, double* w, double* Z)
{
    if (m < 1) return -1;
    for (int i = 0; i < m * m; i++)
        if (!std::isfinite(A[i])) return -2;
    std::vector<double> V((size_t)m * m, 0.0);
    for (int i = 0; i < m; i++) V[(size_t)i * m + i] = 1.0;
    auto a = [&](int i, int j) -> double& { return A[(size_t)i * m + j]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; i++) {
            diag += a(i, i) * a(i, i);
            for (int j = i + 1; j < m; j++) off += a(i, j) * a(i, j);
        }
        if (off <= 1e-34 * diag || off == 0.0) break;
        for (int p = 0; p < m; p++)
            for (int q = p + 1; q < m; q++) {
                const double apq = a(p, q);
                if (apq == 0.0) continue;
                const double th = (a(q, q) - a(p, p)) / (2.0 * apq);
                const double t = (th >= 0.0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < m; k++) {            // A = J^T A J
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < m; k++) {
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                a(p, q) = a(q, p) = 0.0;
                for (int k = 0; k < m; k++) {
                    const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
                    V[(size_t)k * m + p] = c * vkp - s * vkq;
                    V[(size_t)k * m + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> order(m);
    for (int i = 0; i < m; i++) order[i] = i;
    for (int i = 1; i < m; i++)                          // insertion sort by eigenvalue
        for (int j = i; j > 0 && a(order[j], order[j]) < a(order[j - 1], order[j - 1]); j--)
            std::swap(order[j], order[j - 1]);
    for (int i = 0; i < m; i++) {
        w[i] = a(order[i], order[i]);
        for (int k = 0; k < m; k++) Z[(size_t)k * m + i] = V[(size_t)k * m + order[i]];
    }
    return 0;
}

}  // namespace edzt
