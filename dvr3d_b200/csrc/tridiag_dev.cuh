// tridiag_dev.cuh -- device routines on a symmetric tridiagonal matrix T (diag d,
// off-diagonal e): Sturm counts for bisection and inverse iteration for eigenvectors, in
// the manner of LAPACK dstebz / dstein, as used after the Householder reductions.
#pragma once

#include <cfloat>
#include <cmath>

namespace dvr3d {

// ------------------------------------------------------------------ Sturm bisection
// Number of eigenvalues of T (diag d, squared off-diagonals e2) strictly below x.
static __device__ __forceinline__ int sturm_count(const double *d, const double *e2, int n, double x,
                                           double pivmin) {
    int c = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    c += (q < 0.0);
    for (int i = 1; i < n; ++i) {
        q = (d[i] - x) - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        c += (q < 0.0);
    }
    return c;
}

// Eigenvalue j (0-based, ascending) by bisection on [lo, hi].
static __device__ __forceinline__ double bisect_one(const double *d, const double *e2, int n, int j, double lo, double hi,
                             double pivmin) {
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (!(mid > lo && mid < hi)) break;
        if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi))) break;
        if (sturm_count(d, e2, n, mid, pivmin) > j) hi = mid;
        else lo = mid;
    }
    return 0.5 * (lo + hi);
}

static __device__ __forceinline__ unsigned hash32(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Convergence test of one inverse-iteration pass, as dstein applies it: with the right-hand
// side scaled to 1-norm n ||T||_1 max(eps, |u_nn|), the solve has converged when the largest
// component of the (orthogonalised) solution reaches sqrt(0.1 / n). A vector is accepted when
// at least kInvitGrowPasses of the kInvitPasses passes grew that much; otherwise the kernel
// raises its error flag (non-convergence, reported to the host as DVR3D_ERR_NOCONV).
constexpr int kInvitPasses = 4;
constexpr int kInvitGrowPasses = 2;
static __device__ __forceinline__ double invit_growth_limit(int n) { return sqrt(0.1 / (double)n); }

// One thread: eigenvectors of the cluster [j0, j1) of T. Factor arrays interleaved with
// stride T (thread slots), vectors interleaved with stride nsel (eigenvalue slots). A vector
// that fails the growth test sets *err = kDevNoConv (when err is not null).
static __device__ __noinline__ void invit_cluster(const double *d, const double *e, int n, const double *w, int j0,
                              int j1, double onenrm, double *fac, int T, int t, double *X,
                              int nsel, int *err) {
    double *D = fac, *E1 = fac + (size_t)n * T, *E2 = fac + 2 * (size_t)n * T;
    double *Lm = fac + 3 * (size_t)n * T, *P = fac + 4 * (size_t)n * T;
#define F(arr, i) arr[(size_t)(i) * T + t]
#define XV(i, j) X[(size_t)(i) * nsel + (j)]
    const double eps = DBL_EPSILON;
    const double tiny = eps * onenrm;
    const double pertol = 10.0 * eps * onenrm;
    double lamprev = 0.0;
    for (int j = j0; j < j1; ++j) {
        double lam = w[j];
        if (j > j0 && lam - lamprev < pertol) lam = lamprev + pertol;
        lamprev = lam;
        // LU of T - lam I with partial pivoting (U has two superdiagonals)
        double av = d[0] - lam, bv = (n > 1) ? e[0] : 0.0;
        for (int i = 0; i < n - 1; ++i) {
            const double c = e[i];
            const double an = d[i + 1] - lam, bn = (i + 2 < n) ? e[i + 1] : 0.0;
            if (fabs(av) >= fabs(c)) {
                if (av == 0.0) av = tiny;
                const double mlt = c / av;
                F(P, i) = 0.0;
                F(Lm, i) = mlt;
                F(D, i) = av;
                F(E1, i) = bv;
                F(E2, i) = 0.0;
                av = an - mlt * bv;
                bv = bn;
            } else {
                const double mlt = av / c;
                F(P, i) = 1.0;
                F(Lm, i) = mlt;
                F(D, i) = c;
                F(E1, i) = an;
                F(E2, i) = bn;
                av = bv - mlt * an;
                bv = -mlt * bn;
            }
        }
        if (fabs(av) < tiny) av = (av < 0.0) ? -tiny : tiny;
        F(D, n - 1) = av;
        // the last row of U has no superdiagonals; the back substitution reads them (times
        // zero), so they must not hold stale non-finite values
        F(E1, n - 1) = 0.0;
        F(E2, n - 1) = 0.0;
        for (int i = 0; i < n - 1; ++i)
            if (fabs(F(D, i)) < tiny) F(D, i) = (F(D, i) < 0.0) ? -tiny : tiny;
        // deterministic start vector in (-1, 1)
        for (int i = 0; i < n; ++i) {
            const unsigned h = hash32((unsigned)(i * 2654435761u) ^ (unsigned)(j * 40503u + 17u));
            XV(i, j) = ((double)(h & 0xffffff) / 8388608.0) - 1.0;
        }
        const double grow_lim = invit_growth_limit(n);
        int grown = 0;
        for (int it = 0; it < kInvitPasses; ++it) {
            // scale the right-hand side so the solve cannot overflow (as dstein does)
            double s1 = 0.0;
            for (int i = 0; i < n; ++i) s1 += fabs(XV(i, j));
            const double sc = (double)n * onenrm * fmax(eps, fabs(F(D, n - 1))) / fmax(s1, DBL_MIN);
            for (int i = 0; i < n; ++i) XV(i, j) *= sc;
            // forward: P, L
            for (int i = 0; i < n - 1; ++i) {
                double yi = XV(i, j), yn = XV(i + 1, j);
                if (F(P, i) != 0.0) {
                    const double tmp = yi;
                    yi = yn;
                    yn = tmp;
                    XV(i, j) = yi;
                }
                XV(i + 1, j) = yn - F(Lm, i) * yi;
            }
            // backward: U
            double x1 = 0.0, x2 = 0.0;
            for (int i = n - 1; i >= 0; --i) {
                const double xi = (XV(i, j) - F(E1, i) * x1 - F(E2, i) * x2) / F(D, i);
                XV(i, j) = xi;
                x2 = x1;
                x1 = xi;
            }
            // orthogonalise against the earlier members of the cluster (MGS)
            for (int jj = j0; jj < j; ++jj) {
                double dot = 0.0;
                for (int i = 0; i < n; ++i) dot += XV(i, jj) * XV(i, j);
                for (int i = 0; i < n; ++i) XV(i, j) -= dot * XV(i, jj);
            }
            double nrm = 0.0, xinf = 0.0;
            for (int i = 0; i < n; ++i) {
                nrm += XV(i, j) * XV(i, j);
                xinf = fmax(xinf, fabs(XV(i, j)));
            }
            grown += (xinf >= grow_lim);
            nrm = sqrt(nrm);
            const double inv = (nrm > 0.0) ? 1.0 / nrm : 0.0;
            for (int i = 0; i < n; ++i) XV(i, j) *= inv;
        }
        if (grown < kInvitGrowPasses && err) *err = kDevNoConv;
        // sign convention: largest component positive
        double big = 0.0;
        for (int i = 0; i < n; ++i)
            if (fabs(XV(i, j)) > fabs(big)) big = XV(i, j);
        if (big < 0.0)
            for (int i = 0; i < n; ++i) XV(i, j) = -XV(i, j);
    }
#undef F
#undef XV
}


}  // namespace dvr3d
