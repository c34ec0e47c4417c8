// band_bisect.cu -- lowest eigenpairs of a symmetric band matrix without reducing it:
// Sturm-count bisection on LDL^T factorisations of A - sigma I and inverse iteration with the
// same factorisation.
//
// For a symmetric A and a shift sigma that is not an eigenvalue, the number of negative pivots
// of A - sigma I = L D L^T (no pivoting) is the number of eigenvalues below sigma (Sylvester's
// law of inertia). With half-bandwidth b the factorisation touches a (b+1) x (b+1) window that
// slides down the diagonal, O(n b^2) per count; one warp works one count, lane t holding row
// k+1+t of the window at step k (the window in shared memory, rows and columns circular
// modulo b+1; the row entering at k+b+1 is still the original A).
//
//   * band_gersh_kernel: Gershgorin bounds and max |A|.
//   * band_bisect_kernel: one warp per wanted eigenvalue j (ascending), bisection on the
//     count to the rounding level of the bounds.
//   * band_invit_kernel: one warp per cluster of eigenvalues closer than `ctol`; per member,
//     the LDL^T factors of A - lambda I (L to global scratch), three inverse-iteration passes
//     from a deterministic start vector, modified Gram-Schmidt against the cluster's earlier
//     vectors, normalisation; the growth of the last pass below `gmin` sets the error flag.
// The projected matrices this serves (shift-invert Krylov, block size = b) keep their wanted
// eigenvalues far apart relative to the rounding of the factorisation; the FP64 Rayleigh-Ritz
// check of the caller judges the vectors.
#include <cfloat>
#include <cmath>

#include "band_eig.cuh"
#include "common.cuh"

namespace dvr3d {

namespace {

constexpr int kBisWarps = 4;  // warps per CTA
constexpr int kWin = kBandMaxBw + 1;

// A(i, j) of the lower band (i >= j), column-major
__device__ __forceinline__ double aband(const double *A, long long lda, int i, int j) { return A[(size_t)j * lda + i]; }

__global__ void band_gersh_kernel(const double *A, long long lda, int n, int b, double *out) {
    __shared__ double rlo[32], rhi[32], rmx[32];
    double lo = DBL_MAX, hi = -DBL_MAX, mx = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        const int j0 = i - b < 0 ? 0 : i - b, j1 = i + b >= n ? n - 1 : i + b;
        for (int j = j0; j <= j1; ++j) {
            if (j == i) continue;
            const double v = j < i ? aband(A, lda, i, j) : aband(A, lda, j, i);
            s += fabs(v);
            mx = fmax(mx, fabs(v));
        }
        const double d = aband(A, lda, i, i);
        mx = fmax(mx, fabs(d));
        lo = fmin(lo, d - s);
        hi = fmax(hi, d + s);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        rlo[wid] = lo;
        rhi[wid] = hi;
        rmx[wid] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = fmin(lo, rlo[w]);
            hi = fmax(hi, rhi[w]);
            mx = fmax(mx, rmx[w]);
        }
        out[0] = lo;
        out[1] = hi;
        out[2] = mx;
    }
}

// One LDL^T sweep of A - sigma I by a warp (window S: kWin x kWin, circular). Returns the number
// of negative pivots (all lanes). With L / D non-null the factors are stored: L[k * b + t] =
// l(k+1+t, k), D[k] = d(k).
__device__ int ldlt_sweep(const double *A, long long lda, int n, int b, double sigma, double tiny, double *S,
                          double *L, double *D) {
    const int lane = threadIdx.x & 31;
    const int W = b + 1;
    auto at = [&](int r, int c) -> double & { return S[(r % W) * kWin + (c % W)]; };
    // rows 0 .. b: lower band
    for (int r = 0; r < W && r < n; ++r)
        for (int c = lane; c <= r; c += 32) at(r, c) = aband(A, lda, r, c) - (r == c ? sigma : 0.0);
    __syncwarp();
    int neg = 0;
    for (int k = 0; k < n; ++k) {
        double d = at(k, k);
        if (fabs(d) < tiny) d = d < 0.0 ? -tiny : tiny;
        neg += (d < 0.0);
        if (D && lane == 0) D[k] = d;
        const int r = k + 1 + lane;
        if (lane < b && r < n) {
            const double l = at(r, k) / d;
            if (L) L[(size_t)k * b + lane] = l;
            // S(r, c) -= l * S(c, k) for c = k+1 .. r
            for (int c = k + 1; c <= r; ++c) at(r, c) -= l * at(c, k);
        }
        __syncwarp();
        // the row entering the window: k + b + 1, columns k+1 .. k+b+1 (original A)
        const int rn = k + W;
        if (rn < n) {
            for (int c = k + 1 + lane; c <= rn; c += 32) at(rn, c) = aband(A, lda, rn, c) - (rn == c ? sigma : 0.0);
        }
        __syncwarp();
    }
    return neg;
}

__global__ void __launch_bounds__(32 * kBisWarps) band_bisect_kernel(const double *A, long long lda, int n, int b,
                                                                    int nev, const double *bounds, double *w) {
    __shared__ double win[kBisWarps][kWin * kWin];
    const int wid = threadIdx.x >> 5;
    const int j = blockIdx.x * kBisWarps + wid;
    if (j >= nev) return;
    double lo = bounds[0], hi = bounds[1];
    const double anorm = fmax(bounds[2], DBL_MIN);
    const double tiny = DBL_EPSILON * anorm;
    const double span = fmax(fabs(lo), fabs(hi));
    lo -= 2.0 * DBL_EPSILON * span + tiny;
    hi += 2.0 * DBL_EPSILON * span + tiny;
    for (int it = 0; it < 100; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (!(hi - lo > 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 2.0 * DBL_MIN) || mid == lo || mid == hi) break;
        const int cnt = ldlt_sweep(A, lda, n, b, mid, tiny, win[wid], nullptr, nullptr);
        if (cnt > j) hi = mid;
        else lo = mid;
    }
    if ((threadIdx.x & 31) == 0) w[j] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// y <- (L D L^T)^-1 y, y in global (length n)
__device__ void ldlt_solve(const double *L, const double *D, int n, int b, double *y) {
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < n; ++k) {  // L z = y
        const double yk = y[k];
        __syncwarp();
        const int r = k + 1 + lane;
        if (lane < b && r < n) y[r] -= L[(size_t)k * b + lane] * yk;
        __syncwarp();
    }
    for (int k = lane; k < n; k += 32) y[k] /= D[k];
    __syncwarp();
    for (int k = n - 1; k >= 0; --k) {  // L^T x = z
        const int r = k + 1 + lane;
        double s = (lane < b && r < n) ? L[(size_t)k * b + lane] * y[r] : 0.0;
        s = warp_sum_d(s);
        if (lane == 0) y[k] -= s;
        __syncwarp();
    }
}

__global__ void __launch_bounds__(32 * kBisWarps) band_invit_kernel(const double *A, long long lda, int n, int b,
                                                                   const double *w, const int *cstart, int ncl,
                                                                   const double *bounds, double *Lscr, double *Dscr,
                                                                   double *Z, long long ldz, double gmin, int *err) {
    __shared__ double win[kBisWarps][kWin * kWin];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cl = blockIdx.x * kBisWarps + wid;
    if (cl >= ncl) return;
    const double anorm = fmax(bounds[2], DBL_MIN);
    const double tiny = DBL_EPSILON * anorm;
    double *L = Lscr + (size_t)cl * n * b;
    double *D = Dscr + (size_t)cl * n;
    const int j0 = cstart[cl], j1 = cstart[cl + 1];
    for (int j = j0; j < j1; ++j) {
        // members of a cluster get shifts apart by a few rounding units so that their
        // factorisations differ; Gram-Schmidt keeps the vectors apart
        const double lam = w[j] + (double)(j - j0) * 4.0 * DBL_EPSILON * anorm;
        ldlt_sweep(A, lda, n, b, lam, tiny, win[wid], L, D);
        __syncwarp();
        double *y = Z + (size_t)j * ldz;
        for (int i = lane; i < n; i += 32) {
            unsigned x = (unsigned)i * 2654435761u ^ (0x9e3779b9u + 7919u * (unsigned)j);
            x ^= x >> 16;
            x *= 0x7feb352dU;
            x ^= x >> 15;
            x *= 0x846ca68bU;
            x ^= x >> 16;
            y[i] = (double)(x & 0xffffff) / 8388608.0 - 1.0;
        }
        __syncwarp();
        double g = 0.0;
        for (int pass = 0; pass < 3; ++pass) {
            ldlt_solve(L, D, n, b, y);
            // Gram-Schmidt against the cluster's earlier vectors
            for (int q = j0; q < j; ++q) {
                const double *zq = Z + (size_t)q * ldz;
                double s = 0.0;
                for (int i = lane; i < n; i += 32) s += zq[i] * y[i];
                s = warp_sum_d(s);
                for (int i = lane; i < n; i += 32) y[i] -= s * zq[i];
                __syncwarp();
            }
            double s = 0.0;
            for (int i = lane; i < n; i += 32) s += y[i] * y[i];
            s = warp_sum_d(s);
            g = sqrt(s);
            const double inv = g > 0.0 ? 1.0 / g : 0.0;
            for (int i = lane; i < n; i += 32) y[i] *= inv;
            __syncwarp();
        }
        if (lane == 0 && !(g >= gmin)) atomicExch(err, 1);
    }
}

}  // namespace

size_t band_bisect_scratch_doubles(int n, int b, int nclusters) {
    return (size_t)nclusters * n * (size_t)b + (size_t)nclusters * n + 4;
}

cudaError_t launch_band_bounds(const double *A, long long lda, int n, int b, double *bounds, cudaStream_t st) {
    if (n < 1 || b < 1 || b > kBandMaxBw) return cudaErrorInvalidValue;
    DVR3D_COUNT_LAUNCH(1);
    band_gersh_kernel<<<1, 1024, 0, st>>>(A, lda, n, b, bounds);
    return cudaGetLastError();
}

cudaError_t launch_band_bisect(const double *A, long long lda, int n, int b, int nev, const double *bounds, double *w,
                               cudaStream_t st) {
    if (n < 1 || b < 1 || b > kBandMaxBw || nev < 1 || nev > n) return cudaErrorInvalidValue;
    DVR3D_COUNT_LAUNCH(1);
    band_bisect_kernel<<<(nev + kBisWarps - 1) / kBisWarps, 32 * kBisWarps, 0, st>>>(A, lda, n, b, nev, bounds, w);
    return cudaGetLastError();
}

cudaError_t launch_band_invit(const double *A, long long lda, int n, int b, const double *w, const int *cstart, int ncl,
                              const double *bounds, double *scratch, double *Z, long long ldz, double gmin, int *err,
                              cudaStream_t st) {
    if (n < 1 || b < 1 || b > kBandMaxBw || ncl < 1) return cudaErrorInvalidValue;
    double *Ls = scratch, *Ds = scratch + (size_t)ncl * n * b;
    DVR3D_COUNT_LAUNCH(1);
    band_invit_kernel<<<(ncl + kBisWarps - 1) / kBisWarps, 32 * kBisWarps, 0, st>>>(A, lda, n, b, w, cstart, ncl, bounds,
                                                                                  Ls, Ds, Z, ldz, gmin, err);
    return cudaGetLastError();
}

}  // namespace dvr3d
