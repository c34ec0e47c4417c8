// small_syev.cu -- symmetric eigensolver for matrices of dimension <= 160, one CTA per
// matrix, the matrix held in shared memory.
//
// Used where many small problems must be solved with low latency: the Rayleigh-Ritz and
// Gram-matrix problems of the Davidson solver, and small batched blocks. Same method as
// the batched solver (Householder reduction, Sturm bisection, inverse iteration with
// Gram-Schmidt inside clusters, back-transformation), but the reduction runs in shared
// memory with one thread per row, so a 160 x 160 problem takes a fraction of a millisecond.
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "small_syev.cuh"
#include "tridiag_dev.cuh"

namespace dvr3d {

namespace {

constexpr int kSmallThreads = 256;

__global__ void __launch_bounds__(kSmallThreads) small_syev_kernel(SmallSyev p) {
    const int b = blockIdx.x;
    if (b >= p.nmat) return;
    const int n = p.n[b];
    const int ld = n + 1;  // odd stride: conflict-free row and column sweeps
    extern __shared__ double sm[];
    double *S = sm;                       // n x (n+1)
    double *vp = S + (size_t)n * ld;      // pending (v, w) and current v
    double *wp = vp + n;
    double *v = wp + n;
    double *dd = v + n;                   // d, e, e^2, tau
    double *ee = dd + n;
    double *e2 = ee + n;
    double *tau = e2 + n;
    double *wv = tau + n;                 // eigenvalues
    __shared__ double red[32];
    __shared__ double s_tau, s_scal, s_lo, s_hi, s_piv, s_norm;
    const int tid = threadIdx.x;
    const double *A = p.A + p.aoff[b];
    const long long lda = p.lda ? p.lda[b] : n;
    // load (lower triangle, mirrored)
    for (int q = tid; q < n * n; q += blockDim.x) {
        const int i = q % n, j = q / n;
        const double x = (i >= j) ? A[(size_t)j * lda + i] : A[(size_t)i * lda + j];
        S[j * ld + i] = x;
    }
    __syncthreads();
    // ---- Householder reduction with the rank-2 update applied lazily (one thread per row)
    bool pending = false;
    for (int k = 0; k + 2 < n; ++k) {
        if (pending) {
            const double vk = vp[k], wk = wp[k];
            for (int i = k + tid; i < n; i += blockDim.x) S[k * ld + i] -= vp[i] * wk + wp[i] * vk;
        }
        __syncthreads();
        double ss = 0.0;
        for (int i = k + 2 + tid; i < n; i += blockDim.x) ss += S[k * ld + i] * S[k * ld + i];
        ss = block_sum(ss, red);
        if (tid == 0) {
            const double alpha = S[k * ld + k + 1];
            dd[k] = S[k * ld + k];
            if (ss == 0.0) {
                s_tau = 0.0;
                s_scal = 0.0;
                ee[k] = alpha;
            } else {
                const double beta = -copysign(sqrt(alpha * alpha + ss), alpha);
                s_tau = (beta - alpha) / beta;
                s_scal = 1.0 / (alpha - beta);
                ee[k] = beta;
            }
            tau[k] = s_tau;
        }
        __syncthreads();
        const double tk = s_tau, sc = s_scal;
        for (int i = tid; i < n; i += blockDim.x) {
            double vi = 0.0;
            if (i == k + 1) vi = 1.0;
            else if (i > k + 1) {
                vi = S[k * ld + i] * sc;
                S[k * ld + i] = vi;
            }
            v[i] = vi;
        }
        __syncthreads();
        double pvl = 0.0;
        for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            const double vpi = pending ? vp[i] : 0.0, wpi = pending ? wp[i] : 0.0;
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) {
                double x = S[j * ld + i];
                if (pending) {
                    x -= vpi * wp[j] + wpi * vp[j];
                    S[j * ld + i] = x;
                }
                s += x * v[j];
            }
            s *= tk;
            wv[i] = s;  // p_i (temporary)
            pvl += s * v[i];
        }
        const double pv = block_sum(pvl, red);
        const double a2 = -0.5 * tk * pv;
        for (int i = tid; i < n; i += blockDim.x) {
            const double vi = v[i];
            vp[i] = vi;
            wp[i] = (i > k) ? wv[i] + a2 * vi : 0.0;
        }
        pending = (tk != 0.0);
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            double a00 = S[(n - 2) * ld + n - 2], a10 = S[(n - 2) * ld + n - 1], a11 = S[(n - 1) * ld + n - 1];
            if (pending) {
                a00 -= 2.0 * vp[n - 2] * wp[n - 2];
                a10 -= vp[n - 1] * wp[n - 2] + wp[n - 1] * vp[n - 2];
                a11 -= 2.0 * vp[n - 1] * wp[n - 1];
            }
            dd[n - 2] = a00;
            dd[n - 1] = a11;
            ee[n - 2] = a10;
            tau[n - 2] = 0.0;
        } else {
            dd[0] = S[0];
        }
        ee[n - 1] = 0.0;
        tau[n - 1] = 0.0;
    }
    __syncthreads();
    // ---- eigenvalues: bisection, one thread per eigenvalue
    if (tid == 0) {
        double lo = DBL_MAX, hi = -DBL_MAX, emx = 0.0, on = 0.0;
        for (int i = 0; i < n; ++i) {
            const double em = i > 0 ? fabs(ee[i - 1]) : 0.0, ep = i < n - 1 ? fabs(ee[i]) : 0.0;
            lo = fmin(lo, dd[i] - em - ep);
            hi = fmax(hi, dd[i] + em + ep);
            on = fmax(on, fabs(dd[i]) + em + ep);
            if (i < n - 1) {
                e2[i] = ee[i] * ee[i];
                emx = fmax(emx, e2[i]);
            }
        }
        const double tn = fmax(fabs(lo), fabs(hi));
        s_piv = DBL_MIN * fmax(1.0, emx);
        s_lo = lo - 2.0 * DBL_EPSILON * tn * n - 2.0 * s_piv;
        s_hi = hi + 2.0 * DBL_EPSILON * tn * n + 2.0 * s_piv;
        s_norm = fmax(on, DBL_MIN);
    }
    __syncthreads();
    for (int j = tid; j < n; j += blockDim.x) wv[j] = bisect_one(dd, e2, n, j, s_lo, s_hi, s_piv);
    __syncthreads();
    double *W = p.W + p.woff[b];
    for (int j = tid; j < n; j += blockDim.x) W[j] = wv[j];
    if (!p.Z) return;
    // ---- eigenvectors of T: inverse iteration, one thread per cluster (1e-6 ||T|| gaps)
    double *Z = p.Z + p.zoff[b];
    double *fac = p.work + p.workoff[b];  // 5 n T
    double *X = fac + (size_t)5 * n * kSmallThreads;  // n x n interleaved by eigenvalue
    __shared__ int cst[161];
    __shared__ int s_ncl;
    if (tid == 0) {
        const double ortol = 1.0e-6 * s_norm;
        int nc = 0;
        cst[nc++] = 0;
        for (int j = 1; j < n; ++j)
            if (wv[j] - wv[j - 1] > ortol) cst[nc++] = j;
        cst[nc] = n;
        s_ncl = nc;
    }
    __syncthreads();
    const int T = kSmallThreads;
    for (int c = tid; c < s_ncl; c += T) invit_cluster(dd, ee, n, wv, cst[c], cst[c + 1], s_norm, fac, T, tid, X, n, nullptr);
    __syncthreads();
    for (int q = tid; q < n * n; q += blockDim.x) {
        const int j = q / n, i = q % n;
        Z[(size_t)j * n + i] = X[(size_t)i * n + j];
    }
    __syncthreads();
    // ---- back-transformation Z <- H_0 ... H_{n-3} Z, reflectors from shared memory
    const int lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    for (int k = n - 3; k >= 0; --k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        const double *col = S + k * ld;
        for (int c = wid; c < n; c += nw) {
            double *zc = Z + (size_t)c * n;
            double s = 0.0;
            for (int i = k + 1 + lane; i < n; i += 32) s += (i == k + 1 ? 1.0 : col[i]) * zc[i];
            s = warp_sum(s) * tk;
            for (int i = k + 1 + lane; i < n; i += 32) zc[i] -= s * (i == k + 1 ? 1.0 : col[i]);
        }
        __syncthreads();
    }
}

}  // namespace

size_t small_syev_smem(int nmax) { return ((size_t)nmax * (nmax + 1) + 9 * (size_t)nmax) * sizeof(double); }

long long small_syev_work_doubles(int n) { return 5LL * n * kSmallThreads + (long long)n * n; }

cudaError_t launch_small_syev(const SmallSyev &p, int nmax, cudaStream_t st) {
    if (p.nmat <= 0) return cudaSuccess;
    if (nmax > kSmallSyevMax) return cudaErrorInvalidValue;
    const size_t smem = small_syev_smem(nmax);
    int dev = 0;
    cudaGetDevice(&dev);
    static bool attr[kMaxAttrDevices] = {};
    if (dev < 0 || dev >= kMaxAttrDevices || !attr[dev]) {
        // dynamic shared memory of the largest supported problem (static memory comes on top)
        const cudaError_t e = cudaFuncSetAttribute(small_syev_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)small_syev_smem(kSmallSyevMax));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < kMaxAttrDevices) attr[dev] = true;
    }
    DVR3D_COUNT_LAUNCH(1);
    small_syev_kernel<<<p.nmat, kSmallThreads, smem, st>>>(p);
    return cudaGetLastError();
}

}  // namespace dvr3d
