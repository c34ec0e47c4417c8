// eig_dense.cu -- FP64 eigensolver for the final N x N Hamiltonian (lowest K levels).
//
// Replaces diag3d -> diag -> dsyev('V','L') of the reference (:2661-2764, :2638-2659) for
// the plain FP64 path. Same structure as the batched solver (Householder reduction,
// bisection, inverse iteration, back-transformation) but spread over the whole GPU:
//   - the reduction is one cooperative kernel: every CTA owns a slice of rows of the
//     trailing matrix; per column three bounded grid barriers separate the reflector
//     formation, the fused (pending rank-2 update + symmetric product) pass and w;
//   - eigenvalues by multisection: one warp per wanted eigenvalue, 32 Sturm counts per
//     pass, the interval shrinks 33x per pass;
//   - inverse iteration one thread per cluster of close eigenvalues;
//   - back-transformation by the stored reflectors, one warp per 4 eigenvectors.
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "eig_dense.cuh"
#include "tridiag_dev.cuh"

namespace dvr3d {

namespace {

constexpr int kDtThreads = 256;  // 8 warps: lanes = rows, warps = column groups
constexpr int kDtRmax = 8;       // row sub-chunks of 32 per CTA -> trailing size <= G*256

__global__ void __launch_bounds__(kDtThreads) dense_tridiag_kernel(DenseTri t) {
    const int n = t.n;
    const long long ld = t.lda;
    double *A = t.A;
    const int G = gridDim.x, cta = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ double red[32];
    __shared__ double s_part[kDtRmax * 32 * 8];
    __shared__ double s_tau, s_scal, s_beta;
    bool pending = false;
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;                    // trailing rows k+1 .. n-1
        int chunk = (m + G - 1) / G;
        chunk = ((chunk + 31) / 32) * 32;
        const int r0 = k + 1 + cta * chunk;
        const int r1 = min(n, r0 + chunk);
        // (a) finish column k on own rows, partial norm of rows >= k+2
        double ss = 0.0;
        {
            const double vk = pending ? t.vp[k] : 0.0, wk = pending ? t.wp[k] : 0.0;
            if (cta == 0 && tid == 0 && pending) A[(size_t)k * ld + k] -= 2.0 * vk * wk;
            for (int i = r0 + tid; i < r1; i += blockDim.x) {
                double x = A[(size_t)k * ld + i];
                if (pending) {
                    x -= t.vp[i] * wk + t.wp[i] * vk;
                    A[(size_t)k * ld + i] = x;
                }
                if (i >= k + 2) ss += x * x;
            }
        }
        ss = block_sum(ss, red);
        if (tid == 0) t.part[cta] = ss;
        if (!grid_sync(t.bar, t.err)) return;
        // (b) reflector (redundantly in every CTA), fused pass over own rows
        if (tid < 32) {
            double s = 0.0;
            for (int c = tid; c < G; c += 32) s += t.part[c];
            s = warp_sum(s);
            if (tid == 0) {
                const double alpha = A[(size_t)k * ld + k + 1];
                if (s == 0.0) {
                    s_tau = 0.0;
                    s_beta = alpha;
                    s_scal = 0.0;
                } else {
                    const double beta = -copysign(sqrt(alpha * alpha + s), alpha);
                    s_tau = (beta - alpha) / beta;
                    s_beta = beta;
                    s_scal = 1.0 / (alpha - beta);
                }
                if (cta == 0) {
                    t.d[k] = A[(size_t)k * ld + k];
                    t.e[k] = s_beta;
                    t.tau[k] = s_tau;
                    t.scal[k] = s_scal;
                }
            }
        }
        __syncthreads();
        const double tk = s_tau, scal = s_scal;
        const int nsub = (r1 > r0) ? (r1 - r0 + 31) / 32 : 0;
        double acc[kDtRmax];
        double vpi[kDtRmax], wpi[kDtRmax];
#pragma unroll
        for (int r = 0; r < kDtRmax; ++r) {
            acc[r] = 0.0;
            const int i = r0 + r * 32 + lane;
            vpi[r] = (pending && r < nsub && i < r1) ? t.vp[i] : 0.0;
            wpi[r] = (pending && r < nsub && i < r1) ? t.wp[i] : 0.0;
        }
        if (nsub > 0 && (tk != 0.0 || pending)) {
            for (int j = k + 1 + warp; j < n; j += 8) {
                const double vj = (j == k + 1) ? 1.0 : A[(size_t)k * ld + j] * scal;
                const double vpj = pending ? t.vp[j] : 0.0, wpj = pending ? t.wp[j] : 0.0;
                double *col = A + (size_t)j * ld;
#pragma unroll
                for (int r = 0; r < kDtRmax; ++r) {
                    if (r < nsub) {
                        const int i = r0 + r * 32 + lane;
                        if (i < r1) {
                            double x = col[i];
                            if (pending) {
                                x -= vpi[r] * wpj + wpi[r] * vpj;
                                col[i] = x;
                            }
                            acc[r] += x * vj;
                        }
                    }
                }
            }
        }
        // reduce the 8 column groups
#pragma unroll
        for (int r = 0; r < kDtRmax; ++r)
            if (r < nsub) s_part[(warp * kDtRmax + r) * 32 + lane] = acc[r];
        __syncthreads();
        double pv = 0.0;
        for (int q = tid; q < nsub * 32; q += blockDim.x) {
            const int r = q >> 5, l = q & 31;
            const int i = r0 + q;
            double s = 0.0;
            for (int w = 0; w < 8; ++w) s += s_part[(w * kDtRmax + r) * 32 + l];
            if (i < r1) {
                const double vi = (i == k + 1) ? 1.0 : A[(size_t)k * ld + i] * scal;
                const double p = tk * s;
                t.pbuf[i] = p;
                pv += p * vi;
            }
        }
        pv = block_sum(pv, red);
        if (tid == 0) t.part[G + cta] = pv;
        if (!grid_sync(t.bar, t.err)) return;
        // (c) w = p - (tau/2)(p.v) v on own rows; becomes the pending update
        __shared__ double s_pv;
        if (tid < 32) {
            double s = 0.0;
            for (int c = tid; c < G; c += 32) s += t.part[G + c];
            s = warp_sum(s);
            if (tid == 0) s_pv = s;
        }
        __syncthreads();
        const double alpha2 = -0.5 * tk * s_pv;
        for (int i = r0 + tid; i < r1; i += blockDim.x) {
            const double vi = (i == k + 1) ? 1.0 : A[(size_t)k * ld + i] * scal;
            t.vp[i] = vi;
            t.wp[i] = t.pbuf[i] + alpha2 * vi;
        }
        pending = (tk != 0.0);
        if (!grid_sync(t.bar, t.err)) return;
    }
    if (cta == 0 && tid == 0) {
        if (n == 1) {
            t.d[0] = A[0];
            t.e[0] = 0.0;
            t.tau[0] = 0.0;
            t.scal[0] = 0.0;
            return;
        }
        double a00 = A[(size_t)(n - 2) * ld + (n - 2)];
        double a10 = A[(size_t)(n - 2) * ld + (n - 1)];
        double a11 = A[(size_t)(n - 1) * ld + (n - 1)];
        if (pending) {
            a00 -= 2.0 * t.vp[n - 2] * t.wp[n - 2];
            a10 -= t.vp[n - 1] * t.wp[n - 2] + t.wp[n - 1] * t.vp[n - 2];
            a11 -= 2.0 * t.vp[n - 1] * t.wp[n - 1];
        }
        t.d[n - 2] = a00;
        t.d[n - 1] = a11;
        t.e[n - 2] = a10;
        t.e[n - 1] = 0.0;
        t.tau[n - 2] = 0.0;
        t.tau[n - 1] = 0.0;
        t.scal[n - 2] = 0.0;
        t.scal[n - 1] = 0.0;
    }
}

// Gershgorin bounds, pivmin, e^2 and ||T||_1 (one CTA).
__global__ void tri_bounds_kernel(const double *d, const double *e, int n, double *e2, double *info) {
    __shared__ double smin[256], smax[256], se[256];
    const int tid = threadIdx.x;
    double lo = DBL_MAX, hi = -DBL_MAX, emx = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
        const double em = (i > 0) ? fabs(e[i - 1]) : 0.0, ep = (i < n - 1) ? fabs(e[i]) : 0.0;
        lo = fmin(lo, d[i] - em - ep);
        hi = fmax(hi, d[i] + em + ep);
        if (i < n - 1) {
            e2[i] = e[i] * e[i];
            emx = fmax(emx, e2[i]);
        }
    }
    smin[tid] = lo;
    smax[tid] = hi;
    se[tid] = emx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            smin[tid] = fmin(smin[tid], smin[tid + s]);
            smax[tid] = fmax(smax[tid], smax[tid + s]);
            se[tid] = fmax(se[tid], se[tid + s]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        const double tnorm = fmax(fabs(smin[0]), fabs(smax[0]));
        const double piv = DBL_MIN * fmax(1.0, se[0]);
        info[0] = smin[0] - 2.0 * DBL_EPSILON * tnorm * n - 2.0 * piv;
        info[1] = smax[0] + 2.0 * DBL_EPSILON * tnorm * n + 2.0 * piv;
        info[2] = piv;
        info[3] = fmax(tnorm, DBL_MIN);
    }
}

// Multisection: warp w finds eigenvalue j = w (0-based ascending).
__global__ void multisect_kernel(const double *d, const double *e2, int n, int nev, const double *info,
                                 double *w) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= nev) return;
    const int j = gw;
    double lo = info[0], hi = info[1];
    const double piv = info[2];
    for (int pass = 0; pass < 64; ++pass) {
        if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi))) break;
        const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
        const int c = sturm_count(d, e2, n, x, piv);
        const unsigned bal = __ballot_sync(0xffffffffu, c > j);
        const int l = bal ? (__ffs(bal) - 1) : 32;
        const double xl = __shfl_sync(0xffffffffu, x, l > 0 ? l - 1 : 0);
        const double xh = __shfl_sync(0xffffffffu, x, l < 32 ? l : 31);
        const double nlo = (l == 0) ? lo : xl;
        const double nhi = (l == 32) ? hi : xh;
        if (!(nhi - nlo < hi - lo)) break;  // no progress (interval at rounding level)
        lo = nlo;
        hi = nhi;
    }
    if (lane == 0) w[j] = 0.5 * (lo + hi);
}

// Cluster starts for inverse iteration (single thread; nev is at most a few thousand).
__global__ void clusters_kernel(const double *w, int nev, const double *info, int *cstart, int *ncl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double ortol = 1.0e-6 * info[3];
    int nc = 0;
    cstart[nc++] = 0;
    for (int j = 1; j < nev; ++j)
        if (w[j] - w[j - 1] > ortol) cstart[nc++] = j;
    cstart[nc] = nev;
    *ncl = nc;
}

__global__ void invit_dense_kernel(const double *d, const double *e, int n, const double *w, int nev,
                                   const int *cstart, const int *ncl, const double *info, double *fac,
                                   int T, double *X) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nc = *ncl;
    if (t >= T) return;
    for (int c = t; c < nc; c += T)
        invit_cluster(d, e, n, w, cstart[c], cstart[c + 1], info[3], fac, T, t, X, nev);
}

// Z[:, j] = X[:, j] (interleaved -> column-major), then back-transform by the reflectors.
__global__ void untangle_kernel(const double *X, int n, int nev, double *Z, long long ldz) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * nev) return;
    const int j = (int)(idx / n), i = (int)(idx % n);
    Z[(size_t)j * ldz + i] = X[(size_t)i * nev + j];
}

constexpr int kBtCols = 4;
__global__ void backtransform_kernel(const double *A, long long lda, int n, const double *tau,
                                     const double *scal, double *Z, long long ldz, int nev) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int c0 = gw * kBtCols;
    if (c0 >= nev) return;
    const int nc = min(kBtCols, nev - c0);
    for (int k = n - 3; k >= 0; --k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        const double sk = scal[k];
        const double *col = A + (size_t)k * lda;
        double s[kBtCols] = {0.0, 0.0, 0.0, 0.0};
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double vi = (i == k + 1) ? 1.0 : col[i] * sk;
#pragma unroll
            for (int c = 0; c < kBtCols; ++c)
                if (c < nc) s[c] += vi * Z[(size_t)(c0 + c) * ldz + i];
        }
#pragma unroll
        for (int c = 0; c < kBtCols; ++c) s[c] = warp_sum(s[c]) * tk;
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double vi = (i == k + 1) ? 1.0 : col[i] * sk;
#pragma unroll
            for (int c = 0; c < kBtCols; ++c)
                if (c < nc) Z[(size_t)(c0 + c) * ldz + i] -= s[c] * vi;
        }
    }
}

}  // namespace

int dense_tridiag_grid(int device) {
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dense_tridiag_kernel, kDtThreads, 0);
    if (per < 1) per = 1;
    return nsm;  // one CTA per SM (co-resident by construction)
}

cudaError_t launch_dense_tridiag(DenseTri &t, int grid, cudaStream_t st) {
    void *args[] = {&t};
    return cudaLaunchCooperativeKernel((void *)dense_tridiag_kernel, dim3(grid), dim3(kDtThreads), args, 0, st);
}

void launch_dense_eigvals(const double *d, const double *e, int n, int nev, double *e2, double *info,
                          double *w, cudaStream_t st) {
    tri_bounds_kernel<<<1, 256, 0, st>>>(d, e, n, e2, info);
    const int warps_per_block = 4;
    multisect_kernel<<<(nev + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(
        d, e2, n, nev, info, w);
}

void launch_dense_eigvecs(const double *A, long long lda, int n, const double *d, const double *e,
                          const double *tau, const double *scal, const double *w, int nev,
                          const double *info, int *cstart, int *ncl, double *fac, int T, double *X,
                          double *Z, long long ldz, cudaStream_t st) {
    clusters_kernel<<<1, 32, 0, st>>>(w, nev, info, cstart, ncl);
    invit_dense_kernel<<<(T + 63) / 64, 64, 0, st>>>(d, e, n, w, nev, cstart, ncl, info, fac, T, X);
    const long long tot = (long long)n * nev;
    untangle_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(X, n, nev, Z, ldz);
    const int nwarps = (nev + kBtCols - 1) / kBtCols;
    backtransform_kernel<<<(nwarps + 3) / 4, 128, 0, st>>>(A, lda, n, tau, scal, Z, ldz, nev);
}

}  // namespace dvr3d
